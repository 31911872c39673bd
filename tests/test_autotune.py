"""The batch autotuner's choices (spice_b200/autotune.py) with the timed batch runs replaced
by a cost model: every candidate measured once, each bucket's best kept, the other buckets
held. No GPU: the search, not the timing, is under test."""
import spice_b200.autotune as at


def fake_measure(cost):
    calls = []

    def measure(build, idx, targets, w_all, steps, warmup, device, producers=None):
        calls.append((tuple(targets[i] for i in idx), None if producers is None else tuple(producers[i] for i in idx)))
        return cost(idx, targets, producers) * steps

    return measure, calls


def test_scales_search_every_candidate_then_each_bucket(monkeypatch):
    works = [1.0, 2.0, 4.0, 8.0, 16.0, 32.0]
    # the best tile count per net depends on its size: small nets want few tiles, large many
    want = {0: 1, 1: 1, 2: 4, 3: 8, 4: 24, 5: 48}

    def cost(idx, targets, producers):
        return sum(abs(targets[i] - want[i]) for i in idx) + 1.0

    measure, calls = fake_measure(cost)
    monkeypatch.setattr(at, "_measure", measure)
    best, buckets, times = at.autotune(None, works, 148, scales=(0.5, 1.0, 2.0, 4.0), nbuckets=3, steps=10, warmup=1)
    assert buckets == [0, 0, 1, 1, 2, 2]
    assert len(best) == 3 and all(s in (0.5, 1.0, 2.0, 4.0) for s in best)
    # every uniform scale was measured, and the result is no worse than any of them
    for s in (0.5, 1.0, 2.0, 4.0):
        assert "/".join([f"{s:g}"] * 3) in times
    key = "/".join(f"{x:g}" for x in best)
    assert times[key] == min(times.values())
    assert len(calls) == len(times)  # each configuration measured once


def test_producer_warps_per_bucket(monkeypatch):
    works = [1.0, 2.0, 10.0, 20.0, 100.0, 200.0]
    buckets = at.size_buckets(works, 3)
    best_for = {0: 8, 1: 12, 2: 16}  # the fastest split of each bucket in the cost model

    def cost(idx, targets, producers):
        return sum(abs(producers[i] - best_for[buckets[i]]) for i in idx) + 1.0

    measure, calls = fake_measure(cost)
    monkeypatch.setattr(at, "_measure", measure)
    prod, times = at.autotune_producers(None, works, 148, [1.0, 1.0, 1.0], buckets, producers=(8, 12, 16), steps=10,
                                        warmup=1)
    assert prod == [8, 12, 16]
    assert all(k.startswith("producers ") for k in times) and len(calls) == len(times)
    # the tiling was held at the given scales while the split varied
    assert len({c[0] for c in calls}) == 1
