"""Tile counts of nets that share the GPU in a batch, and a measured choice among them.

A net alone takes one window_flat CTA per SM. In a batch, every launch runs every tile of
every net, so the tile count of each net sets both the work per CTA and the number of CTA
waves per launch. The rule here gives net i a share of the SMs by its expected work,

    tiles_i = max(1, round(scale_b * sms * work_i / sum(work))),

with one scale per size bucket b (nets split into buckets by work), and `autotune`
measures scales on the nets themselves (or a sample of them spread over their size range):
first one scale for all, then each bucket's scale in turn with the others held.
`autotune_producers` then chooses, per bucket, how many of window_flat's 32 warps stage and
copy the next steps' arrivals (the rest count and update). Results never depend on the
tiling or the split: only the speed does.
"""
import time

import numpy as np

__all__ = ["layout_work", "tile_targets", "size_buckets", "autotune", "autotune_producers"]


def layout_work(layout):
    """Expected cost of one step of a net: synapses delivered at a nominal rate plus a
    per-neuron update cost, in the units the tiler of the library uses."""
    syn = 0.0
    for s0, s1, d0, d1, p in layout.connections():
        syn += (s1 - s0) * (d1 - d0) * p
    return syn * 0.01 + 1000.0 * layout.size()


def tile_targets(works, sms, scale=1.0, buckets=None):
    """Tiles per net: each net's share of `scale * sms` by work, one at least. `scale` may
    be a list, one per bucket, with buckets[i] the bucket of net i."""
    total = float(sum(works)) or 1.0
    if buckets is None:
        return [max(1, int(round(scale * sms * w / total))) for w in works]
    return [max(1, int(round(scale[b] * sms * w / total))) for w, b in zip(works, buckets)]


def size_buckets(works, count=3):
    """Bucket of each net: equal-sized groups by work, smallest first."""
    order = np.argsort(works, kind="stable")
    out = [0] * len(works)
    for rank, i in enumerate(order):
        out[int(i)] = min(count - 1, rank * count // max(1, len(works)))
    return out


def _sample(works, max_nets):
    if len(works) <= max_nets:
        return list(range(len(works)))
    order = np.argsort(works)
    picks = np.linspace(0, len(works) - 1, max_nets).round().astype(int)
    return sorted(set(int(order[k]) for k in picks))


def _measure(build, idx, targets, w_all, steps, warmup, device, producers=None):
    from . import Batch

    nets = []
    batch = Batch(device=device)
    try:
        for i in idx:
            net = build(i, targets[i])
            if producers is not None:
                net.set_producer_warps(producers[i])
            nets.append(net)
            batch.add(net)
        batch.run(warmup)
        batch.sync()
        t = time.perf_counter()
        batch.run(steps)
        batch.sync()
        return time.perf_counter() - t
    finally:
        batch.close()
        for net in nets:
            net.close()


def autotune(build, works, sms, scales=(0.5, 1.0, 2.0, 4.0), nbuckets=3, steps=150, warmup=30, max_nets=64, device=0):
    """Measure batch runs of the nets under tile scales and return
    (per-bucket scales, buckets of the nets, {description: seconds per step}).

    First every candidate scale for all buckets at once; then, from the best, each bucket's
    scale in turn over the candidates with the other buckets held.

    build(i, tile_target) -> an unstepped Snn equal to net i of the batch (the caller's
    constructor with the tile target passed to Snn.set_tile_target or spk_net_create_ex).
    With more than max_nets nets, a sample spread over their work range is measured, each
    sampled net with the tiles it would get in the full batch, and the sample's time is
    scaled by the whole batch's work over the sample's (an estimate: the sample fills fewer
    SMs than the full batch).
    """
    idx = _sample(works, max_nets)
    buckets = size_buckets(works, nbuckets)
    w_all = float(sum(works)) or 1.0
    w_sub = float(sum(works[i] for i in idx)) or 1.0
    times = {}

    def run(sc):
        key = "/".join(f"{x:g}" for x in sc)
        if key not in times:
            t = _measure(build, idx, tile_targets(works, sms, sc, buckets), w_all, steps, warmup, device)
            times[key] = t / steps * (w_all / w_sub)
        return times[key]

    best = min(([s] * nbuckets for s in scales), key=run)
    for b in range(nbuckets):
        if not any(buckets[i] == b for i in idx):
            continue
        cands = [best[:b] + [s] + best[b + 1:] for s in scales]
        best = min(cands, key=run)
    return best, buckets, times


def autotune_producers(build, works, sms, scale, buckets, producers=(8, 12, 16), steps=150, warmup=30, max_nets=64,
                       device=0):
    """window_flat's producer warps per size bucket, measured on the batch tiled by
    (scale, buckets) as `autotune` chose: each bucket's count in turn over the candidates,
    the other buckets held (at 12, then at their choice). Returns (per-bucket producer warps,
    {description: seconds per step})."""
    idx = _sample(works, max_nets)
    nb = max(buckets) + 1 if buckets else 1
    targets = tile_targets(works, sms, scale, buckets)
    w_all = float(sum(works)) or 1.0
    w_sub = float(sum(works[i] for i in idx)) or 1.0
    times = {}

    def run(pr):
        key = "producers " + "/".join(str(x) for x in pr)
        if key not in times:
            t = _measure(build, idx, targets, w_all, steps, warmup, device, [pr[buckets[i]] for i in range(len(works))])
            times[key] = t / steps * (w_all / w_sub)
        return times[key]

    best = [12] * nb
    for b in range(nb):
        if not any(buckets[i] == b for i in idx):
            continue
        best = min((best[:b] + [x] + best[b + 1:] for x in producers), key=run)
    return best, times
