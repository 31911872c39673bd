"""The CPU oracle pinned against the reference: golden fixtures produced by the
reference's own cpu::snn (tests/golden/make_golden.py), the reference's known-answer
tests (spice_test/util/layout.cpp, spice_test/util/adj_list.cpp, spice_test/util/random.cpp)
and, where the reference build exists, the reference run live."""
import json
import os

import numpy as np
import pytest

import oracle

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
INT_MAX = np.iinfo(np.int32).max
DYN = ["va_n1000_d1", "va_n1000_d8", "brunel_n1000_d15", "brunelp_n600_d15"]


def load(name):
    return np.load(os.path.join(GOLDEN, name + ".npz"))


def ell(lens, ids, width):
    e = np.full((len(lens), width), INT_MAX, dtype=np.int32)
    o = 0
    for i, k in enumerate(lens):
        e[i, :k] = ids[o:o + k]
        o += k
    return e.reshape(-1)


def conns_of(g):
    return [(int(a), int(b), float(np.float32(p))) for a, b, p in g["conns"]]


@pytest.fixture(scope="module", autouse=True)
def _built(oracle_built):
    return oracle_built


# ------------------------------------------------------------------ Philox
def test_philox_known_answers():
    # published known-answer vectors of Philox-4x32-10 (Random123 distribution)
    assert oracle.philox([0, 0, 0, 0], [0, 0]) == [0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8]
    assert oracle.philox([0xFFFFFFFF] * 4, [0xFFFFFFFF] * 2) == [0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD]
    assert oracle.philox([0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344], [0xA4093822, 0x299F31D0]) == [
        0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1]


# ------------------------------------------------------------------ layout
def test_layout_reference_known_answers():
    # spice_test/util/layout.cpp:9-47
    assert oracle.layout([1], [(0, 0, 0.0)]) == (1, [(0, 1, 0, 1, 0.0)], 0)
    assert oracle.layout([1], []) == (1, [], 0)
    n, c, _ = oracle.layout([100], [(0, 0, 0.25)])
    assert n == 100 and c == [(0, 100, 0, 100, 0.25)]
    n, c, _ = oracle.layout([10, 20, 30], [(1, 0, 0.5), (2, 1, 0.25), (1, 2, 0.125)])
    assert n == 60
    assert c == [(10, 30, 0, 10, 0.5), (10, 30, 30, 60, 0.125), (30, 60, 10, 30, 0.25)]
    # spice_test/util/adj_list.cpp:36-45: N=100, p=1 -> width 128; p=0 -> 0
    assert oracle.layout([100], [(0, 0, 1.0)])[2] == 128
    assert oracle.layout([100], [(0, 0, 0.0)])[2] == 0


def test_layout_golden():
    with open(os.path.join(GOLDEN, "layouts.json")) as f:
        gold = json.load(f)
    from golden.make_golden import LAYOUTS

    for name, pops, conns in LAYOUTS:
        n, c, w = oracle.layout(pops, conns)
        g = gold[name]
        assert n == g["size"] and w == g["max_degree"], name
        assert [list(x[:4]) for x in c] == [x[:4] for x in g["connections"]], name
        assert [np.float32(x[4]) for x in c] == [np.float32(x[4]) for x in g["connections"]], name
    # the Brunel 1e9 preset: N = 141,420, width 7,328
    assert gold["brunel_1e9"]["size"] == 141420 and gold["brunel_1e9"]["max_degree"] == 7328


def test_layout_rejects_bad_input():
    for pops, conns in [([], []), ([0], []), ([10], [(1, 0, 0.5)]), ([10], [(0, 0, 1.5)]), ([10], [(0, 0, 0.5), (0, 0, 0.1)])]:
        with pytest.raises(ValueError):
            oracle.layout(pops, conns)


# ------------------------------------------------------------------ generators
def test_reference_generator_golden():
    g = np.load(os.path.join(GOLDEN, "generator.npz"))
    for name, pops, conns in [("adj_10_20_30", [10, 20, 30], [(0, 0, 0.5), (0, 1, 0.1), (0, 2, 0.5), (1, 0, 1.0), (1, 2, 0.5)]),
                              ("n400_p01", [400], [(0, 0, 0.1)])]:
        seed = int(g[f"{name}_seed"])
        e, w = oracle.generate(pops, conns, seed, graph="reference")
        assert w == int(g[f"{name}_width"])
        assert np.array_equal(e, ell(g[f"{name}_lens"], g[f"{name}_ids"], w)), name


def check_graph_invariants(e, w, n, conns):
    """spice_test/util/adj_list.cpp:9-150: rows ascending, targets inside their connection
    ranges, sources without connections have empty rows, INT_MAX padding at the end."""
    rows = e.reshape(n, w) if w else np.zeros((n, 0), np.int32)
    for i in range(n):
        r = rows[i]
        valid = r[r != INT_MAX]
        assert np.all(r[len(valid):] == INT_MAX)
        assert np.all(np.diff(valid) > 0)
        allowed = np.zeros(n, bool)
        for a, b, c, d, p in conns:
            if a <= i < b and p > 0:
                allowed[c:d] = True
        assert np.all(allowed[valid]), i


@pytest.mark.parametrize("graph", ["reference", "philox"])
def test_generator_invariants(graph):
    pops, conns = [10, 20, 30], [(0, 0, 0.5), (0, 1, 0.1), (0, 2, 0.5), (1, 0, 1.0), (1, 2, 0.5)]
    n, flat, w = oracle.layout(pops, conns)
    e, w2 = oracle.generate(pops, conns, 99, graph=graph)
    assert w2 == w
    check_graph_invariants(e, w, n, flat)
    rows = e.reshape(n, w)
    assert np.all(rows[30:] == INT_MAX)  # C has no outgoing connections
    # p = 1: every candidate, ids 0..99 in order (spice_test/util/adj_list.cpp:36-58)
    e, w = oracle.generate([100], [(0, 0, 1.0)], 5, graph=graph)
    assert w == 128
    assert np.all(e.reshape(100, 128)[:, :100] == np.arange(100))
    e, w = oracle.generate([100], [(0, 0, 0.0)], 5, graph=graph)
    assert w == 0 and e.size == 0


def test_philox_generator_rows_random_access():
    pops, conns = [3000], [(0, 0, 0.05)]
    e, w = oracle.generate(pops, conns, 1234, graph="philox")
    rows = e.reshape(3000, w)
    for r in [0, 17, 1500, 2999]:
        assert np.array_equal(oracle.philox_row(pops, conns, 1234, r), rows[r])
    # Bernoulli(p): mean degree within 3 sigma of 150
    deg = (rows != INT_MAX).sum(1)
    assert abs(deg.mean() - 150) < 3 * np.sqrt(150 * 0.95 / 3000) * 3


def test_binomial_edge_cases_via_generator():
    # binornd(N, 0) = 0, binornd(N, 1) = N (spice_test/util/random.cpp:85-93) as seen
    # through the reference generator: p = 0 -> empty rows, p = 1 -> full rows
    for graph in ("reference", "philox"):
        e, w = oracle.generate([64], [(0, 0, 1.0)], 3, graph=graph)
        assert np.all((e.reshape(64, w) != INT_MAX).sum(1) == 64)


# ------------------------------------------------------------------ dynamics
def test_dt_sequence_is_kahan_compensated():
    d = oracle.dt_sequence(np.float32(1e-4), 20000)
    assert d[0] == np.float32(1e-4)
    assert len(np.unique(d)) > 1  # the compensated delta varies
    assert abs(float(d.astype(np.float64).sum()) - 2.0) < 1e-5


@pytest.mark.parametrize("name", DYN)
def test_oracle_matches_reference_golden(name):
    g = load(name)
    pops, conns = [int(x) for x in g["pops"]], conns_of(g)
    w = int(g["width"])
    edges = ell(g["lens"], g["ids"], w)
    net = oracle.OracleNet(str(g["model"]), pops, conns, dt=float(g["dt"]), delay=int(g["delay"]), seed=int(g["seed"]),
                           edges=edges, width=w)
    counts, spikes = g["counts"], g["spikes"]
    o = 0
    for i in range(int(g["steps"])):
        s = net.step()
        assert np.array_equal(s, spikes[o:o + counts[i]]), f"{name}: raster differs at step {i}"
        o += counts[i]
    for k, a in enumerate(net.neurons()):
        assert np.array_equal(a.view(np.uint32), g[f"neuron{k}"].view(np.uint32)), f"{name}: neuron attr {k}"
    if "W" in g:
        syn = net.synapses()
        valid = edges != INT_MAX
        for k, key in enumerate(["W", "Zpre", "Zpost"]):
            assert np.array_equal(syn[k][valid].view(np.uint32), g[key].view(np.uint32)), f"{name}: {key}"
        assert len(np.unique(g["W"])) > 10  # plasticity actually changed weights


def test_fp64_oracle_tracks_fp32():
    g = load("va_n1000_d1")
    pops, conns, w = [int(x) for x in g["pops"]], conns_of(g), int(g["width"])
    edges = ell(g["lens"], g["ids"], w)
    a = oracle.OracleNet("vogels_abbott", pops, conns, delay=1, seed=7, edges=edges, width=w, precision=32)
    b = oracle.OracleNet("vogels_abbott", pops, conns, delay=1, seed=7, edges=edges, width=w, precision=64)
    same = 0
    for _ in range(200):
        same += np.array_equal(a.step(), b.step())
    assert same >= 150
    va, vb = a.neurons()[0].astype(np.float64), b.neurons()[0]
    assert np.max(np.abs(va - vb)) < 1e-2


@pytest.mark.skipif(not oracle.have_reference(), reason="reference build not present")
def test_oracle_matches_reference_live():
    for model, pops, conns, delay in [("vogels_abbott", [700], [(0, 0, 0.03)], 3), ("brunel", [400, 400], [(0, 1, 0.1), (1, 1, 0.1)], 15),
                                      ("brunel_with_plasticity", [200, 200], [(0, 1, 0.1), (1, 1, 0.1)], 4)]:
        r = oracle.ReferenceNet(model, pops, conns, delay=delay, seed=3)
        e, w = r.adj()
        o = oracle.OracleNet(model, pops, conns, delay=delay, seed=3, edges=e, width=w)
        for i in range(1500):
            assert np.array_equal(r.step(), o.step()), (model, i)
        for x, y in zip(r.neurons(), o.neurons()):
            assert np.array_equal(x.view(np.uint32), y.view(np.uint32))


@pytest.mark.parametrize("model,pops,conns,delay", [
    ("brunel", [1500, 1500], [(0, 1, 0.1), (1, 1, 0.1)], 15),
    ("vogels_abbott", [2000], [(0, 0, 0.02)], 1),
    ("brunel_with_plasticity", [300, 300], [(0, 1, 0.1), (1, 1, 0.1)], 15),
])
def test_continuation_from_exported_state(model, pops, conns, delay):
    """A net handed the graph, state, clock and spikes in flight of another net at step S
    continues exactly as the original does: the restatement (set_state / set_progress) and
    the reference's cpu::snn (ReferenceNet.from_state), against an uninterrupted run. The
    GPU parity tests at full size and the benchmark's CPU leg rest on this."""
    o = oracle.OracleNet(model, pops, conns, delay=delay, seed=3, graph="philox", graph_seed=3)
    S = 900
    for _ in range(S - delay):
        o.step()
    rec = [o.step() for _ in range(delay)]
    counts, ids = [len(r) for r in rec], np.concatenate(rec)
    e, w = o.adj()
    st, sy = o.neurons(), o.synapses() or None
    c = oracle.OracleNet(model, pops, conns, delay=delay, seed=3, edges=e, width=w)
    c.set_state(st, sy)
    c.set_progress(S, counts, ids)
    nets = [c]
    if oracle.have_reference():
        nets.append(oracle.ReferenceNet.from_state(model, e, w, st, sy, delay=delay, seed=3, step0=S, counts=counts, ids=ids))
    for i in range(1200):
        want = o.step()
        for x in nets:
            assert np.array_equal(x.step(), want), i
    for x in nets:
        for a, b in zip(x.neurons(), o.neurons()):
            assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
        for a, b in zip(x.synapses(), o.synapses()):
            assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
