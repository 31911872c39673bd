"""Parity at the benchmarked sizes, through the C ABI, against the reference's own cpu::snn
(oracle/_ref, where built) or the CPU restatement pinned to it.

The headline net itself is checked: the GPU net that the benchmark times (1e9 synapses,
148 work-balanced tiles, 10-bit slices, one persistent cooperative launch per run) is run to
a steady state, its last `delay` steps are recorded, and its graph and state are exported.
The reference then continues from exactly that point (clock, Poisson stream, spikes in
flight: the reference's cpu::snn driven through the harness's state import) while the GPU
net continues on its own; rasters must be identical step for step and the final state bit
for bit (spice_test/cuda/snn.d.cpp:104-157 restated at full size). Vogels-Abbott at
4,000 + 1,000 neurons (delay 1) and Brunel+ at 5e8 synapses (through a forced-flush cycle)
follow the same scheme.

The reference keeps its Poisson stream in a process-wide counter, so at most one reference
net exists at a time here.
"""
import numpy as np
import pytest

import oracle
from spice_b200 import Layout, Snn

pytestmark = pytest.mark.gpu

INT_MAX = np.iinfo(np.int32).max


@pytest.fixture(autouse=True)
def _dev(gpu, oracle_built):
    yield


def bits_equal(a, b):
    return np.array_equal(np.asarray(a).view(np.uint32), np.asarray(b).view(np.uint32))


def split(counts, ids):
    o = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
    return [ids[o[k]:o[k + 1]] for k in range(len(counts))]


def continue_on_cpu(model, net, pops, conns, delay, seed, warm, check, synapses=False, reference=True):
    """Run `net` to step warm (recording its last `delay` steps), hand its state to a CPU
    net, then advance both by `check` steps. Returns (GPU rasters, CPU rasters, GPU net,
    CPU net, the edges)."""
    net.run(warm - delay - net.info().steps)
    counts, ids = net.run_record(delay)
    edges, width = net.adj()
    neurons = net.neurons()
    syn = net.synapses() if synapses else None
    if reference and oracle.have_reference():
        cpu = oracle.ReferenceNet.from_state(model, edges, width, neurons, syn, delay=delay, seed=seed, step0=warm,
                                             counts=counts, ids=ids)
    else:
        cpu = oracle.OracleNet(model, pops, conns, delay=delay, seed=seed, edges=edges, width=width)
        cpu.set_state(neurons, syn)
        cpu.set_progress(warm, counts, ids)
    gc, gi = net.run_record(check, cap=sum(pops) * check)
    got = split(gc, gi)
    want = [cpu.step() for _ in range(check)]
    return got, want, cpu, edges


def test_brunel_1e9_headline_net_matches_reference():
    """The benchmark's own net (N = 141,420, width 7,328, delay 15, seeds of the benchmark)
    at steady state: 150 steps identical to the reference's cpu::snn, final V and Twait
    bit-equal."""
    pops, conns, delay = [70710, 70710], [(0, 1, 0.1), (1, 1, 0.1)], 15
    net = Snn("brunel", Layout(pops, conns), dt=1e-4, delay=delay, seed=1, graph_seed=1337)
    info = net.info()
    assert info.width == 7328 and info.persistent == 1 and info.slice_pack == 12 and info.num_tiles <= 148
    got, want, cpu, _ = continue_on_cpu("brunel", net, pops, conns, delay, seed=1, warm=3150, check=150)
    for k, (a, b) in enumerate(zip(got, want)):
        assert np.array_equal(a, b), f"raster differs at step {3150 + k}"
    assert np.mean([len(a) for a in got]) > 300  # the steady-state load the benchmark times
    for a, b in zip(net.neurons(), cpu.neurons()):
        assert bits_equal(a, b)


def test_vogels_abbott_config_size_matches_oracle():
    """4,000 exc + 1,000 inh, p = 0.02, delay 1: the persistent synchronous path of the
    va workload, 1,000 steps from the start against the restatement and 500 more from a
    mid-run hand-over to the reference."""
    pops, conns = [5000], [(0, 0, 0.02)]
    # window_flat's persistent synchronous path (the automatic choice at this size and delay
    # is window_counts: checked against it below)
    net = Snn("vogels_abbott", Layout(pops, conns), dt=1e-4, delay=1, seed=1, graph_seed=1337, options={"kernel": "window"})
    assert net.info().persistent == 1
    auto = Snn("vogels_abbott", Layout(pops, conns), dt=1e-4, delay=1, seed=1, graph_seed=1337)
    assert auto.info().persistent == 0 and auto.info().slice_pack == 0
    ac, ai = auto.run_record(1000)
    edges, width = net.adj()
    ref = oracle.OracleNet("vogels_abbott", pops, conns, delay=1, seed=1, edges=edges, width=width)
    counts, ids = net.run_record(1000)
    assert np.array_equal(counts, ac) and np.array_equal(ids, ai)
    for k, a in enumerate(split(counts, ids)):
        assert np.array_equal(a, ref.step()), f"raster differs at step {k}"
    for a, b in zip(net.neurons(), ref.neurons()):
        assert bits_equal(a, b)
    got, want, cpu, _ = continue_on_cpu("vogels_abbott", net, pops, conns, 1, seed=1, warm=1500, check=500)
    for k, (a, b) in enumerate(zip(got, want)):
        assert np.array_equal(a, b), f"raster differs at step {1500 + k}"
    for a, b in zip(net.neurons(), cpu.neurons()):
        assert bits_equal(a, b)


def ulps(a, b):
    """Distance in units in the last place between float32 arrays of one sign."""
    ia, ib = np.asarray(a, np.float32).view(np.int32).astype(np.int64), np.asarray(b, np.float32).view(np.int32).astype(np.int64)
    return np.abs(ia - ib)


def test_brunel_plus_5e8_matches_oracle_through_a_flush_cycle():
    """N = 100,000 (width 5,216), lazy STDP: from a mid-run hand-over, 80 steps (more than
    the 63-step forced-flush cycle) against the restatement; rasters identical, Twait
    identical, V within 1e-5 relative, weights within 2 ulp and traces identical."""
    pops, conns, delay = [50_000, 50_000], [(0, 1, 0.1), (1, 1, 0.1)], 15
    net = Snn("brunel_with_plasticity", Layout(pops, conns), dt=1e-4, delay=delay, seed=1, graph_seed=1337)
    got, want, cpu, edges = continue_on_cpu("brunel_with_plasticity", net, pops, conns, delay, seed=1, warm=200, check=80,
                                            synapses=True, reference=False)
    for k, (a, b) in enumerate(zip(got, want)):
        assert np.array_equal(a, b), f"raster differs at step {200 + k}"
    (v, tw), (cv, ctw) = net.neurons(), cpu.neurons()
    assert bits_equal(tw, ctw)
    assert np.max(np.abs(v.astype(np.float64) - cv) / np.maximum(np.abs(cv), 0.02)) <= 1e-5
    valid = edges != INT_MAX
    sa, sb = net.synapses(), cpu.synapses()
    assert ulps(sa[0][valid], sb[0][valid]).max() <= 2
    assert bits_equal(sa[1][valid], sb[1][valid]) and bits_equal(sa[2][valid], sb[2][valid])
