"""The reference's own cpu::snn of the tests' model (oracle/_ref/libspice_ref_user.so, built
from tests/user_model/weighted_lif.h) against a numpy restatement of that model and of
cpu::snn's step (spice/cpu/snn.h.cpp:111-157): receive every arrival of the step that fired
`delay` steps ago in ascending source and row order, then update every neuron with the
simulated clock's Kahan-compensated dt (spice/util/numeric.h:9-33). Pins the oracle that
the GPU's generic kernel is checked against (tests/test_gpu_ordered.py). No GPU."""
import numpy as np
import pytest

import oracle

INT_MAX = np.iinfo(np.int32).max
F = np.float32


def kahan_dts(dt, steps):
    c, s, out = F(0), F(0), []
    for _ in range(steps):
        y = F(F(dt) - c)
        t = F(s + y)
        c = F(F(t - s) - y)
        s = t
        out.append(y)
    return out


def restated_run(edges, width, W, n, delay, steps, dt=1e-4):
    """weighted_lif (tests/user_model/weighted_lif.h) stepped as cpu::snn steps it."""
    V, I, Tw = np.zeros(n, F), np.zeros(n, F), np.zeros(n, np.int32)
    rows = edges.reshape(n, width)
    wrows = W.reshape(n, width)
    ids = np.arange(n)
    bias = F(0.021) + F(0.00008) * ((ids * 37) % 101).astype(F)
    inv_mem, inv_syn = F(1) / F(0.02), F(1) / F(0.005)
    queue, rasters = [], []
    for dtk in kahan_dts(dt, steps):
        if len(queue) >= delay:
            for src in queue.pop(0):
                m = rows[src] != INT_MAX
                # one row: every target once, so a fancy-index add keeps the order per target
                I[rows[src][m]] = I[rows[src][m]] + wrows[src][m]
        Tw = Tw - 1
        active = Tw <= 0
        fire = active & (V > F(0.02))
        grow = active & ~fire
        V = np.where(fire, F(0), V)
        Tw = np.where(fire, 20, Tw).astype(np.int32)
        V = np.where(grow, V + (bias - V + I) * (F(dtk) * inv_mem), V).astype(F)
        I = (I - I * (F(dtk) * inv_syn)).astype(F)
        spikes = np.flatnonzero(fire)
        queue.append(spikes)
        rasters.append(spikes)
    return rasters, (V, I, Tw)


def random_graph(n, width, p, rng):
    e = np.full((n, width), INT_MAX, np.int32)
    for i in range(n):
        t = np.flatnonzero(rng.random(n) < p)[:width]
        e[i, :len(t)] = t
    return e.reshape(-1)


@pytest.mark.skipif(not __import__("os").path.exists(oracle.REF_USER_LIB), reason="reference build of the tests' model absent")
@pytest.mark.parametrize("n,p,delay", [(400, 0.1, 1), (600, 0.05, 4)])
def test_reference_cpu_snn_of_the_test_model_matches_restatement(n, p, delay):
    rng = np.random.default_rng(n)
    width = 96
    edges = random_graph(n, width, p, rng)
    W = (rng.standard_normal(edges.size) * 0.003).astype(F)
    W[edges == INT_MAX] = 0
    neurons = [np.zeros(n, F), np.zeros(n, F), np.zeros(n, np.int32)]
    ref = oracle.ReferenceNet.from_state(7, edges, width, neurons, [W], delay=delay, seed=1, lib_path=oracle.REF_USER_LIB,
                                         types=([F, F, np.int32], [F]))
    want, state = restated_run(edges, width, W, n, delay, 400)
    total = 0
    for k in range(400):
        got = ref.step()
        assert np.array_equal(np.sort(got), want[k]), k
        total += len(got)
    assert total > 100
    for a, b in zip(ref.neurons(), state):
        assert np.array_equal(a.view(np.uint32), np.asarray(b).view(np.uint32))
    assert np.array_equal(ref.synapses()[0], W)
