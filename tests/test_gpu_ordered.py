"""The generic window kernel (window_ordered): every arrival through the model's own
receive( src, dst, syn, ... ), per target in the reference CPU simulator's order
(spice/cpu/snn.h.cpp:111-127), for models the counting kernels cannot run (no input
classes, static synapse attributes).

  * the library's own models forced onto it (kernel="ordered") against the counting kernels,
    themselves pinned to the oracle;
  * a model defined only in the tests (tests/user_model/weighted_lif.h: per-synapse static
    weights, no input classes), compiled into a build of the library as model "user",
    against the reference's own cpu::snn of the same header (oracle/_ref/libspice_ref_user.so).
"""
import os
import subprocess
import sys

import numpy as np
import pytest

import oracle
from spice_b200 import Layout, Snn
from spice_b200 import build as sb_build

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
USER_DIR = os.path.join(HERE, "user_model")
USER_HEADER = os.path.join(USER_DIR, "weighted_lif.h")
USER_LIB = os.path.join(USER_DIR, "libspice_b200_weighted_lif.so")


def bits_equal(a, b):
    return np.array_equal(np.asarray(a).view(np.uint32), np.asarray(b).view(np.uint32))


@pytest.fixture(autouse=True)
def _dev(gpu, oracle_built):
    yield


@pytest.mark.parametrize("model,pops,conns,delay,steps", [
    ("vogels_abbott", [4000], [(0, 0, 0.02)], 1, 600),
    ("vogels_abbott", [5000], [(0, 0, 0.02)], 8, 500),
    ("brunel", [10_000, 10_000], [(0, 1, 0.1), (1, 1, 0.1)], 15, 400),
    ("synth", [100_000], [(0, 0, 16 / 100_000)], 4, 200),
    ("brunel_fixed", [5000, 5000], [(0, 1, 0.1), (1, 1, 0.1)], 3, 400),
])
def test_ordered_kernel_matches_counting_kernels(model, pops, conns, delay, steps):
    """A model with input classes through window_ordered (each arrival's receive() in
    ascending source order) against window_flat / window_counts (integer counts replayed per
    class): the same additions in the same order, so identical rasters and state."""
    layout = Layout(pops, conns)
    a = Snn(model, layout, delay=delay, seed=4, graph_seed=4, options={"kernel": "ordered"})
    b = Snn(model, layout, delay=delay, seed=4, graph_seed=4)
    assert a.info().slice_pack == 0 and a.info().persistent == 0
    ca, ia = a.run_record(steps, cap=sum(pops) * steps // 4)
    cb, ib = b.run_record(steps, cap=sum(pops) * steps // 4)
    assert ca.sum() > 0 and np.array_equal(ca, cb) and np.array_equal(ia, ib)
    for x, y in zip(a.neurons(), b.neurons()):
        assert bits_equal(x, y)
    # a checkpoint keeps the kernel choice
    r = Snn.restore(a.checkpoint())
    for k in range(2 * delay + 2):
        assert np.array_equal(r.step(out=True), b.step(out=True)), k


def test_ordered_kernel_against_the_oracle():
    """VA on window_ordered against the oracle's restatement, spike by spike."""
    net = Snn("vogels_abbott", Layout([3000], [(0, 0, 0.02)]), delay=1, seed=3, graph_seed=3, options={"kernel": "ordered"})
    edges, width = net.adj()
    ref = oracle.OracleNet("vogels_abbott", [3000], [(0, 0, 0.02)], delay=1, seed=3, edges=edges, width=width)
    total = 0
    for k in range(1000):
        a, b = net.step(out=True), ref.step()
        assert np.array_equal(a, b), k
        total += len(a)
    assert total > 0
    for x, y in zip(net.neurons(), ref.neurons()):
        assert bits_equal(x, y)


@pytest.fixture(scope="module")
def user_lib():
    """The library built with the tests' model compiled in (built by the package build where
    nvcc is; rebuilt here only if missing or stale)."""
    sb_build.build_user(USER_HEADER, "test_models::weighted_lif", USER_LIB)
    if not oracle.os.path.exists(oracle.REF_USER_LIB):
        pytest.fail(f"{oracle.REF_USER_LIB} is missing: the reference build of the tests' model")
    return USER_LIB


def test_user_model_against_the_reference_cpu_snn(user_lib):
    """A model defined only in the tests (static per-synapse weights, no input classes) on
    the GPU against the reference's own cpu::snn of the same header: synapse init, rasters
    every step and final state bit for bit, windows of `delay` steps, a checkpoint round trip
    and imported weights."""
    env = dict(os.environ, SPICE_B200_LIB=user_lib)
    r = subprocess.run([sys.executable, os.path.join(USER_DIR, "check_weighted_lif.py"), "gpu"], env=env,
                       capture_output=True, text=True, timeout=1200)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "gpu ok" in r.stdout
