"""TEST INFRASTRUCTURE -- the checks of the tests' model (weighted_lif.h) on the generic
kernel, run in a child process whose SPICE_B200_LIB is the build with the model compiled in
(tests/test_gpu_ordered.py starts it). Exits non-zero with a message on the first mismatch.

    python check_weighted_lif.py gpu      # GPU net against the reference's cpu::snn of the model
    python check_weighted_lif.py abi      # the build exports the model (no GPU needed)
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import spice_b200  # noqa: E402
from spice_b200 import Layout, Snn  # noqa: E402


def check(cond, msg):
    if not cond:
        print("FAIL:", msg, flush=True)
        sys.exit(1)


def expected_weights(edges, width, n):
    """The model's synapse init (weighted_lif.h) restated in float32."""
    src = np.repeat(np.arange(n, dtype=np.int64), width)
    dst = edges.astype(np.int64)
    real = edges != np.iinfo(np.int32).max
    k = (1 + (src * 7 + dst * 13) % 5).astype(np.float32)
    w = np.float32(0.0004) * k
    exc = src < int(np.float32(0.8) * np.float32(n))
    out = np.where(exc, w, np.float32(-5.0) * w).astype(np.float32)
    out[~real] = 0
    return out


def abi():
    assert spice_b200.LIB_PATH == os.environ["SPICE_B200_LIB"]
    nt, st = spice_b200.model_attrs("user")
    check([np.dtype(t) for t in nt] == [np.float32, np.float32, np.int32], f"neuron attributes {nt}")
    check([np.dtype(t) for t in st] == [np.float32], f"synapse attributes {st}")
    print("abi ok")


def run_pair(net, ref, steps):
    for k in range(steps):
        a, b = net.step(out=True), ref.step()
        check(np.array_equal(np.sort(a), np.sort(b)), f"raster differs at step {k}: {len(a)} vs {len(b)} spikes")
    for x, y in zip(net.neurons(), ref.neurons()):
        check(np.array_equal(x.view(np.uint32), y.view(np.uint32)), "state differs")


def gpu():
    import oracle

    types = ([np.float32, np.float32, np.int32], [np.float32])
    total = 0
    for n, p, delay, steps, options in [(3000, 0.05, 1, 1000, None), (5000, 0.02, 8, 800, None),
                                        (20_000, 0.01, 15, 400, {"tile_target": 40})]:
        opts = dict(options or {})
        tile_target = opts.pop("tile_target", 0)
        net = Snn("user", Layout(n, p), delay=delay, seed=5, graph_seed=9, tile_target=tile_target, options=opts)
        info = net.info()
        check(info.slice_pack == 0 and info.persistent == 0, "the generic kernel runs the user model")
        edges, width = net.adj()
        W = net.synapses()
        check(len(W) == 1 and np.array_equal(W[0].view(np.uint32), expected_weights(edges, width, n).view(np.uint32)),
              "synapse init differs from the model's")
        ref = oracle.ReferenceNet.from_state(7, edges, width, net.neurons(), W, delay=delay, seed=5,
                                             lib_path=oracle.REF_USER_LIB, types=types)
        for k in range(steps):
            a, b = net.step(out=True), ref.step()
            check(np.array_equal(np.sort(a), np.sort(b)), f"n={n}: raster differs at step {k}")
            total += len(a)
        for x, y in zip(net.neurons(), ref.neurons()):
            check(np.array_equal(x.view(np.uint32), y.view(np.uint32)), f"n={n}: state differs")
        # windows of `delay` steps (run) and the state after them
        net.run(3 * delay + 5)
        for _ in range(3 * delay + 5):
            ref.step()
        for x, y in zip(net.neurons(), ref.neurons()):
            check(np.array_equal(x.view(np.uint32), y.view(np.uint32)), f"n={n}: state after run() differs")
        # a checkpoint holds the synapse attributes; the restored net continues identically
        r = Snn.restore(net.checkpoint())
        check(np.array_equal(r.synapses()[0], net.synapses()[0]), "restored synapses differ")
        for k in range(2 * delay + 3):
            a, b, c = net.step(out=True), r.step(out=True), ref.step()
            check(np.array_equal(a, b) and np.array_equal(np.sort(a), np.sort(c)), f"restored net differs at step {k}")
    check(total > 1000, f"too few spikes ({total})")

    # imported weights (random, mixed signs) on both sides
    n = 4000
    net = Snn("user", Layout(n, 0.03), delay=2, seed=2, graph_seed=3)
    edges, width = net.adj()
    rng = np.random.default_rng(7)
    Wr = (rng.standard_normal(edges.size) * 0.002).astype(np.float32)
    Wr[edges == np.iinfo(np.int32).max] = 0
    net.set_synapses([Wr])
    check(np.array_equal(net.synapses()[0], Wr), "set_synapses round trip")
    ref = oracle.ReferenceNet.from_state(7, edges, width, net.neurons(), [Wr], delay=2, seed=2,
                                         lib_path=oracle.REF_USER_LIB, types=types)
    run_pair(net, ref, 600)
    print(f"gpu ok: {total} spikes, bit-identical to the reference's cpu::snn of the model")


if __name__ == "__main__":
    {"abi": abi, "gpu": gpu}[sys.argv[1]]()
