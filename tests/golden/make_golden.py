"""Generates the golden fixtures in this directory from the reference's own cpu::snn.

    make -C oracle ref && python tests/golden/make_golden.py

Runs in the container that holds the reference checkout (oracle/_ref/libspice_ref.so is
built from its sources with the counter-RNG shim, see oracle/Makefile). Each case stores
the reference's graph, its spike raster and its final state; the tests pin the CPU
restatement (oracle/spice_oracle.cpp) against them and the GPU path against the pinned
restatement. Fresh process per run: the reference seeds its graph generator from a
process-wide counter (spice/util/adj_list.cpp:11,53), so the order below fixes the graphs.
"""
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
import oracle  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))

# (name, model, pops, connections, delay, steps, poisson seed)
DYNAMICS = [
    ("va_n1000_d1", "vogels_abbott", [1000], [(0, 0, 0.02)], 1, 1000, 7),
    ("va_n1000_d8", "vogels_abbott", [1000], [(0, 0, 0.05)], 8, 1000, 7),
    ("brunel_n1000_d15", "brunel", [500, 500], [(0, 1, 0.1), (1, 1, 0.1)], 15, 1000, 11),
    ("brunelp_n600_d15", "brunel_with_plasticity", [300, 300], [(0, 1, 0.1), (1, 1, 0.1)], 15, 2000, 7),
]

# layouts whose flattening / width the reference computes (spice_test/util/layout.cpp and
# the benchmark presets of samples/main.cpp:1271-1294)
LAYOUTS = [
    ("np_1_0", [1], [(0, 0, 0.0)]),
    ("np_100_025", [100], [(0, 0, 0.25)]),
    ("pops_10_20_30", [10, 20, 30], [(1, 0, 0.5), (2, 1, 0.25), (1, 2, 0.125)]),
    ("adj_10_20_30", [10, 20, 30], [(0, 0, 0.5), (0, 1, 0.1), (0, 2, 0.5), (1, 0, 1.0), (1, 2, 0.5)]),
    ("n100_p1", [100], [(0, 0, 1.0)]),
    ("n100_p0", [100], [(0, 0, 0.0)]),
    ("va_5000", [5000], [(0, 0, 0.02)]),
    ("brunel_1e9", [70710, 70710], [(0, 1, 0.1), (1, 1, 0.1)]),
    ("brunel_5e8", [50000, 50000], [(0, 1, 0.1), (1, 1, 0.1)]),
    ("va_1e9", [223606], [(0, 0, 0.02)]),
]


def csr(edges, width):
    e = edges.reshape(-1, width) if width else edges.reshape(-1, 0)
    lens = (e != np.iinfo(np.int32).max).sum(axis=1).astype(np.int32)
    return lens, e[e != np.iinfo(np.int32).max].astype(np.int32)


def ref_layout(pops, conns):
    lib = oracle.ref_lib()
    cap = max(1, len(conns))
    import ctypes as C

    rng, pr = (C.c_int * (4 * cap))(), (C.c_float * cap)()
    md, sz = C.c_uint64(), C.c_uint64()
    k = lib.ref_layout(*oracle._layout_args(pops, conns), rng, pr, cap, C.byref(md), C.byref(sz))
    return {"size": sz.value, "max_degree": md.value,
            "connections": [[rng[4 * i], rng[4 * i + 1], rng[4 * i + 2], rng[4 * i + 3], float(pr[i])] for i in range(k)]}


def main():
    if not oracle.have_reference():
        sys.exit("build the reference first: make -C oracle ref")
    layouts = {name: ref_layout(p, c) for name, p, c in LAYOUTS}
    with open(os.path.join(OUT, "layouts.json"), "w") as f:
        json.dump(layouts, f, indent=1)

    # the reference generator, first call of a fresh process (seed 1337)
    import ctypes as C

    lib = oracle.ref_lib()
    gens = {}
    for name, pops, conns in [("adj_10_20_30", [10, 20, 30], [(0, 0, 0.5), (0, 1, 0.1), (0, 2, 0.5), (1, 0, 1.0), (1, 2, 0.5)]),
                              ("n400_p01", [400], [(0, 0, 0.1)])]:
        n, w = layouts.get(name, {}).get("size"), layouts.get(name, {}).get("max_degree")
        if n is None:
            l = ref_layout(pops, conns)
            n, w = l["size"], l["max_degree"]
        out = (C.c_int * max(1, n * w))()
        seed = lib.ref_generate(*oracle._layout_args(pops, conns), out)
        lens, ids = csr(np.frombuffer(out, dtype=np.int32)[: n * w], w)
        gens[name] = dict(seed=seed, width=w, lens=lens, ids=ids)
    np.savez_compressed(os.path.join(OUT, "generator.npz"),
                        **{f"{k}_{f}": v for k, d in gens.items() for f, v in d.items()})

    for name, model, pops, conns, delay, steps, seed in DYNAMICS:
        net = oracle.ReferenceNet(model, pops, conns, dt=1e-4, delay=delay, seed=seed)
        edges, width = net.adj()
        lens, ids = csr(edges, width)
        counts, spikes = [], []
        for _ in range(steps):
            s = net.step()
            counts.append(len(s))
            spikes.append(s)
        neu = net.neurons()
        extra = {}
        syn = net.synapses()
        if syn:
            valid = edges != np.iinfo(np.int32).max
            extra = {"W": syn[0][valid], "Zpre": syn[1][valid], "Zpost": syn[2][valid]}
        np.savez_compressed(
            os.path.join(OUT, f"{name}.npz"),
            model=model, pops=np.array(pops), conns=np.array(conns, dtype=np.float64), delay=delay, steps=steps, seed=seed,
            dt=np.float32(1e-4), width=width, lens=lens, ids=ids, counts=np.array(counts, dtype=np.int32),
            spikes=np.concatenate(spikes).astype(np.int32) if spikes else np.zeros(0, np.int32),
            **{f"neuron{i}": a for i, a in enumerate(neu)}, **extra)
        print(name, "n", net.n, "width", width, "spikes", sum(counts))


if __name__ == "__main__":
    main()
