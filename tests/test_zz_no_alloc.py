"""spk_generate_adj_list_static: the graph generator for callers that cannot allocate
device memory (a framework's caching allocator owns the device, or the caller cannot pay
cudaMalloc's device-wide synchronisation). Through the C ABI, two calls in a row must
produce exactly the graphs the allocating entry point produces, and a call must leave the
device's free memory unchanged. The test itself allocates the output buffers (with
torch); the entry point allocates nothing."""
import ctypes as C

import numpy as np
import pytest

import spice_b200

pytestmark = pytest.mark.gpu

CASES = [
    ([2000, 2000], [(0, 1, 0.1), (1, 1, 0.1)], 11),
    ([10, 20, 30], [(0, 0, 0.5), (0, 1, 0.1), (0, 2, 0.5), (1, 0, 1.0), (1, 2, 0.5)], 12),
]


def generate(fn, layout, seed, stream, out=None):
    import torch

    n, w = layout.size(), layout.max_degree()
    if out is None:
        out = torch.full((max(1, n * w),), -7, dtype=torch.int32, device="cuda")
    d = layout.desc()
    rc = fn(C.c_void_p(stream.cuda_stream), C.byref(d), seed, C.c_void_p(out.data_ptr()))
    assert rc == spice_b200.OK, spice_b200.library().spk_last_error()
    stream.synchronize()
    return out[: n * w].cpu().numpy()


def test_static_generator_matches_allocating_one(gpu):
    import torch

    lib = spice_b200.library()
    stream = torch.cuda.Stream()
    for pops, conns, seed in CASES:  # two calls in a row, different tables
        layout = spice_b200.Layout(pops, conns)
        want = generate(lib.spk_generate_adj_list, layout, seed, stream)
        got = generate(lib.spk_generate_adj_list_static, layout, seed, stream)
        assert got.size == layout.size() * layout.max_degree()
        assert np.array_equal(got, want)


def test_static_generator_leaves_free_memory_unchanged(gpu):
    """A cudaMalloc would take at least one 2 MiB granule: after a warm-up call, a call on a
    layout this process has not used yet must not change the device's free memory."""
    import torch

    lib = spice_b200.library()
    stream = torch.cuda.Stream()
    warm = spice_b200.Layout([300, 300], [(0, 1, 0.2), (1, 0, 0.1)])
    generate(lib.spk_generate_adj_list_static, warm, 5, stream)
    fresh = spice_b200.Layout([1500, 700, 900], [(0, 1, 0.05), (2, 0, 0.3), (1, 1, 0.02)])
    out = torch.full((fresh.size() * fresh.max_degree(),), -7, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    got = generate(lib.spk_generate_adj_list_static, fresh, 6, stream, out)
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0
    assert np.array_equal(got, generate(lib.spk_generate_adj_list, fresh, 6, stream))


def test_static_generator_limits_are_exact(gpu):
    """Exactly 1024 connections and exactly 1024 populations fit (and match the allocating
    generator); one more of either is refused."""
    import torch

    lib = spice_b200.library()
    stream = torch.cuda.Stream()
    # 32 x 32 populations, every pair connected: 1024 connections, several table pieces
    conns = [(a, b, 0.3 + 0.01 * ((a + b) % 7)) for a in range(32) for b in range(32)]
    full = spice_b200.Layout([3 + (i % 4) for i in range(32)], conns)
    assert len(full.connections()) == 1024
    assert np.array_equal(generate(lib.spk_generate_adj_list_static, full, 21, stream),
                          generate(lib.spk_generate_adj_list, full, 21, stream))
    many = spice_b200.Layout([2] * 1024, [(i, (i * 7) % 1024, 0.5) for i in range(0, 1024, 3)])
    assert np.array_equal(generate(lib.spk_generate_adj_list_static, many, 22, stream),
                          generate(lib.spk_generate_adj_list, many, 22, stream))
    too_many_pops = spice_b200.Layout([2] * 1025, [(0, 1, 0.5)])
    d = too_many_pops.desc()
    assert lib.spk_generate_adj_list_static(None, C.byref(d), 1, None) == spice_b200.ERR_INVALID
    assert b"at most 1024 populations" in lib.spk_last_error()


def test_static_generator_rejects_oversized_tables(gpu):
    lib = spice_b200.library()
    conns = [(a, b, 0.1) for a in range(40) for b in range(40)][:1025]  # 1025 distinct pairs
    layout = spice_b200.Layout([5] * 40, conns)
    d = layout.desc()
    rc = lib.spk_generate_adj_list_static(None, C.byref(d), 1, None)
    assert rc == spice_b200.ERR_INVALID
    assert b"at most 1024 connections" in lib.spk_last_error()
