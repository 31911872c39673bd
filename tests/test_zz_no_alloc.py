"""spk_generate_adj_list_static: the graph generator for callers that cannot allocate
device memory (a framework's caching allocator owns the device, or the caller cannot pay
cudaMalloc's device-wide synchronisation). Through the C ABI, two calls in a row must
produce exactly the graphs the allocating entry point produces. The test itself
allocates the output buffers (with torch); the entry point allocates nothing."""
import ctypes as C

import numpy as np
import pytest

import spice_b200

pytestmark = pytest.mark.gpu

CASES = [
    ([2000, 2000], [(0, 1, 0.1), (1, 1, 0.1)], 11),
    ([10, 20, 30], [(0, 0, 0.5), (0, 1, 0.1), (0, 2, 0.5), (1, 0, 1.0), (1, 2, 0.5)], 12),
]


def generate(fn, layout, seed, stream):
    import torch

    n, w = layout.size(), layout.max_degree()
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


def test_static_generator_rejects_oversized_tables(gpu):
    lib = spice_b200.library()
    conns = [(a, b, 0.1) for a in range(40) for b in range(40)][:1100]  # 1100 distinct pairs
    layout = spice_b200.Layout([5] * 40, conns)
    d = layout.desc()
    rc = lib.spk_generate_adj_list_static(None, C.byref(d), 1, None)
    assert rc == spice_b200.ERR_INVALID
    assert b"at most 1024" in lib.spk_last_error()
