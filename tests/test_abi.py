"""The C-ABI library builds for sm_100a, loads, and exports every entry point that
include/*.h declares (no GPU needed: nothing here launches a kernel)."""
import glob
import os
import re

import pytest

import spice_b200
from spice_b200 import build as sb_build

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names |= set(re.findall(r"\b(spk_[a-z0-9_]+)\s*\(", text))
    return sorted(names)


@pytest.fixture(scope="module")
def lib():
    sb_build.build()
    return spice_b200.library()


def test_every_declared_symbol_is_exported(lib):
    names = declared_functions()
    assert len(names) >= 15
    for n in names:
        assert hasattr(lib, n), n


def test_library_is_sm100a():
    cmd = sb_build.command()
    assert "arch=compute_100a,code=sm_100a" in cmd
    assert "-fmad=false" in cmd and "--use_fast_math" not in cmd


def test_errors_without_device_are_reported_not_fatal(lib):
    # invalid model / invalid layout are rejected before any device work
    import ctypes as C

    assert lib.spk_model_attrs(9, None, None, None, 0) == spice_b200.ERR_INVALID
    assert b"invalid model" in lib.spk_last_error()
    with pytest.raises(spice_b200.InvalidArgument):
        spice_b200.Layout([10], [(0, 0, 1.5)]).max_degree()
    nn, ns = spice_b200.model_attrs("brunel_with_plasticity")
    assert len(nn) == 2 and len(ns) == 3


def test_layout_matches_reference_known_answers(lib):
    L = spice_b200.Layout
    assert L([10, 20, 30], [(1, 0, 0.5), (2, 1, 0.25), (1, 2, 0.125)]).connections() == [
        (10, 30, 0, 10, 0.5), (10, 30, 30, 60, 0.125), (30, 60, 10, 30, 0.25)]
    assert L(100, 1.0).max_degree() == 128
    assert L(100, 0.0).max_degree() == 0
    assert L([70710, 70710], [(0, 1, 0.1), (1, 1, 0.1)]).max_degree() == 7328


def test_net_options_checked_without_device(lib):
    """Build choices (spk_net_options): automatic by default, checked before device work."""
    import ctypes as C

    o = spice_b200.net_options()
    assert o.tile_target == 0
    assert [getattr(o, f) for f in ("kernel", "slice_bits", "tiling", "persistent", "pipelined", "slots")] == [-1] * 6
    o = spice_b200.net_options(7, kernel="direct", slice_bits=16, tiling="uniform", persistent=False, pipelined=False, slots=True)
    assert (o.tile_target, o.kernel, o.slice_bits, o.tiling, o.persistent, o.pipelined, o.slots) == (7, 1, 16, 1, 0, 0, 1)
    with pytest.raises(spice_b200.InvalidArgument):
        spice_b200.net_options(colour="red")
    with pytest.raises(spice_b200.InvalidArgument):
        spice_b200.net_options(slice_bits=12)
    with pytest.raises(spice_b200.InvalidArgument):
        spice_b200.net_options(-1)
    d = spice_b200.Layout([100, 100], [(0, 1, 0.1)]).desc()
    h = C.c_void_p()
    bad = spice_b200.net_options()
    bad.slice_bits = 12
    assert lib.spk_net_create_opts(C.byref(h), 0, C.byref(d), 1e-4, 1, 1, 1, 0, C.byref(bad)) == spice_b200.ERR_INVALID
    assert b"slice_bits" in lib.spk_last_error()
    bad = spice_b200.net_options()
    bad.tile_target = -3
    out = C.c_uint64()
    assert lib.spk_net_estimate_bytes_opts(0, C.byref(d), 1, 0, C.byref(bad), C.byref(out)) == spice_b200.ERR_INVALID
    assert lib.spk_net_estimate_bytes(0, C.byref(d), 1, 0, -3, C.byref(out)) == spice_b200.ERR_INVALID


def test_server_and_batch_arguments_checked_without_device(lib):
    import ctypes as C

    h = C.c_void_p()
    assert lib.spk_server_create(C.byref(h), 0, 0, 10) == spice_b200.ERR_INVALID  # zero budget
    assert lib.spk_server_create(None, 0, 1 << 30, 10) == spice_b200.ERR_INVALID
    assert lib.spk_server_create_ex(C.byref(h), 0, 1 << 30, 10, 9) == spice_b200.ERR_INVALID  # builders 1-8
    assert b"builders" in lib.spk_last_error()
    assert lib.spk_server_wait(None, 0, 0.0) == spice_b200.ERR_INVALID
    assert lib.spk_batch_run(None, 1) == spice_b200.ERR_INVALID
    assert lib.spk_net_set_producer_warps(None, 12) == spice_b200.ERR_INVALID
    assert lib.spk_batch_add(None, None) == spice_b200.ERR_INVALID
    assert lib.spk_server_destroy(None) == spice_b200.OK
    assert lib.spk_batch_destroy(None) == spice_b200.OK


def test_tile_targets_share_sms_by_work():
    from spice_b200.autotune import layout_work, tile_targets

    L = spice_b200.Layout
    w = [layout_work(L([1000, 1000], [(0, 1, 0.1), (1, 1, 0.1)])), layout_work(L([100], [(0, 0, 0.5)]))]
    assert w[0] > w[1] > 0
    t = tile_targets(w, 148)
    assert t[0] >= t[1] >= 1 and sum(t) <= 150
    assert tile_targets(w, 148, 2.0)[0] > t[0]
    assert tile_targets([0.0, 0.0], 148) == [1, 1]
    from spice_b200.autotune import size_buckets

    assert size_buckets([5.0, 1.0, 3.0], 3) == [2, 0, 1]
    assert tile_targets(w, 148, [1.0, 4.0], [0, 1])[1] >= t[1]


def test_restore_rejects_bad_checkpoints_before_device_work(lib):
    import ctypes as C

    h = C.c_void_p()
    junk = (C.c_ubyte * 256)()
    assert lib.spk_net_restore(C.byref(h), junk, 256, 0) == spice_b200.ERR_INVALID
    assert b"not a checkpoint" in lib.spk_last_error()
    assert lib.spk_net_restore(C.byref(h), junk, 8, 0) == spice_b200.ERR_INVALID
    assert b"truncated" in lib.spk_last_error()
    assert lib.spk_net_checkpoint(None, None, 0, None) == spice_b200.ERR_INVALID


def _checkpoint_bytes(edges, n, width, ring_cnt=None, ring_ids=None, threads=64, tile=64, model=1, delay=2):
    """A checkpoint laid out as spk_net_checkpoint writes it (header, tile starts, then
    {u32 id, u64 bytes, data} per buffer) for a one-tile Brunel net."""
    import struct

    import numpy as np

    slots = 2 * delay
    ntiles = (n + tile - 1) // tile
    first = np.array([min(j * tile, n) for j in range(ntiles + 1)], np.int32)
    bufs = [(1, np.asarray(edges, np.int32).tobytes())]
    bufs += [(10, np.zeros(n, np.float32).tobytes()), (11, np.zeros(n, np.int32).tobytes())]
    ids = np.zeros(slots * n, np.int32) if ring_ids is None else np.asarray(ring_ids, np.int32)
    cnt = np.zeros(slots * ntiles, np.uint32) if ring_cnt is None else np.asarray(ring_cnt, np.uint32)
    bufs += [(20, ids.tobytes()), (21, cnt.tobytes()), (22, bytes(24)), (23, bytes(512))]
    head = struct.pack("<8sIiqqifQQ8i2i", b"SPKCKPT1", 1, model, n, width, delay, 1e-4, 1, 0,
                       ntiles, 0, 8, slots, 0, threads, 1, tile, len(bufs), 0)
    assert len(head) == 96
    out = head + first.tobytes()
    for i, b in bufs:
        out += struct.pack("<IQ", i, len(b)) + b
    return out


def test_restore_checks_contents_before_device_work(lib):
    """Corrupted edges, tilings a kernel cannot run and spike-ring entries outside their tile
    are refused with SPK_ERR_INVALID before the restore touches a device."""
    import ctypes as C

    import numpy as np

    n, width = 64, 32
    edges = np.full((n, width), np.iinfo(np.int32).max, np.int32)
    edges[:, 0], edges[:, 1] = 5, 9

    def restore(data):
        h = C.c_void_p()
        buf = (C.c_ubyte * len(data)).from_buffer_copy(data)
        return lib.spk_net_restore(C.byref(h), buf, len(data), 0), lib.spk_last_error()

    bad = edges.copy()
    bad[3, :2] = [9, 5]  # descending row
    rc, msg = restore(_checkpoint_bytes(bad, n, width))
    assert rc == spice_b200.ERR_INVALID and b"edges" in msg
    bad = edges.copy()
    bad[7, 1] = n  # target out of range
    rc, msg = restore(_checkpoint_bytes(bad, n, width))
    assert rc == spice_b200.ERR_INVALID and b"edges" in msg
    rc, msg = restore(_checkpoint_bytes(edges, n, width, threads=48, tile=48))  # not a multiple of 32
    assert rc == spice_b200.ERR_INVALID and b"tiling" in msg
    cnt = np.zeros(4, np.uint32)
    cnt[1] = 65  # more spikes than the tile has neurons
    rc, msg = restore(_checkpoint_bytes(edges, n, width, ring_cnt=cnt))
    assert rc == spice_b200.ERR_INVALID and b"spike ring" in msg
    cnt[1] = 2
    ids = np.zeros(4 * n, np.int32)
    ids[n:n + 2] = [3, 3]  # not ascending
    rc, msg = restore(_checkpoint_bytes(edges, n, width, ring_cnt=cnt, ring_ids=ids))
    assert rc == spice_b200.ERR_INVALID and b"spike ring" in msg


def test_user_model_build_exports_the_model():
    """A build with the tests' model compiled in (spice_b200.build.build_user) exposes it as
    model "user" with its attribute types; the default build rejects that id."""
    import subprocess
    import sys

    here = os.path.join(ROOT, "tests", "user_model")
    out = os.path.join(here, "libspice_b200_weighted_lif.so")
    sb_build.build_user(os.path.join(here, "weighted_lif.h"), "test_models::weighted_lif", out)
    env = dict(os.environ, SPICE_B200_LIB=out)
    r = subprocess.run([sys.executable, os.path.join(here, "check_weighted_lif.py"), "abi"], env=env,
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0 and "abi ok" in r.stdout, r.stdout + r.stderr
    with pytest.raises(spice_b200.InvalidArgument):
        spice_b200.model_attrs("user")
