"""The multi-rank plumbing of bench.py (one process per GPU; replicas only: the path does not
shard) on CPU: two gloo ranks agree on the max over ranks, meet at barriers, and the
reference arm runs on rank 0 alone; and the serving workload's seeded job stream."""
import os
import socket

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import sys

    sys.path.insert(0, ROOT)
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import bench
    import torch.distributed as dist

    r, w = bench.dist_init(world)
    assert (r, w) == (rank, world) and dist.get_backend() == "gloo"
    m = bench.max_over_ranks(1.5 + rank, w)
    bench.barrier(w)
    # the reference arm: rank 0 alone works; the others return at once
    ran = rank == 0 or bench.run_reference(None, r, w) is None
    bench.barrier(w)
    dist.destroy_process_group()
    out.put((rank, m, ran))


def test_two_gloo_ranks_max_and_barrier():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=10) for _ in range(2))
    assert [r[1] for r in res] == [2.5, 2.5] and all(r[2] for r in res)


def test_serving_saturation_runs_the_same_jobs():
    """The serving workload at saturation (--rate 1000 --duration 0.16) submits the very
    jobs of the 20 jobs/s run (--rate 20 --duration 8), only sooner: the arrival gaps scale
    with 1/rate while every other draw comes from the same seeded stream."""
    import sys

    sys.path.insert(0, ROOT)
    import bench

    slow, fast = bench.serving_jobs(20.0, 8.0), bench.serving_jobs(1000.0, 0.16)
    assert len(slow) == len(fast) == 144
    for a, b in zip(slow, fast):
        assert abs(a["t"] / 50.0 - b["t"]) < 1e-9
        assert {k: v for k, v in a.items() if k != "t"} == {k: v for k, v in b.items() if k != "t"}
