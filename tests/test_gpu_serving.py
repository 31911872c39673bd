"""Serving loop (spk_server_*): jobs admitted against a device-memory budget and stepped by
continuous batching give the results of the same nets stepped alone; admission, refusal,
injected allocation failures, cancellation and deadlines are handled on the host."""
import time

import numpy as np
import pytest

import spice_b200
from spice_b200 import Layout, Server, Snn

pytestmark = pytest.mark.gpu

GB = 1 << 30


@pytest.fixture(autouse=True)
def _dev(gpu):
    yield


def bits_equal(a, b):
    return np.array_equal(np.asarray(a).view(np.uint32), np.asarray(b).view(np.uint32))


JOBS = [  # model, pops, conns, delay, steps (not multiples of the quantum)
    ("brunel", [4000, 4000], [(0, 1, 0.1), (1, 1, 0.1)], 15, 777),
    ("vogels_abbott", [6000], [(0, 0, 0.02)], 8, 1234),
    ("brunel_with_plasticity", [800, 800], [(0, 1, 0.1), (1, 1, 0.1)], 15, 500),
    ("vogels_abbott", [2000], [(0, 0, 0.02)], 1, 301),
    ("synth", [100_000], [(0, 0, 16 / 100_000)], 6, 950),
    ("brunel", [20_000, 20_000], [(0, 1, 0.05), (1, 1, 0.05)], 15, 2000),
]


def alone(model, pops, conns, delay, steps, seed):
    net = Snn(model, Layout(pops, conns), delay=delay, seed=seed, graph_seed=seed + 100)
    net.run(steps)
    out = net.neurons()
    net.close()
    return out


def test_jobs_in_a_mix_equal_jobs_alone():
    """The same job gives the same final state whether it runs alone or in a mix of
    jobs joining and leaving the batch at different ticks."""
    with Server(budget_bytes=40 * GB, quantum=200) as srv:
        ids = []
        for i, (model, pops, conns, delay, steps) in enumerate(JOBS):
            ids.append(srv.submit(model, Layout(pops, conns), steps, delay=delay, seed=i + 1, graph_seed=i + 101))
            time.sleep(0.02 * i)  # later jobs join a running batch
        srv.wait(timeout=300)
        for i, (model, pops, conns, delay, steps) in enumerate(JOBS):
            info = srv.info(ids[i])
            assert srv.state(ids[i]) == "done", info.message
            assert info.steps_done == steps and info.t_start >= info.t_submit and info.t_end > info.t_start
            for x, y in zip(srv.neurons(ids[i]), alone(model, pops, conns, delay, steps, i + 1)):
                assert bits_equal(x, y), model
        st = srv.stats()
        assert st["done"] == len(JOBS) and st["bytes_in_use"] == 0 and st["ticks"] > 1
        # the jobs ran together: some job started before another one ended
        infos = [srv.info(j) for j in ids]
        assert any(a.t_start < b.t_end and b.t_start < a.t_end for a in infos for b in infos if a is not b)


def test_budget_bounds_concurrency_and_refuses_oversized_jobs():
    lay = Layout([3000, 3000], [(0, 1, 0.1), (1, 1, 0.1)])
    need = spice_b200.estimate_bytes("brunel", lay, delay=15)
    budget = int(need * 1.5)  # one job at a time
    with Server(budget_bytes=budget, quantum=100) as srv:
        ids = [srv.submit("brunel", lay, 300, delay=15, seed=s) for s in range(4)]
        big = Layout([40_000, 40_000], [(0, 1, 0.1), (1, 1, 0.1)])
        with pytest.raises(spice_b200.SpiceError) as e:
            srv.submit("brunel", big, 100, delay=15)
        assert e.value.code == spice_b200.ERR_NOMEM
        srv.wait(timeout=120)
        st = srv.stats()
        assert st["done"] == 4 and st["refused"] == 1 and st["peak_bytes"] <= budget
        # one at a time: each job starts after the previous one ended
        infos = [srv.info(j) for j in ids]
        for a, b in zip(infos, infos[1:]):
            assert b.t_start >= a.t_end - 1e-6


def test_injected_allocation_failure_fails_one_job_only():
    lay = Layout([2000, 2000], [(0, 1, 0.1), (1, 1, 0.1)])
    with Server(budget_bytes=8 * GB, quantum=100) as srv:
        srv.inject_alloc_failures(1)
        a = srv.submit("brunel", lay, 200, delay=15, seed=1)
        srv.wait(a, timeout=60)
        b = srv.submit("brunel", lay, 200, delay=15, seed=1)
        srv.wait(timeout=60)
        ia = srv.info(a)
        assert srv.state(a) == "failed" and ia.error == spice_b200.ERR_NOMEM and b"injected" in ia.message
        assert srv.state(b) == "done"
        assert len(srv.neurons(b)[0]) == 4000
        assert srv.stats()["bytes_in_use"] == 0


def test_cancel_timeout_and_wait_limit():
    lay = Layout([5000, 5000], [(0, 1, 0.1), (1, 1, 0.1)])
    with Server(budget_bytes=8 * GB, quantum=50) as srv:
        long_job = srv.submit("brunel", lay, 10_000_000, delay=15, seed=1)
        with pytest.raises(spice_b200.SpiceError) as e:
            srv.wait(long_job, timeout=0.2)
        assert e.value.code == spice_b200.ERR_TIMEOUT
        srv.cancel(long_job)
        srv.wait(long_job, timeout=60)
        assert srv.state(long_job) == "cancelled"
        late = srv.submit("brunel", lay, 10_000_000, delay=15, seed=2, timeout=0.3)
        srv.wait(late, timeout=60)
        assert srv.state(late) == "timeout"
        with pytest.raises(spice_b200.InvalidArgument):
            srv.neurons(late)
        srv.release(late)
        with pytest.raises(spice_b200.InvalidArgument):
            srv.info(late)
        assert srv.stats()["bytes_in_use"] == 0


def test_injected_device_error_fails_one_job_only():
    """A job whose net reports a device error (its error word set, as a kernel's bounded wait
    that ran out sets it) fails with SPK_ERR_DEVICE; the jobs beside it, in the shared
    launches and on their own streams, complete with the results they have alone."""
    mix = [JOBS[0], JOBS[2], JOBS[4]]
    with Server(budget_bytes=40 * GB, quantum=100) as srv:
        ids = [srv.submit(m, Layout(p, c), steps, delay=d, seed=i + 1, graph_seed=i + 101)
               for i, (m, p, c, d, steps) in enumerate(mix)]
        victim = srv.submit("brunel", Layout([3000, 3000], [(0, 1, 0.1), (1, 1, 0.1)]), 5000, delay=15, seed=9)
        for _ in range(600):  # running, so that its net exists
            if srv.state(victim) == "running":
                break
            time.sleep(0.01)
        srv.inject_device_error(victim)
        srv.wait(timeout=300)
        iv = srv.info(victim)
        assert srv.state(victim) == "failed" and iv.error == spice_b200.ERR_DEVICE and b"device error flag 4" in iv.message
        for i, (m, p, c, d, steps) in enumerate(mix):
            assert srv.state(ids[i]) == "done", srv.info(ids[i]).message
            for x, y in zip(srv.neurons(ids[i]), alone(m, p, c, d, steps, i + 1)):
                assert bits_equal(x, y), m
        assert srv.stats()["bytes_in_use"] == 0
        with pytest.raises(spice_b200.InvalidArgument):
            srv.inject_device_error(victim)  # finished


SERVED = [  # the serving workload's shapes (bench.py serving_jobs): smallest and largest of each model
    ("vogels_abbott", lambda n: ([n], [(0, 0, 0.02)]), 8, [7071, 100_000]),
    ("brunel", lambda n: ([n // 2, n // 2], [(0, 1, 0.1), (1, 1, 0.1)]), 15, [4472, 63_245]),
    ("brunel_with_plasticity", lambda n: ([n // 2, n // 2], [(0, 1, 0.1), (1, 1, 0.1)]), 15, [4472, 63_245]),
]


@pytest.mark.parametrize("tile_target", [0, 4, 37])
def test_estimate_bounds_the_device_memory_a_net_holds(tile_target):
    """The estimate the server admits jobs by is an upper bound of every net's device memory,
    for each model, size and tiling of the serving mix, and of the mix test's jobs."""
    cases = [(m, *shape(n), d) for m, shape, d, ns in SERVED for n in ns]
    cases += [(m, p, c, d) for m, p, c, d, _ in JOBS]
    for model, pops, conns, delay in cases:
        lay = Layout(pops, conns)
        est = spice_b200.estimate_bytes(model, lay, delay=delay, tile_target=tile_target)
        net = Snn(model, lay, delay=delay, tile_target=tile_target)
        held = net.info().device_bytes
        net.close()
        assert held <= est, (model, pops, tile_target, held, est)
