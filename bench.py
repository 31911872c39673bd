"""Benchmark: wall-clock / biological-time ratio of a 1e9-synapse Brunel network on one B200
(the reference's headline, README.md:39 / samples/main.cpp:1337-1369: 100,000 steps of
0.1 ms = 10 s of biological time, setup excluded).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One bench "step" = 1,050 simulation steps (0.105 s biological, 70 windows of delay 15),
run through the public API (spk_net_run); the default K = 96 covers 10.08 s biological.
The 4.15 GB synapse table is far larger than L2, so no flush is needed between steps.
With N > 1 (torchrun), every rank simulates its own independent replica (the path does
not shard across GPUs on the single-GPU scope); value = max wall over ranks / total
biological time simulated by all ranks.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

POPS = [70710, 70710]                 # N = sqrt(1e9 / 0.05) = 141,420 (samples/main.cpp:1283,1395)
CONNS = [(0, 1, 0.1), (1, 1, 0.1)]
DT, DELAY = 1e-4, 15
SIM_STEPS = 1050                      # per bench step
METRIC = "wall/bio time ratio at 1e9-syn Brunel"


# single-net workloads: model, populations, connections, delay, synapses
MODEL_WORKLOADS = {
    "va": ("vogels_abbott", [5000], [(0, 0, 0.02)], 1, 5000 * 5000 * 0.02),
    "va_ns": ("vogels_abbott_ns", [5000], [(0, 0, 0.02)], 1, 5000 * 5000 * 0.02),
    "brunel_plus": ("brunel_with_plasticity", [50000, 50000], [(0, 1, 0.1), (1, 1, 0.1)], 15, 5e8),
    "brunel_plus_a012": ("brunel_with_plasticity_a012", [50000, 50000], [(0, 1, 0.1), (1, 1, 0.1)], 15, 5e8),
    "brunel_fixed": ("brunel_fixed", [70710, 70710], [(0, 1, 0.1), (1, 1, 0.1)], 15, 1e9),
    # the generic kernel (window_ordered: every arrival through receive(), in order) on nets
    # the counting kernels also run, for comparison with the va and --syn 1e8 lines
    # the reference's published single-GPU sizes (samples/main.cpp:1271-1294, results/bench.sh:26-28):
    # VA at 1e9 synapses (p = 0.02, delay 8) and the sparse synth net (p = 0.00156, delay 1)
    "va_1e9": ("vogels_abbott", [223607], [(0, 0, 0.02)], 8, 1e9),
    "synth_1e9": ("synth", [800641], [(0, 0, 0.00156)], 1, 1e9),
    "va_ordered": ("vogels_abbott", [5000], [(0, 0, 0.02)], 1, 5000 * 5000 * 0.02),
    "brunel_ordered": ("brunel", [22360, 22360], [(0, 1, 0.1), (1, 1, 0.1)], 15, 1e8),
}
WORKLOAD_OPTIONS = {"va_ordered": {"kernel": "ordered"}, "brunel_ordered": {"kernel": "ordered"}}
# the reference's published wall/bio for these workloads (its hardware, unstated)
PUBLISHED = {"va_1e9": (1.08669, "results/spice.json:127"), "synth_1e9": (1.39947, "results/spice.json:31"),
             "brunel_plus": (18.3537, "results/spice.json:367")}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=96)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--sim-steps", type=int, default=SIM_STEPS)
    ap.add_argument("--syn", type=float, default=1e9,
                    help="total synapses of the Brunel net (the benchmark is 1e9; smaller sizes serve profiling)")
    ap.add_argument("--workload", default="brunel", choices=["brunel", "batched", "serving"] + list(MODEL_WORKLOADS),
                    help="brunel: the 1e9 headline; batched: many small nets, batch vs plain per-net loop; "
                         "serving: Poisson job arrivals, server vs plain per-job loop; va: Vogels-Abbott 4000+1000 "
                         "at delay 1; brunel_plus: Brunel with STDP at 5e8 synapses; va_ns, brunel_fixed, "
                         "brunel_plus_a012: the same with the benchmark configurations' model constants; "
                         "va_ordered, brunel_ordered: VA and Brunel 1e8 on the generic window_ordered kernel; "
                         "va_1e9, synth_1e9: the reference's published 1e9-synapse VA (delay 8) and sparse synth "
                         "(delay 1) nets")
    ap.add_argument("--duration", type=float, default=8.0, help="serving: seconds of job arrivals")
    ap.add_argument("--rate", type=float, default=20.0, help="serving: job arrivals per second")
    ap.add_argument("--budget-gb", type=float, default=150.0, help="serving: device-memory budget")
    ap.add_argument("--quantum", type=int, default=600, help="serving: steps per tick")
    ap.add_argument("--nets", type=int, default=256, help="batched: number of nets")
    ap.add_argument("--bio", type=float, default=1.0, help="batched, va, brunel_plus: biological seconds per net")
    args = ap.parse_args()
    if args.syn != 1e9:
        # samples/main.cpp:1283,1395: N = sqrt(syn / 0.05), two populations of N / 2
        half = int((args.syn / 0.05) ** 0.5) // 2
        POPS[:] = [half, half]
    return args


def dist_init(n):
    """One process per GPU (torchrun's RANK / WORLD_SIZE / MASTER_*): NCCL with GPUs, gloo
    without (the CPU tests of the multi-rank plumbing)."""
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        backend = "nccl" if torch.cuda.is_available() else "gloo"
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=600))
    return rank, world


def barrier(world):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


def max_over_ranks(x, world):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist

    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


class Clocks:
    """nvidia-smi samples (SM clock, max clock, throttle reasons) during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.samples = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                          "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.samples.append([x.strip() for x in line.split(",")])

    def stop(self):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
        sm = [float(s[1]) for s in self.samples if len(s) > 2 and s[1].replace(".", "").isdigit()]
        mx = [float(s[2]) for s in self.samples if len(s) > 2 and s[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in self.samples if len(s) >= 9 for i in range(4) if s[5 + i].strip() == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def profile_traffic(syn):
    """DRAM bytes per simulated step of the window kernel from the committed ncu summary
    (bytes per captured launch / steps per captured launch), for the size it was captured
    at (1e9 synapses) only."""
    if syn != 1e9:
        return None
    path = os.path.join(ROOT, "profiles", "window_flat_brunel_1e9.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return float(d["dram_bytes_per_launch_full_size"]) / float(d["steps_per_launch"])
    except Exception:
        return None


L2_BYTES = 126e6


def net_config(syn, width, world):
    """The workload both arms run: the same keys in the GPU and the reference line."""
    n = sum(POPS)
    table = n * width * 4
    l2 = (f"inputs larger than L2 ({table / 1e9:.2f} GB synapse table)" if table > L2_BYTES
          else f"synapse table ({table / 1e6:.0f} MB) fits L2: no flush between steps")
    return {"workload": f"brunel_{syn:.0e}".replace("+0", ""), "neurons": n, "synapses": syn, "ell_width": width,
            "dt": DT, "delay": DELAY, "model": "brunel", "parallelism": f"replicas{world}", "l2": l2}


# CPU steps timed per sample: the reference's cpu::snn takes about 0.065 s per step of the
# 1e9 net at steady state on one core
CPU_SAMPLE_STEPS = 135
CPU_WARM_STEPS = 600  # reference arm: the activity settles within about 300 steps


def cpu_baseline(net):
    """The reference's cpu::snn (oracle/_ref, built with the reference's own -O2 -ffast-math)
    continuing the GPU net at its steady state: the GPU net's last `delay` steps are
    recorded and its graph and state handed to the reference (same clock, Poisson stream and
    spikes in flight), then both advance CPU_SAMPLE_STEPS steps. The reference's time on one
    core is the baseline; its raster and final state, compared with the GPU's, are the
    parity flag. Falls back to the CPU restatement (kind "port") where the reference build
    is absent. Returns (wall/bio, kind, cores, sample text, parity, spikes per step)."""
    import oracle

    counts, ids = net.run_record(DELAY)
    step0 = net.info().steps
    edges, width = net.adj()
    neurons = net.neurons()
    if oracle.have_reference(fast=True):
        cpu = oracle.ReferenceNet.from_state("brunel", edges, width, neurons, dt=DT, delay=DELAY, seed=1, fast=True,
                                             step0=step0, counts=counts, ids=ids)
        kind = "reference"
    else:
        cpu = oracle.OracleNet("brunel", POPS, CONNS, dt=DT, delay=DELAY, seed=1, edges=edges, width=width)
        cpu.set_state(neurons)
        cpu.set_progress(step0, counts, ids)
        kind = "port"
    del edges
    gc, gi = net.run_record(CPU_SAMPLE_STEPS)
    off = np.concatenate([[0], np.cumsum(gc)]).astype(np.int64)
    parity = True
    t0 = time.perf_counter()
    spikes = 0
    for k in range(CPU_SAMPLE_STEPS):
        s = cpu.step()
        spikes += len(s)
        parity = parity and np.array_equal(s, gi[off[k]:off[k + 1]])
    wall = time.perf_counter() - t0
    for a, b in zip(net.neurons(), cpu.neurons()):
        parity = parity and np.array_equal(a.view(np.uint32), b.view(np.uint32))
    del cpu
    ratio = wall / (CPU_SAMPLE_STEPS * DT)
    sample = (f"Brunel {sum(POPS):,} neurons, {CPU_SAMPLE_STEPS} steps continuing the GPU net at steady state "
              f"(steps {step0}-{step0 + CPU_SAMPLE_STEPS - 1}, {spikes / CPU_SAMPLE_STEPS:.0f} spikes per step), single thread, "
              f"graph and state import excluded")
    return ratio, kind, 1, sample, bool(parity), spikes / CPU_SAMPLE_STEPS


REF_SIM_STEPS = 20  # simulation steps timed per reference-arm bench step


def run_reference(args, rank, world):
    """The reference's CPU simulator on the same workload, rank 0 only: the reference's
    cpu::snn builds the net from its own layout and generator, runs CPU_WARM_STEPS untimed
    steps past the initial transient, then each bench step times REF_SIM_STEPS steps
    (setup excluded, like the reference)."""
    if rank != 0:
        return
    import oracle

    t0 = time.perf_counter()
    if oracle.have_reference(fast=True):
        net, kind = oracle.ReferenceNet("brunel", POPS, CONNS, dt=DT, delay=DELAY, seed=1, fast=True), "reference"
    else:
        net, kind = oracle.OracleNet("brunel", POPS, CONNS, dt=DT, delay=DELAY, seed=1, graph="reference",
                                     graph_seed=1337), "port"
    setup = time.perf_counter() - t0
    for _ in range(CPU_WARM_STEPS):
        net.step()
    vals, spikes = [], 0
    for i in range(args.warmup + args.steps):
        t = time.perf_counter()
        for _ in range(REF_SIM_STEPS):
            c = len(net.step())
            if i >= args.warmup:
                spikes += c
        if i >= args.warmup:
            vals.append((time.perf_counter() - t) / (REF_SIM_STEPS * DT))
    value = statistics.median(vals) if vals else None
    first = CPU_WARM_STEPS + args.warmup * REF_SIM_STEPS
    sps = spikes / max(1, args.steps * REF_SIM_STEPS)
    sample = (f"Brunel {sum(POPS):,} neurons, {REF_SIM_STEPS} steps per bench step x {args.steps} (steps {first}-"
              f"{first + args.steps * REF_SIM_STEPS - 1}, after {CPU_WARM_STEPS} steps past the initial transient; "
              f"{sps:.0f} spikes per step), single thread (cpu::snn has no threading), setup {setup:.1f} s excluded")
    line = {"metric": METRIC, "value": value, "unit": "wall_s/bio_s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": value * REF_SIM_STEPS * DT * 1e3 if value else None,
            "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "impl": "reference", "config": net_config(args.syn, int(net.width), world),
            "sim_steps_per_bench_step": REF_SIM_STEPS, "spikes_per_step": sps,
            "cpu_baseline": {"value": value, "unit": "wall_s/bio_s", "cores": 1, "kind": kind, "sample": sample},
            "e2e": {"value": value, "unit": "wall_s/bio_s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_ours(args, rank, world):
    import torch

    from spice_b200 import Layout, Snn

    dev = int(os.environ.get("LOCAL_RANK", 0))
    torch.cuda.set_device(dev)
    t0 = time.perf_counter()
    net = Snn("brunel", Layout(POPS, CONNS), dt=DT, delay=DELAY, seed=1 + rank, graph_seed=1337 + rank, device=dev)
    net.sync()
    setup_s = time.perf_counter() - t0
    info = net.info()
    stream = torch.cuda.ExternalStream(net.stream(), device=dev)
    S = args.sim_steps

    for _ in range(args.warmup):
        net.run(S)
    net.sync()
    # spike rate from a recorded (untimed) sample, for the algorithmic byte count
    counts, _ = net.run_record(S)
    spikes_per_step = float(np.mean(counts))
    net.sync()

    barrier(world)
    torch.cuda.synchronize()
    launches0 = net.info().kernel_launches
    clocks = Clocks(dev)
    clocks.start()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(args.steps):
        net.run(S)
    ev1.record(stream)
    ev1.synchronize()
    torch.cuda.synchronize()
    clk = clocks.stop()
    launches = net.info().kernel_launches - launches0
    persistent = bool(net.info().persistent)
    barrier(world)
    ms = ev0.elapsed_time(ev1)
    ms_max = max_over_ranks(ms, world)

    # end to end through the C ABI: spike raster of every bench step to host memory
    e2e_vals, d2h = [], []
    for _ in range(max(1, min(args.steps, 10))):
        t = time.perf_counter()
        c, ids = net.run_record(S)
        e2e_vals.append(time.perf_counter() - t)
        d2h.append(c.nbytes + ids.nbytes)
    e2e_wall = max_over_ranks(statistics.median(e2e_vals), world)

    bio = args.steps * S * DT
    value = (ms_max / 1e3) / (bio * world)
    # roofline of the window kernel (the only kernel of the timed region), algorithmic bytes
    # per step as the path defines them: every arriving synapse's 4-byte index, one 4-byte
    # pivot per (spike, tile), the neuron state read and written by propagation and by the
    # update, and the spike ids
    n = sum(POPS)
    mean_degree = sum(POPS[a] * p * POPS[b] for a, b, p in CONNS) / n
    state_bytes = 8  # V, Twait
    bytes_per_step = (spikes_per_step * mean_degree * 4 + spikes_per_step * info.num_tiles * 4 + 4 * n * state_bytes
                      + spikes_per_step * 4)
    steps_per_launch = args.steps * S / launches
    bytes_per_launch = steps_per_launch * bytes_per_step
    t_launch = (ms / 1e3) / launches
    peak, peak_kind = measured_peaks()
    achieved = bytes_per_launch / t_launch / 1e9
    traffic_per_step = profile_traffic(args.syn)
    traffic = traffic_per_step * steps_per_launch if traffic_per_step else None
    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": "wall_s/bio_s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": False, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": net_config(args.syn, int(info.width), world),
                "sim_steps_per_bench_step": S, "spikes_per_step": spikes_per_step, "setup_s": setup_s,
                "tiles": info.num_tiles, "tile_size": info.tile_size,
                "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                             "traffic": traffic, "peak_kind": peak_kind, "kernel": "window_flat<brunel>",
                             "bytes_per_launch": bytes_per_launch, "launch_us": t_launch * 1e6,
                             "steps_per_launch": steps_per_launch, "persistent": persistent,
                             "bytes_per_step": bytes_per_step},
                "e2e": {"value": e2e_wall / (S * DT * world), "unit": "wall_s/bio_s", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": int(statistics.median(d2h))},
                "gpu_launches": launches, "clocks": clk}
        if world == 1 and not args.no_cpu_baseline:
            try:
                v, kind, cores, sample, parity, cpu_sps = cpu_baseline(net)
                line["cpu_baseline"] = {"value": v, "unit": "wall_s/bio_s", "cores": cores, "kind": kind, "sample": sample,
                                        "spikes_per_step": cpu_sps}
                line["parity"] = parity
            except Exception as e:  # report, never fail the GPU line
                line["cpu_baseline"] = {"value": None, "unit": "wall_s/bio_s", "cores": 1, "kind": "reference",
                                        "sample": f"unavailable: {e}"}
        print(json.dumps(line), flush=True)
    net.close()


BATCH_MODELS = ("vogels_abbott", "brunel", "brunel_with_plasticity")


def batched_specs(count, seed=0):
    """Nets drawn uniformly from {VA, Brunel, Brunel+} with synapse counts log-uniform in
    1e5-5e7; N = sqrt(syn / p_eff) with p_eff 0.02 (VA layout{N, 0.02}) and 0.05 (Brunel's
    two populations of N/2 at p = 0.1 into the second), delay 8 (VA, the published runs)
    and 15 (Brunel, Brunel+); seeds 1..count."""
    rng = np.random.default_rng(seed)
    specs = []
    for i in range(count):
        model = BATCH_MODELS[int(rng.integers(0, 3))]
        syn = float(np.exp(rng.uniform(np.log(1e5), np.log(5e7))))
        if model == "vogels_abbott":
            n = max(64, int((syn / 0.02) ** 0.5))
            pops, conns, delay = [n], [(0, 0, 0.02)], 8
        else:
            half = max(32, int((syn / 0.05) ** 0.5) // 2)
            pops, conns, delay = [half, half], [(0, 1, 0.1), (1, 1, 0.1)], 15
        specs.append({"model": model, "pops": pops, "conns": conns, "delay": delay, "seed": i + 1, "syn": syn})
    return specs


def run_batched(args, rank, world):
    """Batched workload: the same nets stepped (a) one at a time, the plain per-job loop
    (spice_bench/paper_plots.cpp:184-231 steps one net after another), and (b) together in
    one Batch. Setup is excluded from both; each arm's wall time is taken on the host from
    an idle, synchronised GPU until every net has synchronised again (the batch spans many
    streams). Reports both and the ratio."""
    import torch

    from spice_b200 import Batch, Layout, Snn

    dev = int(os.environ.get("LOCAL_RANK", 0))
    torch.cuda.set_device(dev)
    specs = batched_specs(args.nets)
    steps = int(round(args.bio / DT))
    sms = torch.cuda.get_device_properties(dev).multi_processor_count

    def make(s):
        return Snn(s["model"], Layout(s["pops"], s["conns"]), dt=DT, delay=s["delay"], seed=s["seed"],
                   graph_seed=1000 + s["seed"], device=dev)

    # (a) plain loop: each net alone, its own default tiling, one after another
    t0 = time.perf_counter()
    plain = [make(s) for s in specs]
    for n in plain:
        n.sync()
    setup_plain = time.perf_counter() - t0
    torch.cuda.synchronize()
    clocks = Clocks(dev)
    clocks.start()
    per_model = {m: 0.0 for m in BATCH_MODELS}
    t0 = time.perf_counter()
    for n, s in zip(plain, specs):
        t = time.perf_counter()
        n.run(steps)
        n.sync()
        per_model[s["model"]] += time.perf_counter() - t
    wall_plain = time.perf_counter() - t0
    syn_total = sum(n.num_synapses() for n in plain)
    for n in plain:
        n.close()
    del plain

    # (b) batch: tiles per net by work share at the scale the autotuner measured best
    from spice_b200.autotune import autotune, autotune_producers, layout_work, tile_targets as targets_for

    works = [layout_work(Layout(s["pops"], s["conns"])) for s in specs]

    def build(i, t):
        n = make(specs[i])
        n.set_tile_target(t)
        return n

    t0 = time.perf_counter()
    scale, buckets, tune_times = autotune(build, works, sms, device=dev)
    prod, prod_times = autotune_producers(build, works, sms, scale, buckets, device=dev)
    tune_times.update(prod_times)
    tune_s = time.perf_counter() - t0
    t0 = time.perf_counter()
    nets = [make(s) for s in specs]
    batch = Batch(device=dev)
    for n, t, b in zip(nets, targets_for(works, sms, scale, buckets), buckets):
        n.set_tile_target(t)
        n.set_producer_warps(prod[b])
        batch.add(n)
    for n in nets:
        n.sync()
    setup_batch = time.perf_counter() - t0
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    batch.run(steps)
    for n in nets:
        n.sync()
    wall_batch = time.perf_counter() - t0
    clk = clocks.stop()
    tiles = sum(n.info().num_tiles for n in nets)
    batch.close()
    for n in nets:
        n.close()

    bio_total = len(specs) * steps * DT
    if rank == 0:
        counts = {m: sum(1 for s in specs if s["model"] == m) for m in BATCH_MODELS}
        line = {"metric": "batched synapse-seconds per wall second", "value": syn_total * steps * DT / wall_batch,
                "unit": "syn*bio_s/s", "n_gpus": 1, "steps": 1, "warmup": 0, "ms_per_step": wall_batch * 1e3,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": {"workload": f"batched_{len(specs)}_nets", "nets": counts, "synapses_total": syn_total,
                           "syn_range": [1e5, 5e7], "bio_s_per_net": steps * DT, "dt": DT, "tiles_total": tiles},
                "batch": {"wall_s": wall_batch, "wall_per_bio": wall_batch / bio_total, "setup_s": setup_batch,
                          "tile_scale": scale, "producer_warps": prod, "autotune_s": tune_s,
                          "autotune_ms_per_step": {k: v * 1e3 for k, v in tune_times.items()}},
                "plain_loop": {"wall_s": wall_plain, "wall_per_bio": wall_plain / bio_total, "setup_s": setup_plain,
                               "wall_s_by_model": per_model,
                               "value": syn_total * steps * DT / wall_plain},
                "speedup_vs_plain_loop": wall_plain / wall_batch, "clocks": clk}
        print(json.dumps(line), flush=True)


def serving_jobs(rate, duration, seed=0):
    """Poisson arrivals at `rate` jobs/s over `duration` s; models uniform over {VA, Brunel,
    Brunel+}, synapses log-uniform in 1e6-2e8, biological time uniform in 0.1-2 s."""
    rng = np.random.default_rng(seed)
    t, jobs = 0.0, []
    while True:
        t += float(rng.exponential(1.0 / rate))
        if t >= duration:
            break
        model = BATCH_MODELS[int(rng.integers(0, 3))]
        syn = float(np.exp(rng.uniform(np.log(1e6), np.log(2e8))))
        bio = float(rng.uniform(0.1, 2.0))
        if model == "vogels_abbott":
            n = int((syn / 0.02) ** 0.5)
            pops, conns, delay = [n], [(0, 0, 0.02)], 8
        else:
            half = int((syn / 0.05) ** 0.5) // 2
            pops, conns, delay = [half, half], [(0, 1, 0.1), (1, 1, 0.1)], 15
        jobs.append({"t": t, "model": model, "pops": pops, "conns": conns, "delay": delay, "syn": syn,
                     "steps": int(round(bio / DT)), "seed": len(jobs) + 1})
    return jobs


def run_serving(args, rank, world):
    """Serving workload: the same seeded job arrivals served (a) by the plain per-job loop
    (build, run and free one net at a time in arrival order, spice_bench/paper_plots.cpp:184-231)
    and (b) by Server (admission against the budget, continuous batching). Latency = job
    completion minus arrival; throughput = synapses x biological seconds of all jobs per wall
    second from the first arrival to the last completion."""
    import torch

    from spice_b200 import Layout, Server, Snn

    dev = int(os.environ.get("LOCAL_RANK", 0))
    torch.cuda.set_device(dev)
    jobs = serving_jobs(args.rate, args.duration)
    work = sum(j["syn"] * j["steps"] * DT for j in jobs)
    syn_steps = sum(j["syn"] * j["steps"] for j in jobs)  # synapse updates: every synapse every step

    def pct(x, q):
        return float(np.percentile(np.asarray(x), q)) if x else None

    clocks = Clocks(dev)
    clocks.start()
    # (a) plain loop, real time
    lat_plain, build_plain = [], 0.0
    run_plain = {m: 0.0 for m in BATCH_MODELS}
    t0 = time.perf_counter()
    for j in jobs:
        now = time.perf_counter() - t0
        if now < j["t"]:
            time.sleep(j["t"] - now)
        tb = time.perf_counter()
        net = Snn(j["model"], Layout(j["pops"], j["conns"]), dt=DT, delay=j["delay"], seed=j["seed"],
                  graph_seed=1000 + j["seed"], device=dev)
        net.sync()
        tr = time.perf_counter()
        build_plain += tr - tb
        net.run(j["steps"])
        net.sync()
        run_plain[j["model"]] += time.perf_counter() - tr
        net.close()
        lat_plain.append(time.perf_counter() - t0 - j["t"])
    span_plain = time.perf_counter() - t0

    # (b) server, real time
    srv = Server(budget_bytes=int(args.budget_gb * 1e9), quantum=args.quantum, device=dev)
    ids = []
    t0 = time.perf_counter()
    for j in jobs:
        now = time.perf_counter() - t0
        if now < j["t"]:
            time.sleep(j["t"] - now)
        ids.append(srv.submit(j["model"], Layout(j["pops"], j["conns"]), j["steps"], dt=DT, delay=j["delay"],
                              seed=j["seed"], graph_seed=1000 + j["seed"]))
    srv.wait(timeout=1800)
    infos = [srv.info(i) for i in ids]
    st = srv.stats()
    srv.close()
    clk = clocks.stop()
    states = [i.state for i in infos]
    failures = {}  # "state error: message" of every job that did not complete, with counts
    for i in infos:
        if i.state != 2:
            key = f"{i.state} {i.error}: {i.message.decode(errors='replace')}"
            failures[key] = failures.get(key, 0) + 1
    lat = [i.t_end - i.t_submit for i in infos if i.state == 2]
    first = min(i.t_submit for i in infos)
    span = max(i.t_end for i in infos) - first
    if rank == 0:
        counts = {m: sum(1 for j in jobs if j["model"] == m) for m in BATCH_MODELS}
        line = {"metric": "served synapse-seconds per wall second", "value": work / span, "unit": "syn*bio_s/s",
                "n_gpus": 1, "steps": 1, "warmup": 0, "ms_per_step": span * 1e3, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": {"workload": f"serving_poisson_{args.rate:g}_per_s", "jobs": len(jobs), "models": counts,
                           "syn_range": [1e6, 2e8], "bio_range_s": [0.1, 2.0], "arrival_s": args.duration,
                           "budget_gb": args.budget_gb, "quantum_steps": args.quantum},
                "server": {"p50_s": pct(lat, 50), "p99_s": pct(lat, 99), "span_s": span, "done": states.count(2),
                           "not_done": failures,
                           "sims_per_s": states.count(2) / span, "synapse_steps_per_s": syn_steps / span,
                           "peak_gb": st["peak_bytes"] / 1e9, "ticks": st["ticks"],
                           "build_s": st["build_seconds"], "tick_s": st["tick_seconds"]},
                "plain_loop": {"p50_s": pct(lat_plain, 50), "p99_s": pct(lat_plain, 99), "span_s": span_plain,
                               "value": work / span_plain, "sims_per_s": len(jobs) / span_plain,
                               "synapse_steps_per_s": syn_steps / span_plain, "build_s": build_plain,
                               "run_s_by_model": run_plain},
                "speedup_vs_plain_loop": span_plain / span, "clocks": clk}
        print(json.dumps(line), flush=True)


def run_model_workload(args, rank, world):
    """Vogels-Abbott (4,000 + 1,000 neurons, p = 0.02, delay 1; the reference's CPU-runnable
    case) or Brunel+ (N = 100,000, 5e8 synapses, delay 15, lazy STDP): wall/bio through
    spk_net_run, the raster through spk_net_run_record (e2e), and the reference's cpu::snn on
    one core (the whole second for VA; a small Brunel+ net, since its CPU STDP sweep touches
    every synapse every step)."""
    import torch

    from spice_b200 import Layout, Snn

    dev = int(os.environ.get("LOCAL_RANK", 0))
    torch.cuda.set_device(dev)
    model, pops, conns, delay, syn = MODEL_WORKLOADS[args.workload]
    steps = int(round(args.bio / DT))
    t0 = time.perf_counter()
    options = WORKLOAD_OPTIONS.get(args.workload)
    net = Snn(model, Layout(pops, conns), dt=DT, delay=delay, seed=1 + rank, graph_seed=1337 + rank, device=dev,
              options=options)
    net.sync()
    setup_s = time.perf_counter() - t0
    stream = torch.cuda.ExternalStream(net.stream(), device=dev)
    for _ in range(max(3, args.warmup)):
        net.run(max(delay, 15))
    net.sync()
    barrier(world)
    clocks = Clocks(dev)
    clocks.start()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    net.run(steps)
    ev1.record(stream)
    ev1.synchronize()
    clk = clocks.stop()
    ms = max_over_ranks(ev0.elapsed_time(ev1), world)
    t = time.perf_counter()
    counts, ids = net.run_record(steps, cap=sum(pops) * steps // 20 + 1024)
    e2e = max_over_ranks(time.perf_counter() - t, world)
    info = net.info()
    net.close()
    kernel = " on window_ordered" if options and options.get("kernel") == "ordered" else ""
    line = {"metric": f"wall/bio time ratio, {model}{kernel}", "value": ms / 1e3 / (steps * DT), "unit": "wall_s/bio_s",
            "n_gpus": world, "steps": 1, "warmup": max(3, args.warmup), "ms_per_step": ms, "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": args.workload, "neurons": sum(pops), "synapses": syn, "delay": delay, "dt": DT,
                       "bio_s": steps * DT, "sim_steps": steps, "setup_s": setup_s, "persistent": bool(info.persistent),
                       "tiles": info.num_tiles, "spikes_per_step": float(np.mean(counts))},
            "e2e": {"value": e2e / (steps * DT), "unit": "wall_s/bio_s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": int((counts.nbytes + ids.nbytes) / 1)},
            "gpu_launches": info.kernel_launches, "clocks": clk}
    rates = {}
    if counts.sum():
        n = sum(pops)
        groups = {"exc": (0, int(0.8 * n)), "inh": (int(0.8 * n), n)} if model.startswith("vogels") else \
                 {"all": (0, n)} if model == "synth" else \
                 {"poisson": (0, n // 2), "exc": (n // 2, int(0.9 * n)), "inh": (int(0.9 * n), n)}
        hist = np.bincount(ids, minlength=n)
        rates = {k: float(hist[a:b].sum()) / (b - a) / (steps * DT) for k, (a, b) in groups.items()}
    line["rates_hz"] = rates
    if args.workload in PUBLISHED:
        v, src = PUBLISHED[args.workload]
        line["reference_published"] = {"value": v, "unit": "wall_s/bio_s", "source": src}
    if rank == 0 and not args.no_cpu_baseline:
        import oracle

        small = syn > 1e7  # the CPU runs the full net only where it finishes in seconds
        reference_model = model in oracle.REFERENCE_MODELS
        fast = oracle.have_reference(fast=True) and reference_model
        cpu_pops = ([2000, 2000] if len(pops) == 2 else [4000]) if small else pops
        cpu_steps = 200 if small else steps
        mk = (lambda: oracle.ReferenceNet(model, cpu_pops, conns, dt=DT, delay=delay, seed=1, fast=True)) if fast else \
             (lambda: oracle.OracleNet(model, cpu_pops, conns, dt=DT, delay=delay, seed=1, graph="reference", graph_seed=1337))
        cpu = mk()
        t = time.perf_counter()
        for _ in range(cpu_steps):
            cpu.step()
        wall = time.perf_counter() - t
        line["cpu_baseline"] = {"value": wall / (cpu_steps * DT), "unit": "wall_s/bio_s", "cores": 1,
                                "kind": "reference" if fast else "port",
                                "sample": f"{model} N={sum(cpu_pops)}, {cpu_steps} steps, single thread"
                                          + (" (small N: the full net takes minutes per step on one core)" if small else "")
                                          + ("" if reference_model else " (the reference has no such model: the port runs it)")}
    if rank == 0:
        print(json.dumps(line), flush=True)


def main():
    args = parse()
    rank, world = dist_init(args.gpus)
    try:
        if args.impl == "reference":
            run_reference(args, rank, world)
        elif args.workload == "batched":
            run_batched(args, rank, world)
        elif args.workload == "serving":
            run_serving(args, rank, world)
        elif args.workload in MODEL_WORKLOADS:
            run_model_workload(args, rank, world)
        else:
            run_ours(args, rank, world)
    finally:
        if world > 1:
            import torch.distributed as dist

            dist.destroy_process_group()


if __name__ == "__main__":
    main()
