"""spice_b200 -- Python binding of the B200 simulation path (libspice_b200.so, C ABI in
include/spice_b200.h).

Mirrors the reference's interface (spice/snn.h, spice/cuda/snn.h, spice/util/layout.h):

    from spice_b200 import Layout, Snn
    net = Snn("brunel", Layout([70710, 70710], [(0, 1, 0.1), (1, 1, 0.1)]), dt=1e-4, delay=15)
    spikes = net.step(out=True)          # snn::step(std::vector<int>*)
    net.run(100_000)                     # 100k x step(nullptr): one persistent launch or graph windows
    edges, width = net.adj()             # snn::adj()
    V, Twait = net.neurons()             # snn::neurons() as structure of arrays

The compute path is the CUDA library only: importing this module without the built
library, or constructing a net without a GPU, raises.
"""
import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
# SPICE_B200_LIB selects another build of the library: one with a model of the user's
# compiled in (spice_b200.build.build_user), reached as model "user"
LIB_PATH = os.environ.get("SPICE_B200_LIB") or os.path.join(_HERE, "libspice_b200.so")

MODELS = {"vogels_abbott": 0, "brunel": 1, "brunel_with_plasticity": 2, "synth": 3,
          # the benchmark configurations' constants (include/spice/models/*.h)
          "vogels_abbott_ns": 4, "brunel_fixed": 5, "brunel_with_plasticity_a012": 6,
          # SPK_USER_MODEL_ID: present in user builds only
          "user": 7}
MODEL_NAMES = {v: k for k, v in MODELS.items()}

OK, ERR_INVALID, ERR_CUDA, ERR_NOMEM, ERR_DEVICE, ERR_CAPACITY, ERR_TIMEOUT = range(7)


class SpiceError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"[{code}] {msg}")
        self.code = code


class InvalidArgument(SpiceError, ValueError):
    pass


class CapacityError(SpiceError):
    pass


class _LayoutDesc(C.Structure):
    _fields_ = [
        ("npops", C.c_int),
        ("pops", C.POINTER(C.c_uint64)),
        ("nconn", C.c_int),
        ("conn_src", C.POINTER(C.c_int)),
        ("conn_dst", C.POINTER(C.c_int)),
        ("conn_p", C.POINTER(C.c_float)),
    ]


class NetInfo(C.Structure):
    _fields_ = [
        ("model", C.c_int),
        ("device", C.c_int),
        ("num_neurons", C.c_uint64),
        ("num_synapses", C.c_uint64),
        ("width", C.c_uint64),
        ("delay", C.c_int),
        ("dt", C.c_float),
        ("steps", C.c_uint64),
        ("tile_size", C.c_uint64),
        ("num_tiles", C.c_uint64),
        ("device_bytes", C.c_uint64),
        ("kernel_launches", C.c_uint64),
        ("persistent", C.c_int),
        ("slice_pack", C.c_int),
        ("slot_vecs", C.c_int),
    ]


class JobInfo(C.Structure):  # spk_job_info
    _fields_ = [
        ("state", C.c_int),
        ("error", C.c_int),
        ("steps_done", C.c_uint64),
        ("steps_total", C.c_uint64),
        ("num_neurons", C.c_uint64),
        ("device_bytes", C.c_uint64),
        ("t_submit", C.c_double),
        ("t_start", C.c_double),
        ("t_end", C.c_double),
        ("message", C.c_char * 160),
    ]


class ServerStats(C.Structure):  # spk_server_stats
    _fields_ = [(k, C.c_uint64) for k in ("queued", "running", "done", "failed", "cancelled", "timed_out", "refused",
                                          "bytes_in_use", "peak_bytes", "budget_bytes", "ticks")] + [
        ("build_seconds", C.c_double), ("tick_seconds", C.c_double)]


JOB_STATES = ("queued", "running", "done", "failed", "cancelled", "timeout", "refused")

class _NetOptions(C.Structure):
    _fields_ = [(f, C.c_int) for f in ("tile_target", "kernel", "slice_bits", "tiling", "persistent", "pipelined", "slots")]


# build choices (spk_net_options): name -> (field, {value: int})
_OPTION_VALUES = {
    "kernel": {"window": 0, "direct": 1, "ordered": 2},
    "slice_bits": {10: 10, 16: 16},
    "tiling": {"balanced": 0, "uniform": 1},
    "persistent": {False: 0, True: 1},
    "pipelined": {False: 0, True: 1},
    "slots": {False: 0, True: 1},
}


def net_options(tile_target=0, **choices):
    """spk_net_options from keyword choices (kernel="window"|"direct"|"ordered", slice_bits=10|16,
    tiling="balanced"|"uniform", persistent=bool, pipelined=bool, slots=bool); a choice
    left out is automatic."""
    o = _NetOptions()
    library().spk_net_options_init(C.byref(o))
    if int(tile_target) < 0:
        raise InvalidArgument(ERR_INVALID, "tile target must be >= 0")
    o.tile_target = int(tile_target)
    for k, v in choices.items():
        if k not in _OPTION_VALUES:
            raise InvalidArgument(ERR_INVALID, f"unknown net option {k!r}")
        if v is None:
            continue
        table = _OPTION_VALUES[k]
        if v not in table:
            raise InvalidArgument(ERR_INVALID, f"net option {k}={v!r} is not one of {list(table)}")
        setattr(o, k, table[v])
    return o


_lib = None


def library():
    """The loaded libspice_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with `python -m spice_b200.build`")
    lib = C.CDLL(LIB_PATH)
    P, U64, I, F, VP = C.POINTER, C.c_uint64, C.c_int, C.c_float, C.c_void_p
    sig = {
        "spk_last_error": (C.c_char_p, []),
        "spk_layout_flatten": (I, [P(_LayoutDesc), P(I), P(F), I, P(I), P(U64), P(U64)]),
        "spk_generate_adj_list": (I, [VP, P(_LayoutDesc), U64, VP]),
        "spk_generate_adj_list_static": (I, [VP, P(_LayoutDesc), U64, VP]),
        "spk_net_create": (I, [P(VP), I, P(_LayoutDesc), F, I, U64, U64, I]),
        "spk_net_create_from_adj": (I, [P(VP), I, VP, U64, U64, F, I, U64, I]),
        "spk_net_set_neurons": (I, [VP, P(VP)]),
        "spk_net_set_synapses": (I, [VP, P(VP)]),
        "spk_net_destroy": (I, [VP]),
        "spk_net_step": (I, [VP, VP, U64, P(U64)]),
        "spk_net_run": (I, [VP, U64]),
        "spk_net_run_record": (I, [VP, U64, VP, VP, U64, P(U64)]),
        "spk_net_sync": (I, [VP]),
        "spk_net_stream": (I, [VP, P(VP)]),
        "spk_net_get_info": (I, [VP, P(NetInfo)]),
        "spk_net_adj": (I, [VP, VP, U64]),
        "spk_net_neurons": (I, [VP, P(VP)]),
        "spk_net_synapses": (I, [VP, P(VP)]),
        "spk_model_attrs": (I, [I, P(I), P(I), C.c_char_p, I]),
        "spk_net_set_tile_target": (I, [VP, I]),
        "spk_net_set_producer_warps": (I, [VP, I]),
        "spk_net_checkpoint": (I, [VP, VP, U64, P(U64)]),
        "spk_net_restore": (I, [P(VP), VP, U64, I]),
        "spk_net_create_ex": (I, [P(VP), I, P(_LayoutDesc), F, I, U64, U64, I, I]),
        "spk_net_estimate_bytes": (I, [I, P(_LayoutDesc), I, I, I, P(U64)]),
        "spk_net_options_init": (None, [P(_NetOptions)]),
        "spk_net_create_opts": (I, [P(VP), I, P(_LayoutDesc), F, I, U64, U64, I, P(_NetOptions)]),
        "spk_net_estimate_bytes_opts": (I, [I, P(_LayoutDesc), I, I, P(_NetOptions), P(U64)]),
        "spk_batch_run_nets": (I, [VP, I, P(VP), P(U64)]),
        "spk_server_create": (I, [P(VP), I, U64, U64]),
        "spk_server_create_ex": (I, [P(VP), I, U64, U64, I]),
        "spk_server_submit": (I, [VP, I, P(_LayoutDesc), F, I, U64, U64, U64, C.c_double, P(U64)]),
        "spk_server_job_info": (I, [VP, U64, P(JobInfo)]),
        "spk_server_job_neurons": (I, [VP, U64, P(VP)]),
        "spk_server_cancel": (I, [VP, U64]),
        "spk_server_release": (I, [VP, U64]),
        "spk_server_wait": (I, [VP, U64, C.c_double]),
        "spk_server_get_stats": (I, [VP, P(ServerStats)]),
        "spk_server_inject_alloc_failures": (I, [VP, I]),
        "spk_server_inject_device_error": (I, [VP, U64]),
        "spk_server_destroy": (I, [VP]),
        "spk_batch_create": (I, [P(VP), I]),
        "spk_batch_add": (I, [VP, VP]),
        "spk_batch_remove": (I, [VP, VP]),
        "spk_batch_run": (I, [VP, U64]),
        "spk_batch_destroy": (I, [VP]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _lib = lib
    return lib


def _check(code):
    if code == OK:
        return
    msg = library().spk_last_error().decode(errors="replace")
    if code == ERR_INVALID:
        raise InvalidArgument(code, msg)
    if code == ERR_CAPACITY:
        raise CapacityError(code, msg)
    raise SpiceError(code, msg)


def model_attrs(model):
    """(neuron attribute dtypes, synapse attribute dtypes) as exported for `model`."""
    m = MODELS[model] if isinstance(model, str) else int(model)
    nn, ns = C.c_int(), C.c_int()
    buf = C.create_string_buffer(32)
    _check(library().spk_model_attrs(m, C.byref(nn), C.byref(ns), buf, 32))
    t = buf.value.decode()
    dt = [np.float32 if c == "f" else np.int32 for c in t]
    return dt[: nn.value], dt[nn.value: nn.value + ns.value]


class Layout:
    """Populations and (src_pop, dst_pop, p) connections (spice/util/layout.h:30-33).
    Layout(n, p) is the single-population form."""

    def __init__(self, pops, connections=None):
        if connections is None:  # Layout(n, p)
            n, p = pops
            pops, connections = [int(n)], [(0, 0, float(p))]
        elif not hasattr(pops, "__len__"):
            n, p = pops, connections
            pops, connections = [int(n)], [(0, 0, float(p))]
        self.pops = [int(x) for x in pops]
        self.conns = [(int(a), int(b), float(p)) for a, b, p in connections]
        self._keep = None

    def desc(self):
        pops = (C.c_uint64 * max(1, len(self.pops)))(*self.pops)
        src = (C.c_int * max(1, len(self.conns)))(*[c[0] for c in self.conns])
        dst = (C.c_int * max(1, len(self.conns)))(*[c[1] for c in self.conns])
        p = (C.c_float * max(1, len(self.conns)))(*[c[2] for c in self.conns])
        self._keep = (pops, src, dst, p)
        return _LayoutDesc(len(self.pops), pops, len(self.conns), src, dst, p)

    def _flatten(self):
        d = self.desc()
        cap = max(1, len(self.conns))
        rng = (C.c_int * (4 * cap))()
        pr = (C.c_float * cap)()
        cnt, size, width = C.c_int(), C.c_uint64(), C.c_uint64()
        _check(library().spk_layout_flatten(C.byref(d), rng, pr, cap, C.byref(cnt), C.byref(size), C.byref(width)))
        conns = [(rng[4 * i], rng[4 * i + 1], rng[4 * i + 2], rng[4 * i + 3], pr[i]) for i in range(cnt.value)]
        return size.value, conns, width.value

    def size(self):
        return self._flatten()[0]

    def connections(self):
        """Flattened (src_first, src_last, dst_first, dst_last, p) tuples, sorted."""
        return self._flatten()[1]

    def max_degree(self):
        return self._flatten()[2]


def _arr_ptrs(arrays):
    return (C.c_void_p * len(arrays))(*[a.ctypes.data for a in arrays])


class Snn:
    """One simulated network on one GPU: the reference's cuda::snn<Model>.

    Snn(model, layout, dt, delay=1, seed=1, graph_seed=1337)   generate the graph on device
                                                                (tile_target: tiles for a GPU shared with others;
                                                                options: build choices, see net_options)
    Snn(model, adj=(edges, width), dt=..., delay=...)           import an ELL adjacency
    Snn.from_state(model, edges, width, neurons, synapses, ...)  conversion constructor
    """

    def __init__(self, model, layout=None, dt=1e-4, delay=1, seed=1, graph_seed=1337, device=0, adj=None, tile_target=0,
                 options=None):
        lib = library()
        self.model = model if isinstance(model, str) else MODEL_NAMES[int(model)]
        m = MODELS[self.model]
        self._h = C.c_void_p()
        if adj is not None:
            edges, width = adj
            edges = np.ascontiguousarray(edges, dtype=np.int32)
            width = int(width)
            n = edges.size // width if width else 0
            _check(lib.spk_net_create_from_adj(C.byref(self._h), m, edges.ctypes.data, n, width, float(dt), int(delay),
                                               int(seed), int(device)))
        else:
            if layout is None:
                raise InvalidArgument(ERR_INVALID, "layout or adj required")
            d = layout.desc()
            o = net_options(tile_target, **(options or {}))
            _check(lib.spk_net_create_opts(C.byref(self._h), m, C.byref(d), float(dt), int(delay), int(seed), int(graph_seed),
                                           int(device), C.byref(o)))
        self._ndt, self._sdt = model_attrs(self.model)

    @classmethod
    def from_state(cls, model, edges, width, neurons, synapses=None, dt=1e-4, delay=1, seed=1, device=0):
        """cuda::snn(const snn&) (spice/cuda/snn.d.cpp:201-221): same graph, same state."""
        net = cls(model, adj=(edges, width), dt=dt, delay=delay, seed=seed, device=device)
        net.set_neurons(neurons)
        if synapses is not None and len(net._sdt):
            net.set_synapses(synapses)
        return net

    # --- lifecycle ------------------------------------------------------------------
    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            _check(library().spk_net_destroy(self._h))
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # --- stepping -------------------------------------------------------------------
    def step(self, out=False):
        """Advance one step. out=True returns the ids that fired (ascending int32)."""
        lib = library()
        if not out:
            _check(lib.spk_net_step(self._h, None, 0, None))
            return None
        n = self.num_neurons()
        buf = np.empty(max(1, n), dtype=np.int32)
        cnt = C.c_uint64()
        _check(lib.spk_net_step(self._h, buf.ctypes.data, buf.size, C.byref(cnt)))
        return buf[: cnt.value].copy()

    def run(self, nsteps):
        _check(library().spk_net_run(self._h, int(nsteps)))

    def run_record(self, nsteps, cap=None):
        """Advance nsteps and return (counts[nsteps], ids) of the spike raster."""
        nsteps = int(nsteps)
        if cap is None:
            cap = max(1024, nsteps * max(1, self.num_neurons() // 20))
        counts = np.empty(max(1, nsteps), dtype=np.uint32)
        ids = np.empty(max(1, cap), dtype=np.int32)
        tot = C.c_uint64()
        _check(library().spk_net_run_record(self._h, nsteps, counts.ctypes.data, ids.ctypes.data, cap, C.byref(tot)))
        return counts[:nsteps], ids[: tot.value]

    def sync(self):
        _check(library().spk_net_sync(self._h))

    def stream(self):
        """cudaStream_t (as int) the net's kernels run on."""
        v = C.c_void_p()
        _check(library().spk_net_stream(self._h, C.byref(v)))
        return v.value or 0

    # --- queries --------------------------------------------------------------------
    def info(self):
        i = NetInfo()
        _check(library().spk_net_get_info(self._h, C.byref(i)))
        return i

    def num_neurons(self):
        return self.info().num_neurons

    def num_synapses(self):
        return self.info().num_synapses

    def dt(self):
        return self.info().dt

    def delay(self):
        return self.info().delay

    def adj(self):
        i = self.info()
        e = np.empty(max(1, i.num_synapses), dtype=np.int32)
        _check(library().spk_net_adj(self._h, e.ctypes.data, e.size))
        return e[: i.num_synapses], i.width

    def neurons(self):
        n = self.num_neurons()
        arrs = [np.empty(n, dtype=t) for t in self._ndt]
        _check(library().spk_net_neurons(self._h, _arr_ptrs(arrs)))
        return arrs

    def synapses(self):
        s = self.num_synapses()
        arrs = [np.empty(s, dtype=t) for t in self._sdt]
        if arrs:
            _check(library().spk_net_synapses(self._h, _arr_ptrs(arrs)))
        return arrs

    def set_neurons(self, arrays):
        arrs = [np.ascontiguousarray(a, dtype=t) for a, t in zip(arrays, self._ndt)]
        _check(library().spk_net_set_neurons(self._h, _arr_ptrs(arrs)))

    def set_synapses(self, arrays):
        arrs = [np.ascontiguousarray(a, dtype=t) for a, t in zip(arrays, self._sdt)]
        _check(library().spk_net_set_synapses(self._h, _arr_ptrs(arrs)))

    def checkpoint(self):
        """Everything the net needs to continue bit for bit (bytes): edges, state, the spike
        ring, the clock and the lazy-STDP state. Snn.restore(data) continues from it."""
        lib = library()
        size = C.c_uint64()
        _check(lib.spk_net_checkpoint(self._h, None, 0, C.byref(size)))
        buf = np.empty(size.value, dtype=np.uint8)
        _check(lib.spk_net_checkpoint(self._h, buf.ctypes.data, buf.size, C.byref(size)))
        return buf.tobytes()

    @classmethod
    def restore(cls, data, device=0):
        """A new net continuing from checkpoint() bytes."""
        net = cls.__new__(cls)
        net._h = C.c_void_p()
        arr = np.frombuffer(data, dtype=np.uint8)
        _check(library().spk_net_restore(C.byref(net._h), arr.ctypes.data, arr.size, int(device)))
        net.model = MODEL_NAMES[net.info().model]
        net._ndt, net._sdt = model_attrs(net.model)
        return net

    def set_producer_warps(self, warps):
        """window_flat's producer warps (4-24, default 12): a tuning choice, same results."""
        _check(library().spk_net_set_producer_warps(self._h, int(warps)))

    def set_tile_target(self, target):
        """Re-tile (before the first step) into about `target` tiles, for sharing the GPU."""
        _check(library().spk_net_set_tile_target(self._h, int(target)))


class Batch:
    """Many independent nets stepped together by shared launches (one CTA per net tile).

    Nets of the models without plasticity; each keeps its own state, stream and results,
    identical to stepping it alone. A net is in at most one batch.
    """

    def __init__(self, device=0):
        self._h = C.c_void_p()
        self._nets = []
        _check(library().spk_batch_create(C.byref(self._h), int(device)))

    def add(self, net):
        _check(library().spk_batch_add(self._h, net._h))
        self._nets.append(net)

    def remove(self, net):
        _check(library().spk_batch_remove(self._h, net._h))
        self._nets.remove(net)

    @property
    def nets(self):
        return list(self._nets)

    def run(self, nsteps):
        """Advance every net by nsteps steps."""
        _check(library().spk_batch_run(self._h, int(nsteps)))

    def sync(self):
        for n in self._nets:
            n.sync()

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            _check(library().spk_batch_destroy(self._h))
            self._h = C.c_void_p()
            self._nets = []

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


def estimate_bytes(model, layout, delay=1, device=0, tile_target=0, options=None):
    """Upper estimate of the device memory a net of this model and layout would hold."""
    m = MODELS[model] if isinstance(model, str) else int(model)
    d = layout.desc()
    out = C.c_uint64()
    o = net_options(tile_target, **(options or {}))
    _check(library().spk_net_estimate_bytes_opts(m, C.byref(d), int(delay), int(device), C.byref(o), C.byref(out)))
    return out.value


class Server:
    """Simulation jobs admitted against a device-memory budget and stepped by continuous
    batching on one GPU (native builder threads and a ticker thread; see spk_server_* in spice_b200.h).
    Creation maps the budget (at most the free memory less 1 GiB) into the device's
    stream-ordered pool, which the jobs' nets are built from; close() hands it back.

    srv = Server(budget_bytes=150e9, quantum=1500)
    job = srv.submit("brunel", layout, nsteps=10_000, delay=15, seed=1)
    srv.wait(job); V, Twait = srv.neurons(job)
    """

    def __init__(self, budget_bytes, quantum=1500, device=0, builders=0):
        self._h = C.c_void_p()
        self._models = {}
        _check(library().spk_server_create_ex(C.byref(self._h), int(device), int(budget_bytes), int(quantum),
                                              int(builders)))

    def submit(self, model, layout, nsteps, dt=1e-4, delay=1, seed=1, graph_seed=1337, timeout=0.0):
        """Queue a job; returns its id. Raises SpiceError (ERR_NOMEM) if it alone exceeds the budget."""
        name = model if isinstance(model, str) else MODEL_NAMES[int(model)]
        d = layout.desc()
        job = C.c_uint64()
        code = library().spk_server_submit(self._h, MODELS[name], C.byref(d), float(dt), int(delay), int(seed),
                                           int(graph_seed), int(nsteps), float(timeout), C.byref(job))
        self._models[job.value] = name
        _check(code)
        return job.value

    def info(self, job):
        i = JobInfo()
        _check(library().spk_server_job_info(self._h, int(job), C.byref(i)))
        return i

    def state(self, job):
        return JOB_STATES[self.info(job).state]

    def neurons(self, job):
        """Final neuron state of a completed job (one array per attribute)."""
        i = self.info(job)
        ndt, _ = model_attrs(self._models[int(job)])
        arrs = [np.empty(i.num_neurons, dtype=t) for t in ndt]
        _check(library().spk_server_job_neurons(self._h, int(job), _arr_ptrs(arrs)))
        return arrs

    def cancel(self, job):
        _check(library().spk_server_cancel(self._h, int(job)))

    def release(self, job):
        _check(library().spk_server_release(self._h, int(job)))
        self._models.pop(int(job), None)

    def wait(self, job=0, timeout=-1.0):
        """Block until `job` (0 = all jobs) is finished; raises SpiceError(ERR_TIMEOUT) if timeout runs out."""
        _check(library().spk_server_wait(self._h, int(job), float(timeout)))

    def stats(self):
        st = ServerStats()
        _check(library().spk_server_get_stats(self._h, C.byref(st)))
        return {k: getattr(st, k) for k, _ in ServerStats._fields_}

    def inject_alloc_failures(self, count):
        _check(library().spk_server_inject_alloc_failures(self._h, int(count)))

    def inject_device_error(self, job):
        """At its next tick the job's net reports a device error (as a bounded wait that ran
        out does); the job fails alone."""
        _check(library().spk_server_inject_device_error(self._h, int(job)))

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            _check(library().spk_server_destroy(self._h))
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()
