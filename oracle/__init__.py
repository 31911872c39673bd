"""TEST INFRASTRUCTURE ONLY -- the CPU oracle (the checker).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline / reference leg may use
this package, and only as the checker or the timed CPU baseline, never as the product.

  OracleNet     the independent CPU restatement (libspice_oracle.so, spice_oracle.cpp),
                FP32 (bit-exact with the reference) or FP64
  ReferenceNet  the reference's own cpu::snn compiled from its sources with the
                counter-RNG shim (_ref/libspice_ref.so, built only where the reference
                checkout exists)
"""
import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_LIB = os.path.join(HERE, "libspice_oracle.so")
REF_LIB = os.path.join(HERE, "_ref", "libspice_ref.so")
REF_FAST_LIB = os.path.join(HERE, "_ref", "libspice_ref_fast.so")
# the reference's cpu::snn of the tests' model (tests/user_model), as model 7
REF_USER_LIB = os.path.join(HERE, "_ref", "libspice_ref_user.so")
# the reference checkout the `ref` build compiles from (no default: set by the build recipe)
REFERENCE_SRC = os.environ.get("SPICE_REFERENCE_SRC", "")

MODELS = {"vogels_abbott": 0, "brunel": 1, "brunel_with_plasticity": 2, "synth": 3,
          "vogels_abbott_ns": 4, "brunel_fixed": 5, "brunel_with_plasticity_a012": 6}
NEURON_ATTRS = {0: [np.float32] * 3 + [np.int32], 1: [np.float32, np.int32], 2: [np.float32, np.int32], 3: [np.int32],
                4: [np.float32] * 3 + [np.int32], 5: [np.float32, np.int32], 6: [np.float32, np.int32]}
PLASTIC = (2, 6)
REFERENCE_MODELS = ("vogels_abbott", "brunel", "brunel_with_plasticity", "synth")  # the reference's own structs

U64P, IP, FP = C.POINTER(C.c_uint64), C.POINTER(C.c_int), C.POINTER(C.c_float)


def build(reference=True, reference_src=None):
    """Compile the restatement and, where the reference sources exist (reference_src, else
    the SPICE_REFERENCE_SRC environment variable), the reference."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    src = reference_src or REFERENCE_SRC
    if reference and src and os.path.isdir(os.path.join(src, "spice")):
        subprocess.run(["make", "-s", "-C", HERE, "ref", f"REF={src}"], check=True)


def have_reference(fast=False):
    return os.path.exists(REF_FAST_LIB if fast else REF_LIB)


def _layout_args(pops, conns):
    a = lambda t, v: (t * max(1, len(v)))(*v)
    return (len(pops), a(C.c_uint64, pops), len(conns), a(C.c_int, [c[0] for c in conns]),
            a(C.c_int, [c[1] for c in conns]), a(C.c_float, [c[2] for c in conns]))


_olib = None


def oracle_lib():
    global _olib
    if _olib is None:
        if not os.path.exists(ORACLE_LIB):
            build(reference=False)
        lib = C.CDLL(ORACLE_LIB)
        lib.oracle_last_error.restype = C.c_char_p
        lib.oracle_layout.argtypes = [C.c_int, U64P, C.c_int, IP, IP, FP, IP, FP, C.c_int, U64P, U64P]
        lib.oracle_generate.argtypes = [C.c_int, C.c_uint64, C.c_int, U64P, C.c_int, IP, IP, FP, IP]
        lib.oracle_philox_row.argtypes = [C.c_uint64, C.c_int, U64P, C.c_int, IP, IP, FP, C.c_int, IP]
        lib.oracle_create.restype = C.c_void_p
        lib.oracle_create.argtypes = [C.c_int, C.c_int, C.c_int, U64P, C.c_int, IP, IP, FP, C.c_float, C.c_int, C.c_uint64,
                                      C.c_int, C.c_uint64, IP, C.c_uint64]
        lib.oracle_destroy.argtypes = [C.c_void_p]
        lib.oracle_step.argtypes = [C.c_void_p, IP, C.c_int]
        lib.oracle_num_neurons.argtypes = [C.c_void_p]
        lib.oracle_num_neurons.restype = C.c_uint64
        lib.oracle_width.argtypes = [C.c_void_p]
        lib.oracle_width.restype = C.c_uint64
        lib.oracle_adj.argtypes = [C.c_void_p, IP]
        lib.oracle_neurons.argtypes = [C.c_void_p, C.POINTER(C.c_void_p)]
        lib.oracle_synapses.argtypes = [C.c_void_p, C.POINTER(C.c_void_p)]
        lib.oracle_neurons_f32.argtypes = [C.c_void_p, C.POINTER(C.c_void_p)]
        lib.oracle_synapses_f32.argtypes = [C.c_void_p, C.POINTER(C.c_void_p)]
        lib.oracle_dt_sequence.argtypes = [C.c_float, C.c_int, FP]
        lib.oracle_philox.argtypes = [C.POINTER(C.c_uint32), C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)]
        lib.oracle_set_state.argtypes = [C.c_void_p, C.POINTER(C.c_void_p), C.POINTER(C.c_void_p)]
        lib.oracle_set_progress.argtypes = [C.c_void_p, C.c_uint64, C.c_int, C.POINTER(C.c_uint32), IP]
        _olib = lib
    return _olib


def layout(pops, conns):
    """(size, flattened connections, max_degree) as the oracle restates layout."""
    lib = oracle_lib()
    cap = max(1, len(conns))
    rng, pr = (C.c_int * (4 * cap))(), (C.c_float * cap)()
    md, sz = C.c_uint64(), C.c_uint64()
    k = lib.oracle_layout(*_layout_args(pops, conns), rng, pr, cap, C.byref(md), C.byref(sz))
    if k < 0:
        raise ValueError(lib.oracle_last_error().decode())
    return sz.value, [(rng[4 * i], rng[4 * i + 1], rng[4 * i + 2], rng[4 * i + 3], pr[i]) for i in range(k)], md.value


def generate(pops, conns, seed, graph="philox"):
    """ELL edges from the reference generator (graph="reference") or the Philox one."""
    n, _, w = layout(pops, conns)
    out = np.empty(max(1, n * w), dtype=np.int32)
    r = oracle_lib().oracle_generate(0 if graph == "reference" else 1, seed, *_layout_args(pops, conns),
                                     out.ctypes.data_as(IP))
    if r:
        raise ValueError(oracle_lib().oracle_last_error().decode())
    return out[: n * w], w


def philox_row(pops, conns, seed, row):
    n, _, w = layout(pops, conns)
    out = np.empty(max(1, w), dtype=np.int32)
    oracle_lib().oracle_philox_row(seed, *_layout_args(pops, conns), int(row), out.ctypes.data_as(IP))
    return out[:w]


def philox(ctr, key):
    c = (C.c_uint32 * 4)(*ctr)
    k = (C.c_uint32 * 2)(*key)
    o = (C.c_uint32 * 4)()
    oracle_lib().oracle_philox(c, k, o)
    return list(o)


def dt_sequence(dt, count):
    out = np.empty(count, dtype=np.float32)
    oracle_lib().oracle_dt_sequence(dt, count, out.ctypes.data_as(FP))
    return out


class OracleNet:
    """The CPU restatement of cpu::snn. Give `edges`/`width` to import a graph (the
    conversion constructor's view), else the graph comes from `graph` ("philox" or
    "reference") with `graph_seed`."""

    def __init__(self, model, pops, conns, dt=1e-4, delay=1, seed=1, precision=32, edges=None, width=0, graph="philox",
                 graph_seed=1337):
        lib = oracle_lib()
        self.model = MODELS[model] if isinstance(model, str) else int(model)
        self.precision = precision
        e = None
        if edges is not None:
            self._edges = np.ascontiguousarray(edges, dtype=np.int32)
            e = self._edges.ctypes.data_as(IP)
        self._h = lib.oracle_create(self.model, precision, *_layout_args(pops, conns), dt, delay, seed,
                                    0 if graph == "reference" else 1, graph_seed, e, width)
        if not self._h:
            raise ValueError(lib.oracle_last_error().decode())
        self.n = lib.oracle_num_neurons(self._h)
        self.width = lib.oracle_width(self._h)
        self._buf = np.empty(max(1, self.n), dtype=np.int32)

    def __del__(self):
        if getattr(self, "_h", None):
            oracle_lib().oracle_destroy(self._h)
            self._h = None

    def step(self):
        k = oracle_lib().oracle_step(self._h, self._buf.ctypes.data_as(IP), self._buf.size)
        return self._buf[:k].copy()

    def adj(self):
        e = np.empty(max(1, self.n * self.width), dtype=np.int32)
        oracle_lib().oracle_adj(self._h, e.ctypes.data_as(IP))
        return e[: self.n * self.width], self.width

    def neurons(self):
        """Exact attribute arrays (float32/int32) for precision 32, float64 for 64."""
        if self.precision == 32:
            arrs = [np.empty(self.n, dtype=t) for t in NEURON_ATTRS[self.model]]
            oracle_lib().oracle_neurons_f32(self._h, (C.c_void_p * len(arrs))(*[a.ctypes.data for a in arrs]))
        else:
            arrs = [np.empty(self.n, dtype=np.float64) for _ in NEURON_ATTRS[self.model]]
            oracle_lib().oracle_neurons(self._h, (C.c_void_p * len(arrs))(*[a.ctypes.data for a in arrs]))
        return arrs

    def set_state(self, neurons, synapses=None):
        """Replace the neuron state (the model's attribute arrays, float32 / int32) and, for
        Brunel+, the synapse state (W, Zpre, Zpost over all n x width slots, float32)."""
        na = [np.ascontiguousarray(a, dtype=t) for a, t in zip(neurons, NEURON_ATTRS[self.model])]
        sa = [np.ascontiguousarray(a, dtype=np.float32) for a in synapses] if synapses else []
        oracle_lib().oracle_set_state(self._h, (C.c_void_p * len(na))(*[a.ctypes.data for a in na]),
                                      (C.c_void_p * 3)(*[a.ctypes.data for a in sa]) if sa else None)

    def set_progress(self, step0, counts=(), ids=()):
        """Continue a run at step `step0` with the spikes of the last len(counts) steps
        (counts per step, ids concatenated, oldest first) in flight."""
        c = np.ascontiguousarray(counts, dtype=np.uint32)
        i = np.ascontiguousarray(ids, dtype=np.int32)
        if oracle_lib().oracle_set_progress(self._h, int(step0), len(c), c.ctypes.data_as(C.POINTER(C.c_uint32)),
                                            i.ctypes.data_as(IP)):
            raise ValueError(oracle_lib().oracle_last_error().decode())

    def synapses(self):
        if self.model not in PLASTIC:
            return []
        dt = np.float32 if self.precision == 32 else np.float64
        arrs = [np.empty(self.n * self.width, dtype=dt) for _ in range(3)]
        f = oracle_lib().oracle_synapses_f32 if self.precision == 32 else oracle_lib().oracle_synapses
        f(self._h, (C.c_void_p * 3)(*[a.ctypes.data for a in arrs]))
        return arrs


_rlibs = {}


def ref_lib(fast=False, path=None):
    path = path or (REF_FAST_LIB if fast else REF_LIB)
    if path not in _rlibs:
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path}: the reference build is not available")
        lib = C.CDLL(path)
        lib.ref_last_error.restype = C.c_char_p
        lib.ref_create.restype = C.c_void_p
        lib.ref_create.argtypes = [C.c_int, C.c_int, U64P, C.c_int, IP, IP, FP, C.c_float, C.c_int, C.c_uint64]
        lib.ref_destroy.argtypes = [C.c_void_p]
        lib.ref_step.argtypes = [C.c_void_p, IP, C.c_int]
        for f in ("ref_num_neurons", "ref_width", "ref_num_synapse_attrs"):
            getattr(lib, f).argtypes = [C.c_void_p]
            getattr(lib, f).restype = C.c_uint64
        lib.ref_adj.argtypes = [C.c_void_p, IP]
        lib.ref_neurons.argtypes = [C.c_void_p, C.POINTER(C.c_void_p)]
        lib.ref_synapses.argtypes = [C.c_void_p, C.POINTER(C.c_void_p)]
        lib.ref_generate.restype = C.c_uint64
        lib.ref_generate.argtypes = [C.c_int, U64P, C.c_int, IP, IP, FP, IP]
        lib.ref_layout.argtypes = [C.c_int, U64P, C.c_int, IP, IP, FP, IP, FP, C.c_int, U64P, U64P]
        lib.ref_create_from_state.restype = C.c_void_p
        lib.ref_create_from_state.argtypes = [C.c_int, C.c_uint64, C.c_uint64, IP, C.POINTER(C.c_void_p),
                                              C.POINTER(C.c_void_p), C.c_float, C.c_int, C.c_uint64, C.c_uint64,
                                              C.c_int, C.POINTER(C.c_uint32), IP]
        _rlibs[path] = lib
    return _rlibs[path]


class ReferenceNet:
    """The reference's cpu::snn (with the counter-RNG Poisson stream)."""

    def __init__(self, model, pops, conns, dt=1e-4, delay=1, seed=1, fast=False, _state=None, lib_path=None,
                 types=None):
        lib = ref_lib(fast, lib_path)
        self.lib = lib
        self.model = MODELS[model] if isinstance(model, str) else int(model)
        # attribute dtypes (neuron, synapse): the built-in models' unless given
        if types is None:
            types = (NEURON_ATTRS[self.model], [np.float32] * 3 if self.model in PLASTIC else [])
        self.neuron_types, self.synapse_types = list(types[0]), list(types[1])
        if _state is None:
            self._h = lib.ref_create(self.model, *_layout_args(pops, conns), dt, delay, seed)
        else:
            edges, width, neurons, synapses, step0, counts, ids = _state
            e = np.ascontiguousarray(edges, dtype=np.int32)
            n = e.size // width if width else len(neurons[0])
            na = [np.ascontiguousarray(a, dtype=t) for a, t in zip(neurons, self.neuron_types)]
            sa = [np.ascontiguousarray(a, dtype=t) for a, t in zip(synapses, self.synapse_types)] if synapses else []
            c = np.ascontiguousarray(counts, dtype=np.uint32)
            i = np.ascontiguousarray(ids, dtype=np.int32)
            self._h = lib.ref_create_from_state(self.model, n, width, e.ctypes.data_as(IP),
                                                (C.c_void_p * len(na))(*[a.ctypes.data for a in na]),
                                                (C.c_void_p * len(sa))(*[a.ctypes.data for a in sa]) if sa else None,
                                                dt, delay, seed, int(step0), len(c), c.ctypes.data_as(C.POINTER(C.c_uint32)),
                                                i.ctypes.data_as(IP))
        if not self._h:
            raise ValueError(lib.ref_last_error().decode())
        self.n = lib.ref_num_neurons(self._h)
        self.width = lib.ref_width(self._h)
        self._buf = np.empty(max(1, self.n), dtype=np.int32)

    @classmethod
    def from_state(cls, model, edges, width, neurons, synapses=None, dt=1e-4, delay=1, seed=1, fast=False, step0=0,
                   counts=(), ids=(), lib_path=None, types=None):
        """The reference's cpu::snn over a given graph (n x width ELL) and state (neuron
        attribute arrays; for Brunel+ also W, Zpre, Zpost over all slots): a simulation that
        continues where another one stands at step `step0` (clock and Poisson stream keyed by
        `seed`), with the spikes of the last len(counts) steps in flight (counts per step, ids
        concatenated, oldest first)."""
        return cls(model, None, None, dt=dt, delay=delay, seed=seed, fast=fast,
                   _state=(edges, int(width), neurons, synapses, step0, counts, ids), lib_path=lib_path, types=types)

    def __del__(self):
        if getattr(self, "_h", None):
            self.lib.ref_destroy(self._h)
            self._h = None

    def step(self):
        k = self.lib.ref_step(self._h, self._buf.ctypes.data_as(IP), self._buf.size)
        return self._buf[:k].copy()

    def adj(self):
        e = np.empty(max(1, self.n * self.width), dtype=np.int32)
        self.lib.ref_adj(self._h, e.ctypes.data_as(IP))
        return e[: self.n * self.width], self.width

    def neurons(self):
        arrs = [np.empty(self.n, dtype=t) for t in self.neuron_types]
        self.lib.ref_neurons(self._h, (C.c_void_p * len(arrs))(*[a.ctypes.data for a in arrs]))
        return arrs

    def synapses(self):
        if not self.synapse_types:
            return []
        arrs = [np.empty(self.n * self.width, dtype=t) for t in self.synapse_types]
        self.lib.ref_synapses(self._h, (C.c_void_p * len(arrs))(*[a.ctypes.data for a in arrs]))
        return arrs
