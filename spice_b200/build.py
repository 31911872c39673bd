"""Build recipe of libspice_b200.so (in-tree, sm_100a).

    python -m spice_b200.build            # builds spice_b200/libspice_b200.so

A model of the user's is compiled in beside the library's own models by build_user(header,
type, out): the same sources with -DSPK_USER_MODEL_HEADER / -DSPK_USER_MODEL, the model
reachable as C-ABI id SPK_USER_MODEL_ID (7). Models are template arguments of the kernels,
as in the reference (spice/cuda/snn.d.cpp:247-250), so a new model means a new build.

Flags that matter:
  -gencode arch=compute_100a,code=sm_100a   B200 only
  -fmad=false     no contraction of a*b+c into fma: the models' arithmetic stays
                  operation-for-operation the reference's (explicit fmaf still fuses)
  no --use_fast_math: IEEE division / expf, denormals kept
"""
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIB = os.path.join(HERE, "libspice_b200.so")
SOURCES = [os.path.join(HERE, "csrc", "net.cu"), os.path.join(HERE, "csrc", "server.cpp")]
DEPS = SOURCES + [os.path.join(HERE, "csrc", f) for f in
                  ("kernels.cuh", "plastic.cuh", "flat.cuh", "slots.cuh", "ordered.cuh", "models.cuh", "device_common.cuh")]
USER_MODEL_ID = 7


def nvcc_path():
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(cand):
        raise RuntimeError("nvcc not found")
    return cand


def command(out=LIB, extra=()):
    return [
        nvcc_path(),
        "-gencode", "arch=compute_100a,code=sm_100a",
        "-lineinfo", "-O3", "-std=c++17",
        "-fmad=false",
        "--expt-relaxed-constexpr",
        "-Xcompiler", "-fPIC", "-Xcompiler", "-ffp-contract=off", "-Xcompiler", "-pthread",
        "-shared",
        "-I", os.path.join(ROOT, "include"),
        "-o", out,
        *SOURCES,
        "-lcudart",
        *extra,
    ]


def build_user(header, model, out, force=False, verbose=False):
    """libspice_b200 with the model `model` (a C++ type name) of `header` compiled in as model
    id USER_MODEL_ID; written to `out`. Rebuilt when a source, header or the model header is
    newer than `out`."""
    header = os.path.abspath(header)
    if not force and os.path.exists(out):
        t = os.path.getmtime(out)
        if all(os.path.getmtime(f) <= t for f in DEPS + _headers() + [header]):
            return out
    os.makedirs(os.path.dirname(os.path.abspath(out)), exist_ok=True)
    cmd = command(out=out, extra=[f'-DSPK_USER_MODEL_HEADER="{header}"', f"-DSPK_USER_MODEL={model}",
                                  "-I", os.path.dirname(header)])
    if verbose:
        print(" ".join(cmd))
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("nvcc failed:\n" + r.stdout + r.stderr)
    return out


def _headers():
    inc = os.path.join(ROOT, "include")
    out = []
    for d, _, fs in os.walk(inc):
        out += [os.path.join(d, f) for f in fs]
    return out


def up_to_date(out=LIB):
    if not os.path.exists(out):
        return False
    t = os.path.getmtime(out)
    return all(os.path.getmtime(f) <= t for f in DEPS + _headers())


def build(force=False, verbose=False, extra=()):
    if not force and up_to_date():
        return LIB
    cmd = command(extra=extra)
    if verbose:
        print(" ".join(cmd))
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("nvcc failed:\n" + r.stdout + r.stderr)
    if verbose and (r.stdout or r.stderr):
        print(r.stdout + r.stderr)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True, extra=[a for a in sys.argv[1:] if a != "--force"])
