"""The C++17 surface (include/spice/cuda/snn.h over the C ABI): compiles a small program
against the in-tree library and runs it on the GPU (tests/cpp/test_snn.cpp)."""
import os
import shutil
import subprocess

import pytest

import spice_b200
from spice_b200 import build as sb_build

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def compile_cpp(out):
    sb_build.build()
    cuda_inc = "/usr/local/cuda/include"
    cmd = [shutil.which("g++") or "g++", "-std=c++17", "-O1", "-Wall", "-I", os.path.join(ROOT, "include"), "-I", cuda_inc,
           os.path.join(ROOT, "tests", "cpp", "test_snn.cpp"), "-L", os.path.dirname(spice_b200.LIB_PATH), "-lspice_b200",
           f"-Wl,-rpath,{os.path.dirname(spice_b200.LIB_PATH)}", "-o", out]
    subprocess.run(cmd, check=True, capture_output=True, text=True)


def test_cpp_header_compiles(tmp_path):
    compile_cpp(str(tmp_path / "test_snn"))


@pytest.mark.gpu
def test_cpp_surface_runs(gpu, tmp_path):
    exe = str(tmp_path / "test_snn")
    compile_cpp(exe)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "cpp ok" in r.stdout
