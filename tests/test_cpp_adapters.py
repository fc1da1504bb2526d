"""Builds the C++ adapter check (tests/cpp/test_adapters.cpp, over
include/gfgpu.hpp and libgfgpu.so) and runs it on the GPU."""
import os
import shutil
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
LIB = ROOT / "geoflow_b200"


def _build(tmp_path):
    cxx = shutil.which("g++")
    cuda = "/usr/local/cuda"
    exe = tmp_path / "test_adapters"
    cmd = [cxx, "-std=c++17", "-O2", str(ROOT / "tests" / "cpp" / "test_adapters.cpp"),
           f"-I{cuda}/include", f"-L{cuda}/lib64", f"-L{LIB}", "-lgfgpu", "-lcudart",
           f"-Wl,-rpath,{LIB}", f"-Wl,-rpath,{cuda}/lib64", "-o", str(exe)]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    return exe


def test_cpp_adapters_compile(tmp_path):
    """The C++ adapter header compiles against the C ABI (no GPU needed)."""
    assert _build(tmp_path).exists()


@pytest.mark.gpu
def test_cpp_adapters_run(tmp_path):
    exe = _build(tmp_path)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "adapters ok" in r.stdout
