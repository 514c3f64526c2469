"""The C++ adapter (MGSolCuda over the C ABI, tests/adapter/mgsol_cuda_adapter.cpp) compiles
against include/exfemus_b200.h and links the library; on a B200 it runs a lid-driven
cavity through MGDofBcOp / MGTimeStep in FP64 and mixed precision."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "adapter", "mgsol_cuda_adapter.cpp")


def _compile(out):
    from exfemus_b200 import build
    so = build.build()
    libdir = os.path.dirname(so)
    cxx = shutil.which("g++") or "/usr/bin/g++"
    cmd = [cxx, "-std=c++17", "-O2", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"), SRC, "-o", out,
           so, "-Wl,-rpath," + libdir]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    return out


def test_adapter_compiles_against_the_header(tmp_path):
    _compile(str(tmp_path / "adapter"))


@pytest.mark.gpu
def test_adapter_runs_the_cavity(tmp_path):
    exe = _compile(str(tmp_path / "adapter"))
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "adapter ok" in r.stdout
