"""The header-only C++ adapter include/nrg_b200.hpp: it compiles with g++ against the C-ABI
library (CPU), and its checks -- the reference's 2x2 diagonalisation known answers, a
batched step, dsyevr with diagratio, product/transform/rotate against plain loops and the
reference's error conventions -- pass when run on the GPU."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cpp", "adapter_check.cpp")


def compile_adapter(tmp_path):
    from nrgljubljana_b200 import build
    lib = build.build()
    exe = str(tmp_path / "adapter_check")
    cmd = ["g++", "-std=c++17", "-O1", "-Wall", "-Wextra", "-I", os.path.join(ROOT, "include"), SRC, "-o", exe,
           lib, f"-Wl,-rpath,{os.path.dirname(lib)}"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "warning" not in r.stderr, r.stderr
    return exe


def test_adapter_compiles(tmp_path):
    compile_adapter(tmp_path)


@pytest.mark.gpu
def test_adapter_runs_on_gpu(tmp_path):
    exe = compile_adapter(tmp_path)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and "ADAPTER OK" in r.stdout, r.stdout + r.stderr
