"""The header-only C++ layer (include/pmg/pmg.hpp) compiles and links against
libpmg_b200.so together with a caller-side program (tests/adapter/adapter_check.cpp, a
stand-in for the reference's deal.II classes with a device vector exposing get_values()),
and on a GPU that program's checks pass: an operator from caller maps equals the box
operator, and a mixed-precision multigrid CG solve through the C++ classes converges."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, "portable-multigrid_b200")
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")


def build_check(out_dir):
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("no g++")
    exe = os.path.join(out_dir, "adapter_check")
    cmd = [gxx, "-std=c++17", "-O1", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"),
           "-I", os.path.join(CUDA, "include"), os.path.join(ROOT, "tests", "adapter", "adapter_check.cpp"),
           "-L", LIBDIR, "-lpmg_b200", "-Wl,-rpath," + LIBDIR, "-L", os.path.join(CUDA, "lib64"), "-lcudart",
           "-o", exe]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def test_adapter_compiles_and_links(tmp_path):
    exe = build_check(str(tmp_path))
    assert os.path.exists(exe)


@pytest.mark.gpu
def test_adapter_program_runs_on_gpu(tmp_path):
    exe = build_check(str(tmp_path))
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "adapter ok" in r.stdout
