"""ForEach with caller-defined device functors: tests/cpp/for_each_test.cu is
compiled by nvcc against include/b2co/b2co.hpp (which pulls in
include/b2co/for_each.cuh) and libb2co.so, then run on the GPU.  A CPU test
checks that it compiles for sm_100a."""
import os
import subprocess

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(REPO, "tests", "cpp", "for_each_test.cu")
LIBDIR = os.path.join(REPO, "ops-collections_b200", "lib")
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")


def build(out):
    cmd = [os.path.join(CUDA, "bin", "nvcc"), "-std=c++17", "-O2", "-gencode", "arch=compute_100a,code=sm_100a",
           "--expt-relaxed-constexpr", "-I", os.path.join(REPO, "include"), SRC, "-o", out, "-L", LIBDIR, "-lb2co",
           f"-Xlinker=-rpath,{LIBDIR}"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


def test_for_each_compiles(tmp_path):
    build(str(tmp_path / "for_each_test"))


@pytest.mark.gpu
def test_for_each_runs(tmp_path):
    exe = str(tmp_path / "for_each_test")
    build(exe)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    assert "for_each test ok" in r.stdout
