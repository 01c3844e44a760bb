"""Builds tests/cpp/api_test.cpp against the C++ mirror (include/b2co/b2co.hpp)
and libb2co.so, and runs it on the GPU.  A CPU test checks that it compiles."""
import os
import subprocess

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(REPO, "tests", "cpp", "api_test.cpp")
LIBDIR = os.path.join(REPO, "ops-collections_b200", "lib")
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")


def build(out):
    cmd = ["g++", "-std=c++17", "-O1", "-I", os.path.join(REPO, "include"), "-I", os.path.join(CUDA, "include"),
           SRC, "-o", out, "-L", LIBDIR, "-lb2co", f"-Wl,-rpath,{LIBDIR}", "-L", os.path.join(CUDA, "lib64"),
           "-lcudart", f"-Wl,-rpath,{os.path.join(CUDA, 'lib64')}"]
    subprocess.run(cmd, check=True, capture_output=True, text=True)


def test_cpp_api_compiles(tmp_path):
    build(str(tmp_path / "api_test"))


@pytest.mark.gpu
def test_cpp_api_runs(tmp_path):
    exe = str(tmp_path / "api_test")
    build(exe)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    assert "cpp api test ok" in r.stdout
