"""The C++ host wrapper (include/spc5cuda.hpp) compiles and links against the
library; on a GPU the example program runs and checks its own result."""
import os
import shutil
import subprocess

import pytest

from spc5_b200 import build as B

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def build_example(tmp_path):
    if not os.path.exists(B.LIB):
        B.build()
    exe = str(tmp_path / "spmv_example")
    cxx = shutil.which("g++") or "/usr/bin/g++"
    cuda = "/usr/local/cuda"
    cmd = [cxx, "-std=c++17", "-O2", "-I", os.path.join(ROOT, "include"), "-I", f"{cuda}/include",
           os.path.join(ROOT, "tests", "cpp", "spmv_example.cpp"), "-o", exe,
           "-L", os.path.dirname(B.LIB), "-lspc5cuda", "-L", f"{cuda}/lib64", "-lcudart",
           f"-Wl,-rpath,{os.path.dirname(B.LIB)}"]
    res = subprocess.run(cmd, capture_output=True, text=True)
    assert res.returncode == 0, res.stderr[-3000:]
    return exe


def test_cpp_wrapper_compiles_and_links(tmp_path):
    assert os.path.exists(build_example(tmp_path))


@pytest.mark.gpu
def test_cpp_example_runs(tmp_path):
    exe = build_example(tmp_path)
    res = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    assert res.returncode == 0, res.stdout + res.stderr
    assert "max |diff|" in res.stdout
