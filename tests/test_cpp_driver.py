"""The C++ reference-style API (include/dcsr_b200.hpp) compiles against the
C ABI; on a GPU the Fill_Test-shaped driver runs and checks itself."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cpp", "fill_test.cpp")


def compile_driver(out):
    from dcsr_b200.build import LIB, build
    build()
    cuda = "/usr/local/cuda"
    cmd = ["g++", "-O2", "-std=c++17", "-I" + os.path.join(ROOT, "include"), "-I" + cuda + "/include", SRC,
           "-o", out, LIB, "-L" + cuda + "/lib64", "-lcudart", "-Wl,-rpath," + os.path.dirname(LIB),
           "-Wl,-rpath," + cuda + "/lib64"]
    subprocess.run(cmd, check=True, capture_output=True, text=True)


def test_cpp_api_compiles(tmp_path):
    compile_driver(str(tmp_path / "fill_test"))
    assert os.path.exists(tmp_path / "fill_test")


@pytest.mark.gpu
def test_cpp_fill_driver_runs(tmp_path, dcsr):
    exe = str(tmp_path / "fill_test")
    compile_driver(exe)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    assert "FILL_TEST OK" in r.stdout
