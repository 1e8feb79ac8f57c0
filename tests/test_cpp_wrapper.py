"""The header-only C++ wrapper (include/abhsf/abhsf_gpu.hpp) used the way the
reference's programs use their formats: compiles, links against the C-ABI
library, converts statuses into std::runtime_error, and (on a GPU) computes
y += A x."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cpp", "wrapper_demo.cpp")
LIBDIR = os.path.join(ROOT, "abhsf_b200")


def _build(tmp_path):
    exe = str(tmp_path / "wrapper_demo")
    subprocess.run(["g++", "-std=c++17", "-O1", "-I", os.path.join(ROOT, "include"), SRC, "-o", exe,
                    "-L", LIBDIR, "-labhsf_b200", f"-Wl,-rpath,{LIBDIR}"], check=True)
    return exe


def test_wrapper_compiles_and_throws(tmp_path):
    exe = _build(tmp_path)
    r = subprocess.run([exe], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "caught: abhsf: block_size" in r.stdout


@pytest.mark.gpu
def test_wrapper_spmv_on_gpu(tmp_path):
    exe = _build(tmp_path)
    r = subprocess.run([exe, "--gpu"], capture_output=True, text=True)
    assert r.returncode == 0 and "OK" in r.stdout, r.stdout + r.stderr
