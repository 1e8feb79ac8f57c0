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
    # the reference's own language level, warnings as errors
    subprocess.run(["g++", "-std=c++11", "-Wall", "-Wextra", "-Werror", "-pedantic", "-O1", "-I",
                    os.path.join(ROOT, "include"), SRC, "-o", exe,
                    "-L", LIBDIR, "-labhsf_b200", f"-Wl,-rpath,{LIBDIR}"], check=True)
    return exe


def test_wrapper_compiles_and_throws(tmp_path):
    exe = _build(tmp_path)
    r = subprocess.run([exe], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "caught: abhsf: block_size" in r.stdout


@pytest.mark.parametrize("name", ["real_general", "pattern_symmetric_upper", "crlf_and_case"])
def test_wrapper_reader_has_the_reference_shape(tmp_path, name):
    """abhsf::read_mtx_real_or_binary(filename, elements, props) appends the
    elements the reference's reader returned (tests/golden/mtx_ref.npz) and
    sets m, n, nnz; abhsf::read_mm reads the .mm made from the same file."""
    import numpy as np

    from abhsf_b200 import matrix as mx
    ref = np.load(os.path.join(ROOT, "tests", "golden", "mtx_ref.npz"))
    rows, cols, vals = ref[name + "__rows"], ref[name + "__cols"], ref[name + "__vals"]
    m, n = ref[name + "__shape"].tolist()
    k = np.arange(1, rows.size + 1, dtype=np.float64)
    want = [m, n, rows.size, rows.size + 1]
    exe = _build(tmp_path)
    src = os.path.join(ROOT, "tests", "golden", "mtx", name + ".mtx")
    mm = str(tmp_path / (name + ".mm"))
    mx.mtx2mm(src, mm)
    for flag, path in (("--read", src), ("--read-mm", mm)):
        r = subprocess.run([exe, flag, path], capture_output=True, text=True)
        assert r.returncode == 0, r.stdout + r.stderr
        f = r.stdout.split()
        assert f[0] == "read" and [int(v) for v in f[1:5]] == want
        np.testing.assert_allclose([float(v) for v in f[5:]],
                                   [float(k @ rows), float(k @ cols), float(vals.sum())], rtol=1e-12)


@pytest.mark.gpu
def test_wrapper_spmv_on_gpu(tmp_path):
    exe = _build(tmp_path)
    r = subprocess.run([exe, "--gpu"], capture_output=True, text=True)
    assert r.returncode == 0 and "OK" in r.stdout, r.stdout + r.stderr
