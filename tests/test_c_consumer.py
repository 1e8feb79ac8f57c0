"""The C ABI from a plain C99 program (tests/c/c_consumer.c): the header
compiles as C with warnings as errors, the library links, and the host-side
entry points give the known answers (the 512 x 512 2D Laplacian's 64 x 64 ABHSF storage,
98,444,896 bits, from its histogram; the reader fixtures round-trip through
the .mm layout)."""
import os
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, "abhsf_b200")


def test_c_program_uses_the_abi(tmp_path):
    exe = str(tmp_path / "c_consumer")
    subprocess.run(["gcc", "-std=c99", "-Wall", "-Wextra", "-Werror", "-pedantic", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "c", "c_consumer.c"), "-o", exe, "-L", LIBDIR, "-labhsf_b200",
                    f"-Wl,-rpath,{LIBDIR}"], check=True)
    mtx = os.path.join(ROOT, "tests", "golden", "mtx", "real_symmetric_lower.mtx")
    r = subprocess.run([exe, mtx, str(tmp_path / "a.mm")], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    out = r.stdout.splitlines()
    assert "abhsf_bits 98444896" in out
    assert "coo_bits " + str(12 + 12 * 64) in out
    assert any(l.startswith("refused: ") and "block_size" in l for l in out)
    assert "read 4 4 6 same 1" in out and out[-1] == "OK"
