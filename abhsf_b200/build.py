"""Compiles the sm_100a CUDA sources of abhsf_b200/csrc into the in-tree shared
library abhsf_b200/libabhsf_b200.so with nvcc (no torch involvement), so the
built library ships with the source tree.

    python -m abhsf_b200.build [--force] [--verbose]
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import glob
import os
import subprocess

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
OBJ = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "libabhsf_b200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC",
                "-Xcompiler", "-fvisibility=hidden", "-I", os.path.join(ROOT, "include"), "-I", CSRC]


def _sources() -> list[str]:
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")))


def _deps() -> list[str]:
    return (_sources() + glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.inc")) +
            glob.glob(os.path.join(ROOT, "include", "abhsf", "*.h")))


def up_to_date() -> bool:
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    return all(os.path.getmtime(d) <= t for d in _deps())


def _compile(src: str, verbose: bool, extra: list[str]) -> str:
    obj = os.path.join(OBJ, os.path.basename(src)[:-3] + ".o")
    cmd = [NVCC] + FLAGS + extra + ["-c", src, "-o", obj]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed on {src}:\n{r.stdout}\n{r.stderr}")
    if verbose and r.stderr.strip():
        print(r.stderr, flush=True)
    return obj


def build(force: bool = False, verbose: bool = False, extra: list[str] | None = None) -> str:
    """Builds libabhsf_b200.so if a source is newer; returns its path."""
    if not force and up_to_date():
        return LIB
    os.makedirs(OBJ, exist_ok=True)
    extra = extra or []
    # a source is recompiled when it, a shared header or the flags changed
    headers = [d for d in _deps() if not d.endswith(".cu")]
    stamp = os.path.join(OBJ, "flags.txt")
    flags = " ".join(FLAGS + extra)
    same_flags = os.path.exists(stamp) and open(stamp).read() == flags

    def fresh(src: str) -> bool:
        obj = os.path.join(OBJ, os.path.basename(src)[:-3] + ".o")
        if force or not same_flags or not os.path.exists(obj):
            return False
        t = os.path.getmtime(obj)
        return all(os.path.getmtime(d) <= t for d in [src] + headers)

    def one(src: str) -> str:
        if fresh(src):
            return os.path.join(OBJ, os.path.basename(src)[:-3] + ".o")
        return _compile(src, verbose, extra)

    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        objs = list(ex.map(one, _sources()))
    with open(stamp, "w") as f:
        f.write(flags)
    tmp = LIB + ".tmp"
    cmd = [NVCC] + ARCH + ["-shared", "-o", tmp] + objs + ["-cudart", "static"]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--ptxas-v", action="store_true", help="print registers / spills per kernel")
    a = ap.parse_args()
    print(build(force=a.force or a.ptxas_v, verbose=a.verbose or a.ptxas_v,
                extra=["-Xptxas", "-v"] if a.ptxas_v else None))
