"""Build the sm_100a shared library lib/libmhy_b200.so from csrc/ with nvcc.

--fmad=false: no contraction of a*b+c into FMA, so every floating-point
operation rounds exactly as written (the CPU oracle is built with
-ffp-contract=off); IEEE division and square root are nvcc's defaults.
"""
from __future__ import annotations

import os
import pathlib
import shutil
import subprocess
import sys

HERE = pathlib.Path(__file__).resolve().parent
CSRC = HERE / "csrc"
LIB_DIR = HERE / "lib"
LIB = LIB_DIR / "libmhy_b200.so"
SOURCES = ["mhy_kernels.cu", "mhy_cycle.cu", "mhy_multi.cu", "mhy_capi.cu", "mhy_csr.cu", "mhy_noalloc.cu"]
HEADERS = ["mhy_kernels.cuh", "mhy_device.cuh", "mhy_pow_third.h", "mhy_line.cuh", "mhy_lagrange.cuh"]

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "--fmad=false", "-std=c++17", "-Xcompiler", "-fPIC,-ffp-contract=off", "-Xptxas", "-v"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and pathlib.Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def _stale() -> bool:
    if not LIB.exists():
        return True
    t = LIB.stat().st_mtime
    deps = [CSRC / s for s in SOURCES + HEADERS] + [HERE.parent / "include" / "mhy.h", pathlib.Path(__file__)]
    return any(p.exists() and p.stat().st_mtime > t for p in deps)


def build(force: bool = False, verbose: bool = False) -> pathlib.Path:
    if not force and not _stale():
        return LIB
    LIB_DIR.mkdir(exist_ok=True)
    objs = []
    logs = []
    for src in SOURCES:
        obj = LIB_DIR / (pathlib.Path(src).stem + ".o")
        cmd = [nvcc(), *ARCH, *FLAGS, "-rdc=false", "-c", str(CSRC / src), "-o", str(obj)]
        r = subprocess.run(cmd, capture_output=True, text=True)
        logs.append(r.stdout + r.stderr)
        if r.returncode != 0:
            sys.stderr.write(r.stdout + r.stderr)
            raise RuntimeError(f"nvcc failed on {src}")
        objs.append(str(obj))
    cmd = [nvcc(), *ARCH, "-shared", "-o", str(LIB), *objs, "-lcudart"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("nvcc link failed")
    (LIB_DIR / "ptxas.log").write_text("\n".join(logs))
    if verbose:
        print("\n".join(logs))
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
    print(LIB)
