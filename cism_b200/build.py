"""Build recipe for libcismgpu.so (sm_100a), in-tree under cism_b200/_lib/.

nvcc -gencode arch=compute_100a,code=sm_100a -lineinfo -O3 --fmad=false ...

--fmad=false keeps every FP64 a*b+c as a separate multiply and add, the operation
order of the Fortran reference (gfortran does not contract to FMA on x86-64);
FP32 kernels that want FMA call fmaf() explicitly.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT_DIR = os.path.join(HERE, "_lib")
OUT = os.path.join(OUT_DIR, "libcismgpu.so")
SOURCES = ["cismgpu.cu"]


def nvcc_path() -> str:
    p = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(p):
        raise RuntimeError("nvcc not found")
    return p


def flags(verbose: bool = False) -> list[str]:
    f = ["-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "-O3", "--fmad=false", "-std=c++17",
         "-Xcompiler", "-fPIC", "-Xcompiler", "-O2", "-shared", "-lineinfo"]
    if verbose:
        f += ["-Xptxas", "-v"]
    return f


def _stale() -> bool:
    if not os.path.exists(OUT):
        return True
    t = os.path.getmtime(OUT)
    deps = [os.path.join(CSRC, n) for n in os.listdir(CSRC)]
    deps.append(os.path.join(HERE, "..", "include", "cismgpu.h"))
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(force: bool = False, verbose: bool = False) -> str:
    """Compile libcismgpu.so if a source is newer than it; returns its path."""
    if not force and not _stale():
        return OUT
    os.makedirs(OUT_DIR, exist_ok=True)
    tmp = OUT + ".tmp"
    cmd = [nvcc_path()] + flags(verbose) + ["-o", tmp] + [os.path.join(CSRC, s) for s in SOURCES]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("nvcc failed building libcismgpu.so")
    if verbose:
        sys.stderr.write(r.stderr)
    os.replace(tmp, OUT)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
