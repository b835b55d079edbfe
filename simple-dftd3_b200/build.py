"""Build the B200 DFT-D3 shared library in-tree.

Compiles the CUDA kernels, the host engine, the C ABI and the parameter tables
with nvcc for sm_100a and links ``lib/libsdftd3_b200.so``.  Objects are cached
in ``_build/`` and rebuilt when a source or header is newer.

Usage: python simple-dftd3_b200/build.py [--verbose-ptxas]
"""
import os
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIB = PKG / "lib" / "libsdftd3_b200.so"
INCLUDE = PKG.parent / "include"

SOURCES = ["d3_kernels.cu", "d3_pair.cu", "d3_pair_tt.cu", "d3_atm.cu", "d3_atm_mol.cu", "d3_pairwise.cu", "d3_hessian.cu", "d3_engine.cu", "d3_noalloc.cu", "d3_api.cpp", "d3_tables.c", "d3_params.c"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc():
    cuda = os.environ.get("CUDA_HOME", "/usr/local/cuda")
    return str(Path(cuda) / "bin" / "nvcc")


def _stale(obj, deps):
    if not obj.exists():
        return True
    t = obj.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def build(verbose_ptxas=False, force=False):
    BUILD.mkdir(exist_ok=True)
    LIB.parent.mkdir(exist_ok=True)
    headers = list(CSRC.glob("*.h")) + list(CSRC.glob("*.cuh")) + list(INCLUDE.glob("*.h"))
    objs = []
    for src in SOURCES:
        path = CSRC / src
        obj = BUILD / (src + ".o")
        objs.append(obj)
        if not force and not _stale(obj, [path] + headers):
            continue
        cmd = [nvcc(), "-c", str(path), "-o", str(obj), "-O3", "-std=c++17", "-Xcompiler", "-fPIC",
               "-I", str(CSRC), "-I", str(INCLUDE)]
        if src.endswith(".cu"):
            cmd += ARCH + ["-lineinfo", "--expt-relaxed-constexpr"]
            if verbose_ptxas:
                cmd += ["-Xptxas", "-v"]
        elif src.endswith(".c"):
            cmd = [nvcc(), "-c", str(path), "-o", str(obj), "-O2", "-Xcompiler", "-fPIC", "-I", str(CSRC)] + ARCH
        else:
            cmd += ARCH
        print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    if force or _stale(LIB, objs):
        cmd = [nvcc(), "-shared", "-o", str(LIB)] + [str(o) for o in objs] + ARCH + ["-cudart", "static"]
        print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(verbose_ptxas="--verbose-ptxas" in sys.argv, force="--force" in sys.argv)
