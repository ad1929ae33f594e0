"""Build libtvs_cuda.so (the engine) in-tree for sm_100a.

    python total-viewsheds_b200/build.py

Device code is compiled without FMA contraction (-fmad=false) and with IEEE
division/sqrt and denormals (the nvcc defaults, spelled out): the exact-f32
sweep relies on every add, multiply and divide rounding once, as in the
reference.  Host code is compiled with -ffp-contract=off for the same reason.
"""

import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
LIB = PKG / "libtvs_cuda.so"
CLI = PKG / "tvs"
SOURCES = ["capi.cu", "shape.cu", "sweep.cu", "sweep_queue.cu", "sweep_split.cu", "noalloc.cu",
           "batch.cu", "shape_cache.cu", "rings_compact.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc():
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def flags():
    return ARCH + [
        "-O3", "-lineinfo", "-std=c++17",
        "-fmad=false", "-prec-div=true", "-prec-sqrt=true", "-ftz=false",
        "-Xcompiler", "-fPIC,-ffp-contract=off,-O2",
        "-I", str(ROOT / "include"), "-I", str(CSRC),
    ]


def _stale(target, deps):
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def build(force=False, verbose=False, ptxas_info=False):
    deps = [CSRC / s for s in SOURCES] + list(CSRC.glob("*.cuh")) + [ROOT / "include" / "tvs.h"]
    if force or ptxas_info or _stale(LIB, deps):
        cmd = [nvcc()] + flags() + (["-Xptxas", "-v"] if ptxas_info else []) + [
            "-shared", "-o", str(LIB)] + [str(CSRC / s) for s in SOURCES]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    cli_src = PKG / "host" / "tvs_cli.cpp"
    if force or _stale(CLI, [cli_src, ROOT / "include" / "tvs.h", LIB]):
        cxx = shutil.which("g++") or "g++"
        cmd = [cxx, "-O2", "-std=c++17", "-ffp-contract=off", "-I", str(ROOT / "include"),
               str(cli_src), "-L", str(PKG), "-ltvs_cuda", "-Wl,-rpath,$ORIGIN", "-o", str(CLI)]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True, ptxas_info="--ptxas-info" in sys.argv)
