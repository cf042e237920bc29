"""Build libefdc_xm.so in-tree for sm_100a (nvcc; no PyTorch involved).

    python efdcplus8.5_b200/build.py [--force]
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
OUT = PKG / "libefdc_xm.so"
BUILD = PKG / "_build"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-Wall",
          "-ccbin", "/usr/bin/g++"]
# per-file flags: the FP64 step kernels keep the reference's rounding (no FMA)
SOURCES = {
    "xm_step.cu": ["-fmad=false"],
    "xm_mixed.cu": [],
    "xm_capi.cu": [],
    "xm_noalloc.cu": ["-fmad=false"],
    "xm_adjoint.cu": [],
    "xm_chan.cu": ["-fmad=false"],
    "xm_loop.cu": [],
    "xm_explicit.cu": ["-fmad=false"],
}


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def build(force: bool = False, verbose: bool = False) -> Path:
    deps = list(CSRC.glob("*.cu")) + list(CSRC.glob("*.h")) + list(CSRC.glob("*.cuh")) + [
        PKG.parent / "include" / "efdc_xm.h", Path(__file__)]
    if OUT.exists() and not force and OUT.stat().st_mtime > max(d.stat().st_mtime for d in deps):
        return OUT
    BUILD.mkdir(exist_ok=True)
    objs = []
    nv = nvcc()
    for src, extra in SOURCES.items():
        obj = BUILD / (Path(src).stem + ".o")
        cmd = [nv, *ARCH, *COMMON, *extra, "-c", str(CSRC / src), "-o", str(obj)]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
        objs.append(str(obj))
    tmp = OUT.with_suffix(".so.tmp")
    subprocess.run([nv, *ARCH, "-shared", "-o", str(tmp), *objs, "-ccbin", "/usr/bin/g++"],
                   check=True)
    os.replace(tmp, OUT)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
