"""Build of the in-tree CUDA library ``libcdm_apt.so`` (sm_100a only).

The shared library is compiled with nvcc straight from ``csrc/`` into the
package directory, so that it travels with the source tree.  The FP64 kernels
are compiled with ``-fmad=false``: the reference evaluates every multiply and
add separately, and keeping them separate makes the FP64 path reproduce the
CPU restatement bit for bit.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIB = PKG / "libcdm_apt.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", f"-I{ROOT / 'include'}", f"-I{CSRC}",
          "-Xptxas", "-warn-spills"]
# translation unit -> extra flags
UNITS = {
    "apt_sweep_fp64.cu": ["-fmad=false"],
    "apt_march2d.cu": ["-fmad=false"],
    "apt_march2d_fast.cu": [],
    "apt_march3d.cu": [],
    "apt_aux.cu": ["-fmad=false"],
    "engine.cu": ["-fmad=false"],
    "apt_mixed.cu": [],
    "apt_noalloc.cu": ["-fmad=false"],
    "autotune.cu": [],
    "net_kernels.cu": [],
    "net_conv_tc.cu": [],
    "net.cu": [],
    "implicit.cu": ["-fmad=false"],
}


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def _stale(obj: Path, src: Path) -> bool:
    if not obj.exists():
        return True
    deps = [src] + list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.h")) + [ROOT / "include" / "cdm_apt.h"]
    return any(d.stat().st_mtime > obj.stat().st_mtime for d in deps)


def build(verbose: bool = False, force: bool = False) -> Path:
    BUILD.mkdir(exist_ok=True)
    objs = []
    for unit, extra in UNITS.items():
        src = CSRC / unit
        obj = BUILD / (src.stem + ".o")
        objs.append(obj)
        if force or _stale(obj, src):
            cmd = [nvcc(), *ARCH, *COMMON, *extra, "-c", str(src), "-o", str(obj)]
            if verbose:
                print(" ".join(cmd), flush=True)
            subprocess.run(cmd, check=True)
    if force or not LIB.exists() or any(o.stat().st_mtime > LIB.stat().st_mtime for o in objs):
        cmd = [nvcc(), *ARCH, "-shared", "-cudart", "static", "-o", str(LIB), *map(str, objs)]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(verbose=True, force="--force" in sys.argv)
