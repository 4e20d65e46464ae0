"""Build libheddle_b200.so in-tree with nvcc for sm_100a.

Usage: python -m heddle_b200.build [--verbose]

Each translation unit under heddle_b200/csrc is compiled to an object in
heddle_b200/_build and the objects are linked into heddle_b200/libheddle_b200.so.
Objects are rebuilt when their source or any header is newer.
"""

from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIB = PKG / "libheddle_b200.so"
INCLUDE = PKG.parent / "include"

SOURCES = ["hb_api.cu", "hb_nlist.cu", "hb_pair.cu", "hb_spme.cu", "hb_integ.cu", "hb_cons.cu",
           "hb_baro.cu", "hb_bonded.cu", "hb_mlp.cu", "hb_couple.cu", "hb_min.cu"]

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# Units whose kernels must round alike however their device functions are
# combined: the Langevin + SETTLE step head runs either as four kernels or
# as one fused kernel built from the same device functions, and the
# velocity-Verlet final kick runs plain or fused with a thermostat's
# rescale; without multiply-add contraction every form rounds each
# operation the same way.
FILE_FLAGS = {name: ["-fmad=false"] for name in ("hb_cons.cu", "hb_integ.cu", "hb_couple.cu")}
NVCC_FLAGS = [
    "-O3",
    "-std=c++17",
    "-lineinfo",
    "-Xcompiler",
    "-fPIC,-ffp-contract=off",
    "--expt-relaxed-constexpr",
]


def nvcc_path() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(cand).exists():
        raise RuntimeError("nvcc not found")
    return cand


def host_compiler() -> list[str]:
    # prefer the system g++ (the CC/CXX of some images point at a compiler
    # without OpenMP specs; nvcc only needs a plain C++17 host compiler)
    for c in ("/usr/bin/g++", shutil.which("g++") or ""):
        if c and Path(c).exists():
            return ["-ccbin", c]
    return []


def _newer(src: Path, dst: Path, deps: list[Path]) -> bool:
    if not dst.exists():
        return True
    t = dst.stat().st_mtime
    return src.stat().st_mtime > t or any(d.stat().st_mtime > t for d in deps)


def build(verbose: bool = False, extra: list[str] | None = None) -> Path:
    BUILD.mkdir(exist_ok=True)
    nvcc = nvcc_path()
    deps = list(CSRC.glob("*.cuh")) + list(INCLUDE.glob("*.h")) + [Path(__file__)]
    objs = []
    for name in SOURCES:
        src = CSRC / name
        obj = BUILD / (src.stem + ".o")
        objs.append(obj)
        if _newer(src, obj, deps):
            cmd = [nvcc, *host_compiler(), *ARCH, *NVCC_FLAGS, *FILE_FLAGS.get(name, []),
                   *(extra or []), "-I", str(INCLUDE), "-c", str(src), "-o", str(obj)]
            if verbose:
                print(" ".join(cmd))
            subprocess.run(cmd, check=True)
    if not LIB.exists() or any(o.stat().st_mtime > LIB.stat().st_mtime for o in objs):
        tmp = LIB.with_suffix(".so.tmp")
        cmd = [nvcc, *host_compiler(), *ARCH, "-shared", "-o", str(tmp),
               *[str(o) for o in objs], "-lcudart"]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
        os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    build(verbose="--verbose" in sys.argv)
    print(LIB)
