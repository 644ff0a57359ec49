"""In-tree build of the CUDA library for sm_100a (B200).

``python -m pyeulerale_b200.build`` compiles every ``csrc/*.cu`` with nvcc into an object under
``pyeulerale_b200/_build/`` (in parallel, recompiling only sources older than their inputs) and
links ``pyeulerale_b200/libeuler_b200.so``. The library is loaded with ctypes (``_lib.py``); it
stays in the source tree (not installed) so that it ships with the repository snapshot.
"""

from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
OBJ = PKG / "_build"
LIB = PKG / "libeuler_b200.so"
INCLUDE = PKG.parent / "include"

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC",
]
# The Jacobian kernels evaluate without FMA contraction: derivatives of the reference's branch
# primitives (abs_c, max_c) are decided by exact ties and cancellations at degenerate states (an
# exact free stream), and only uncontracted evaluation keeps equal inputs bitwise equal across
# the differently inlined call sites. The residual itself is continuous there and keeps FMA.
PER_FILE_FLAGS = {"jacobians.cu": ["-fmad=false"], "second_order.cu": ["-fmad=false"],
                  "jac_tiled.cu": ["-fmad=false"]}
# The library links only the CUDA runtime: its dense products are its own kernels (dense.cu).
LINK_FLAGS = []


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def sources() -> list[Path]:
    return sorted(CSRC.glob("*.cu"))


def _headers_mtime() -> float:
    return max(p.stat().st_mtime for p in [*CSRC.glob("*.cuh"), *INCLUDE.glob("*.h")])


def _compile(src: Path, force: bool, verbose: bool) -> Path:
    obj = OBJ / (src.stem + ".o")
    if not force and obj.exists() and obj.stat().st_mtime >= max(src.stat().st_mtime,
                                                                  _headers_mtime()):
        return obj
    cmd = [_nvcc(), *NVCC_FLAGS, *PER_FILE_FLAGS.get(src.name, []), "-I", str(INCLUDE), "-c",
           str(src), "-o", str(obj) + ".tmp"]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)
    os.replace(str(obj) + ".tmp", obj)
    return obj


def build_library(force: bool = False, verbose: bool = False) -> Path:
    """Compiles the CUDA sources (stale ones only unless forced) and links the library."""
    OBJ.mkdir(exist_ok=True)
    with ThreadPoolExecutor(max_workers=len(sources())) as pool:
        objs = list(pool.map(lambda s: _compile(s, force, verbose), sources()))
    if not force and LIB.exists() and LIB.stat().st_mtime >= max(o.stat().st_mtime
                                                                 for o in objs):
        return LIB
    cmd = [_nvcc(), "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o",
           str(LIB) + ".tmp", *[str(o) for o in objs], *LINK_FLAGS]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)
    os.replace(str(LIB) + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    print(build_library(force="--force" in sys.argv, verbose=True))
