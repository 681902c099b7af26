# SPDX-License-Identifier: Apache-2.0
"""Build of liballoy_dfsph.so (sm_100a) in-tree: ``python -m alloy_b200.build``.

Flags: sm_100a only; -fmad=false so that no multiply-add is fused except the explicit ones the kernels spell out
(their CPU restatement evaluates the same operations in the same order); IEEE division and square root.
"""

from __future__ import annotations

import os
import shutil
import subprocess
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
LIBDIR = PKG / "lib"
LIB = LIBDIR / "liballoy_dfsph.so"
SOURCES = [CSRC / "dfsph_capi.cu", CSRC / "dfsph_noalloc.cu", CSRC / "dfsph_mlp.cu"]
DEPENDS = SOURCES + [CSRC / "dfsph_kernels.cuh", CSRC / "dfsph_mlp.cuh", CSRC / "dfsph_math.cuh", CSRC / "dfsph_reduce.cuh",
                     CSRC / "dfsph_port.cuh", CSRC / "dfsph_skin.cuh", CSRC / "dfsph_persist.cuh",
                     PKG.parent / "include" / "alloy_dfsph.h"]
NVCC_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "-fmad=false", "-prec-div=true",
              "-prec-sqrt=true", "-ftz=false", "-std=c++17", "-Xcompiler", "-fPIC", "-shared"]


def nvcc() -> str:
    path = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(path).exists():
        raise RuntimeError("nvcc not found: the CUDA toolkit is needed to build liballoy_dfsph.so")
    return path


def build(force: bool = False, verbose: bool = False) -> Path:
    """Compile the library if it is missing or older than a source; returns its path."""
    if not force and LIB.exists():
        newest = max(p.stat().st_mtime for p in DEPENDS if p.exists())
        if LIB.stat().st_mtime >= newest:
            return LIB
    LIBDIR.mkdir(exist_ok=True)
    tmp = LIB.with_suffix(f".{os.getpid()}.tmp")
    cmd = [nvcc(), *NVCC_FLAGS, *(["-Xptxas", "-v"] if verbose else []), "-o", str(tmp), *map(str, SOURCES)]
    subprocess.run(cmd, check=True, cwd=str(CSRC))
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force=True, verbose=True))
