"""Build recipe of ``libtreed3d.so``, the sm_100a CUDA library behind the C ABI.

``python -m tree_d_3d_b200.build`` (or ``__graft_entry__.build()``) compiles every
``csrc/*.cu`` for sm_100a only (``-gencode arch=compute_100a,code=sm_100a``) with
``nvcc`` and links them into ``tree_d_3d_b200/libtreed3d.so`` next to this file.
Objects go to ``_build/`` beside it; sources newer than their object are rebuilt.
"""

from __future__ import annotations

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent
CSRC = HERE / "csrc"
BUILD = HERE / "_build"
LIBRARY = HERE / "libtreed3d.so"
INCLUDE = ROOT / "include"

NVCC = os.environ.get("NVCC", "nvcc")
FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC",
    "--expt-relaxed-constexpr",
    f"-I{INCLUDE}", f"-I{CSRC}",
]


#: Sources whose every multiply-add must round twice, as the reference's CPU code
#: (integer / decision work and the moments): compiled without FMA contraction.
NO_FMA = {"build.cu", "moments.cu", "traverse.cu"}


def _headers_mtime() -> float:
    files = list(CSRC.glob("*.cuh")) + list(INCLUDE.glob("*.h"))
    return max((f.stat().st_mtime for f in files), default=0.0)


def _compile(source: Path, verbose: bool) -> Path:
    obj = BUILD / (source.stem + ".o")
    newest = max(source.stat().st_mtime, _headers_mtime())
    if obj.exists() and obj.stat().st_mtime >= newest:
        return obj
    cmd = [NVCC, *FLAGS, "-c", str(source), "-o", str(obj)]
    if source.name in NO_FMA:
        cmd.insert(1, "--fmad=false")
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    subprocess.run(cmd, check=True)
    return obj


def build(verbose: bool = False) -> Path:
    BUILD.mkdir(exist_ok=True)
    sources = sorted(CSRC.glob("*.cu"))
    with ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as pool:
        objects = list(pool.map(lambda s: _compile(s, verbose), sources))
    newest = max(o.stat().st_mtime for o in objects)
    if not LIBRARY.exists() or LIBRARY.stat().st_mtime < newest:
        cmd = [NVCC, "-shared", "-gencode", "arch=compute_100a,code=sm_100a",
               *(str(o) for o in objects), "-o", str(LIBRARY), "-lcudart"]
        subprocess.run(cmd, check=True)
    return LIBRARY


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
