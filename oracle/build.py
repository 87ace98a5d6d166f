"""Build recipe of the CPU oracle: ``oracle/oracle.c`` -> ``oracle/liboracle_td3.so``.

Test infrastructure: the library is the checker of the CUDA path and the timed CPU
baseline of ``bench.py``.  ``-ffp-contract=off`` keeps every multiply-add as the two
rounded operations of the reference's CPU kernels; OpenMP parallelises the loops the
reference parallelises (disjoint outputs per iteration).
"""

from __future__ import annotations

import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
SOURCE = HERE / "oracle.c"
LIBRARY = HERE / "liboracle_td3.so"


def build(force: bool = False) -> Path:
    if not force and LIBRARY.exists() and LIBRARY.stat().st_mtime >= SOURCE.stat().st_mtime:
        return LIBRARY
    cmd = [
        "gcc",
        "-O2",
        "-fPIC",
        "-shared",
        "-fopenmp",
        "-ffp-contract=off",
        "-fno-fast-math",
        "-o",
        str(LIBRARY),
        str(SOURCE),
        "-lm",
    ]
    subprocess.run(cmd, check=True)
    return LIBRARY


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
