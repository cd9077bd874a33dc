"""Build the sm_100a shared library ``libpycfd_b200.so`` in-tree with nvcc.

    python -m pycfd_b200.build        (or __graft_entry__.build())

The library is the C ABI of include/pycfd_b200.h: one translation unit
(csrc/solver.cu including the kernel headers), compiled for sm_100a only.  FMA
contraction is on; the stencils that must keep the reference's rounding form
their products with rmul (csrc/common.cuh), which is never fused.
"""

from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIB = os.path.join(HERE, "libpycfd_b200.so")
SOURCES = [os.path.join(HERE, "csrc", "solver.cu")]
HEADERS = [os.path.join(HERE, "csrc", f) for f in os.listdir(os.path.join(HERE, "csrc"))
           if f.endswith((".cuh", ".h"))] + [os.path.join(ROOT, "include", "pycfd_b200.h")]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr", "--extended-lambda",
    "-Xcompiler", "-fPIC", "-shared",
]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.isabs(cand) and os.path.exists(cand) or not os.path.isabs(cand)):
            return cand
    return "nvcc"


def up_to_date() -> bool:
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    return all(os.path.getmtime(f) <= t for f in SOURCES + HEADERS)


def build(force: bool = False, verbose: bool = False) -> str:
    """Compile the library unless it is newer than every source; return its path."""
    if not force and up_to_date():
        return LIB
    # PYCFD_B200_DEFINES: extra -D options (strip heights PCFD_STRIP_ROWS and
    # PCFD_BSTRIP_ROWS, resident-block bounds PCFD_BSTRIP_MINB and PCFD_BELL_MINB,
    # PCFD_BELL_ROUNDS), e.g. "-DPCFD_BSTRIP_ROWS=4"
    extra = os.environ.get("PYCFD_B200_DEFINES", "").split()
    if any(not d.startswith("-D") for d in extra):
        raise ValueError("PYCFD_B200_DEFINES takes -D options only")
    cmd = [nvcc(), *NVCC_FLAGS, *extra, "-o", LIB, *SOURCES]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
