"""Build the engine library in-tree for sm_100a (``python -m dynlattice_b200.build``).

Runs ``make`` in ``dynlattice_b200/csrc``; the result is
``dynlattice_b200/libdynlattice_b200.so``.  nvcc cross-compiles, so this works
on a machine without a GPU.
"""
from __future__ import annotations

import subprocess
import sys
from pathlib import Path

CSRC = Path(__file__).resolve().parent / "csrc"


def build(jobs: int = 8, verbose: bool = False) -> Path:
    out = None if verbose else subprocess.DEVNULL
    subprocess.run(["make", "-C", str(CSRC), f"-j{jobs}"], check=True, stdout=out)
    return CSRC.parent / "libdynlattice_b200.so"


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
