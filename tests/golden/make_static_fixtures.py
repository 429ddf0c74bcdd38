#!/usr/bin/env python3
"""Build tests/golden/static_literature.npz from the reference's quasi-static
benchmark data (dynLattice tests/plastic/ref_data and tests/contact/test1.py):

* plastic test 1, 2a, 2b: Smriti et al. (2021) hysteresis loops (axial strain
  in 1e-3 for test 1, axial load per yield limit), compared by the reference
  through their envelopes (tests/plastic/test1.py, test2a.py, test2b.py);
* plastic test 3: Herrnboeck et al. (2023) force and moment curves over the
  load factor, with the column pairing of tests/plastic/test3.py (the
  reference's rod runs along y, so its dy force is the paper's axial n3);
* contact test 1: the contact force per load step of Zavarise & Wriggers
  (2000), the array `ref_disp` of tests/contact/test1.py.

Usage: python tests/golden/make_static_fixtures.py /path/to/dynLattice
Run once where the reference checkout exists; the tests read the .npz only.
"""
import re
import sys
from pathlib import Path

import numpy as np


def _sorted(a):
    return a[a[:, 0].argsort()]


def main(ref_root):
    d = Path(ref_root) / "tests" / "plastic" / "ref_data"
    out = {}
    for name in ("test1", "test2a", "test2b"):
        out[f"plastic_{name}"] = np.loadtxt(d / f"{name}_ref.csv", delimiter=",")
    f, m = d / "test3_ref_force.csv", d / "test3_ref_torque.csv"
    # (columns, max_rows) exactly as tests/plastic/test3.py reads them
    out["plastic_test3_n0"] = _sorted(np.loadtxt(f, delimiter=",", skiprows=2, usecols=(0, 1)))
    out["plastic_test3_n1"] = _sorted(np.loadtxt(f, delimiter=",", skiprows=2, usecols=(4, 5), max_rows=32))
    out["plastic_test3_n2"] = _sorted(np.loadtxt(f, delimiter=",", skiprows=2, usecols=(2, 3), max_rows=27))
    out["plastic_test3_m0"] = _sorted(np.loadtxt(m, delimiter=",", skiprows=2, usecols=(0, 1), max_rows=32))
    out["plastic_test3_m1"] = _sorted(np.loadtxt(m, delimiter=",", skiprows=2, usecols=(4, 5), max_rows=33))
    out["plastic_test3_m2"] = _sorted(np.loadtxt(m, delimiter=",", skiprows=2, usecols=(2, 3)))
    src = (Path(ref_root) / "tests" / "contact" / "test1.py").read_text()
    arr = re.search(r"ref_disp\s*=\s*np\.array\(\[([^\]]*)\]\)", src)
    out["contact_test1_force"] = np.array([float(x) for x in arr.group(1).split(",")])
    target = Path(__file__).resolve().parent / "static_literature.npz"
    np.savez_compressed(target, **out)
    print("wrote", target, {k: v.shape for k, v in out.items()})


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit(f"usage: python {Path(__file__).name} <path of the dynLattice source tree>")
    main(sys.argv[1])
