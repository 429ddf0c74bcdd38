#!/usr/bin/env python3
"""Build tests/golden/transient_literature.npz from the reference's transient
test data (tests/transient/ref_data of dynLattice): digitised literature curves
the reference compares its own runs against at 5 % (Simo & Vu-Quoc 1988
example 5.1 for test 1, Lang et al. 2011 example 1 for test 2).

Usage: python tests/golden/make_transient_fixtures.py /path/to/dynLattice
Run once where the reference checkout exists; the tests read the .npz only.
"""
import sys
from pathlib import Path

import numpy as np


def _semicolon_decimal_comma(path):
    """';'-separated, ','-decimal pairs.  The reference's test reads these with
    pandas' default header=0, so the first line is a header and not data."""
    rows = []
    for line in Path(path).read_text().splitlines()[1:]:
        line = line.strip()
        if not line or ";" not in line:
            continue
        a, b = line.split(";")[:2]
        try:
            rows.append((float(a.replace(",", ".")), float(b.replace(",", "."))))
        except ValueError:
            continue  # header
    return np.array(rows)


def main(ref_root):
    d = Path(ref_root) / "tests" / "transient" / "ref_data"
    out = {}
    out["test1_bc"] = np.loadtxt(d / "test1_ref_BC.csv", delimiter=",")
    out["test1_angle"] = _semicolon_decimal_comma(d / "test1_ref_angle.csv")
    out["test1_u1"] = _semicolon_decimal_comma(d / "test1_ref_u1.csv")
    out["test1_u2"] = _semicolon_decimal_comma(d / "test1_ref_u2.csv")
    lines = (d / "test2_ref.csv").read_text().splitlines()
    times = lines[0].split(",")
    data = [[float(x) if x.strip() else np.nan for x in ln.split(",")] for ln in lines[2:] if ln.strip()]
    data = np.array(data)
    snap_t = []
    for j in range(0, len(times), 2):
        t = float(times[j][1:])
        xy = data[:, j:j + 2]
        xy = xy[~np.isnan(xy).any(axis=1)]
        out[f"test2_t{t:.1f}"] = xy
        snap_t.append(t)
    out["test2_times"] = np.array(snap_t)
    target = Path(__file__).resolve().parent / "transient_literature.npz"
    np.savez_compressed(target, **out)
    print("wrote", target, {k: v.shape for k, v in out.items()})


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit(f"usage: python {Path(__file__).name} <path of the dynLattice source tree>")
    main(sys.argv[1])
