#!/usr/bin/env python3
"""Copy the reference's transient, contact and plastic benchmark inputs (.pro
and .geo files of dynLattice's tests/transient, tests/contact and
tests/plastic) into tests/golden/pro/, so that the .pro front end is tested on
the inputs the reference itself runs and the static benchmark models of
tests/static_cases.py can be read beside the files they restate.

Usage: python tests/golden/make_pro_fixtures.py /path/to/dynLattice
"""
import shutil
import sys
from pathlib import Path


def main(ref_root):
    out = Path(__file__).resolve().parent / "pro"
    for sub, names in (("transient", ["test1.pro", "test1.geo", "test2.pro", "test2.geo", "test3.pro", "test3.geo",
                                      "input.pro", "model.pro", "output.pro"]),
                       ("contact", ["test1.pro", "test1.geo", "input.pro", "model.pro", "output.pro"]),
                       ("plastic", ["test1.pro", "test1.geo", "test2a.pro", "test2a.geo", "test2b.pro", "test2b.geo",
                                    "test3.pro", "test3.geo", "input.pro", "model.pro", "output.pro"])):
        d = out / sub
        d.mkdir(parents=True, exist_ok=True)
        for n in names:
            shutil.copyfile(Path(ref_root) / "tests" / sub / n, d / n)
    print("wrote", out)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit(f"usage: python {Path(__file__).name} <path of the dynLattice source tree>")
    main(sys.argv[1])
