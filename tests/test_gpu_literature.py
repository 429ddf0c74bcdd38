"""The engine on the reference's transient benchmark with linear elements
(tests/transient/test2 of dynLattice, Lang et al. 2011 swinging rod): rod
shapes against the digitised literature curves at the reference test's 5 %
tolerance, and the state against the oracle."""
import numpy as np
import pytest

import transient_cases as tc
from dynlattice_b200.abi import DL_MIXED, DL_PLAIN_FP64
from dynlattice_b200.engine import Lattice
from helpers import rel_err
from oracle_ffi import Oracle

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", [DL_PLAIN_FP64, DL_MIXED])
def test_swinging_rod_literature(gpu, precision):
    lit = tc.literature()
    spec = tc.swinging_rod()
    g = Lattice(spec, precision)
    shapes, step = [], 0
    for t in lit["test2_times"]:
        k = int(round(t / spec.dt)) - step
        if k > 0:
            g.run(k)
            step += k
        u, _, _ = g.state()
        x = spec.coords + u
        shapes.append(np.stack([x[:, 0], x[:, 2]], 1))
    g.synchronize()
    errs = tc.swinging_errors(lit["test2_times"], shapes, lit)
    assert max(errs.values()) <= 0.05, errs


def test_swinging_rod_vs_oracle(gpu):
    spec = tc.swinging_rod()
    o = Oracle(spec, threads=1)
    g = Lattice(spec, DL_PLAIN_FP64)
    o.run(100000)
    g.run(100000)
    g.synchronize()
    uo, _, vo = o.state()
    ug, _, vg = g.state()
    assert rel_err(ug, uo) < 1e-9
    assert rel_err(vg, vo) < 1e-8
