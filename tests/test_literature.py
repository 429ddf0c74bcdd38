"""The oracle against the reference's own transient benchmarks
(tests/transient/test1 and test2 of dynLattice): the same models, the same
comparison metrics and the same 5 % tolerance against the digitised
literature curves those tests use (tests/golden/transient_literature.npz,
made by tests/golden/make_transient_fixtures.py).  The reference integrates
them with MilneDevice; the oracle uses LeapFrog at the same dt."""
import numpy as np

import transient_cases as tc
from oracle_ffi import Oracle

TOL = 0.05


def test_spin_up_beam_simo_vu_quoc():
    lit = tc.literature()
    spec = tc.spin_up_beam()
    o = Oracle(spec, threads=1)
    free = spec.coords.shape[0] - 1
    o.set_sampling(20, [0, free])
    o.run(int(round(30.0 / spec.dt)))
    steps, rows, _ = o.samples()
    errs = tc.spin_up_errors(steps * spec.dt, rows[:, 0, 5], rows[:, 1, 0:3], rows[:, 1, 5], lit)
    assert max(errs.values()) <= TOL, errs


def test_swinging_rod_lang():
    lit = tc.literature()
    spec = tc.swinging_rod()
    o = Oracle(spec, threads=1)
    shapes, step = [], 0
    for t in lit["test2_times"]:
        k = int(round(t / spec.dt)) - step
        if k > 0:
            o.run(k)
            step += k
        u, _, _ = o.state()
        x = spec.coords + u
        shapes.append(np.stack([x[:, 0], x[:, 2]], 1))
    errs = tc.swinging_errors(lit["test2_times"], shapes, lit)
    assert max(errs.values()) <= TOL, errs
