"""GPU rod--rod contact and rigid plates against the oracle.

The oracle searches every rod pair every step (the reference's algorithm);
the engine evaluates a candidate list built between chunks of steps.  Both
evaluate each pair with the same branch logic in FP64, so the plain FP64
engine must agree with the oracle to 1e-9 relative on the state and the set
of closed pairs must be identical; the mixed path (FP32 element force) to
1e-5.  The engine sums each node's contact forces in the order of its sorted
pair list, which differs from the oracle's serial loop but is the same in
every run.
"""
import numpy as np
import pytest

import contact_cases as cc
from dynlattice_b200 import lattices
from dynlattice_b200.abi import DL_MIXED, DL_PLAIN_FP64
from dynlattice_b200.engine import Lattice
from helpers import rel_err
from oracle_ffi import Oracle

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-9
MIXED_TOL = 1e-5
# closed-pair sets of the mixed path may differ from the oracle's only by
# pairs whose gap d - 2r lies within CONTACT_EPS * r of the threshold (the
# mixed state differs from FP64 by about 1e-5 of the displacement, a few nm
# here, against r = 0.1 mm)
CONTACT_EPS = 1e-4


def _pair_run(spec, steps, u0=None, v0=None, precision=DL_PLAIN_FP64, threads=4):
    o = Oracle(spec, threads=threads)
    g = Lattice(spec, precision)
    if u0 is not None or v0 is not None:
        o.set_state(u=u0, v=v0)
        g.set_state(u=u0, v=v0)
    o.run(steps)
    g.run(steps)
    g.synchronize()
    return o, g


def _compare_states(o, g, tol, v_floor=1e-3):
    """Displacements relative to their largest value; translational
    velocities relative to the larger of their largest value and v_floor (m/s:
    rigidly moved rods carry round-off velocities of 1e-15 m/s)."""
    uo, to, vo = o.state()
    ug, tg, vg = g.state()
    assert rel_err(ug, uo) < tol
    assert rel_err(vg[:, :3], vo[:, :3], max(np.abs(vo[:, :3]).max(), v_floor)) < tol * 10


@pytest.mark.parametrize("case,rod,dz,expect", [
    ("cross", 1, -(0.05e-3 + 0.02e-3), 1),
    ("tee_b_end", 1, -(0.05e-3 + 0.03e-3), 1),
    ("tee_a_end", 0, -(0.05e-3 + 0.03e-3), 0),
    ("parallel", 1, -(cc.PZ - 2 * cc.R + 0.01e-3), None),
])
def test_branch_cases_one_step(gpu, case, rod, dz, expect):
    spec = getattr(cc, case)()
    u0 = cc.shift_rod(spec, rod, (0, 0, dz))
    o, g = _pair_run(spec, 1, u0=u0)
    po, go = o.contact_pairs()
    pg, gg = g.contact_pairs()
    assert np.array_equal(po, pg)
    if expect is not None:
        assert po.shape[0] == expect
    assert np.allclose(gg, go, rtol=1e-12, atol=0)
    # one step of contact gives velocities of ~1e-5 m/s
    _compare_states(o, g, FP64_TOL, v_floor=1e-6)
    assert g.energies()["contact"] == pytest.approx(o.energies()["contact"], rel=1e-12)
    assert g.error_word() == 0


@pytest.mark.parametrize("precision,tol", [(DL_PLAIN_FP64, FP64_TOL), (DL_MIXED, MIXED_TOL)])
def test_cross_impact_history(gpu, precision, tol):
    """Rod 1 thrown onto rod 0 (clamped) at 2 m/s: 4000 steps of approach,
    contact and rebound."""
    spec = cc.rods_spec([((-cc.LEN / 2, 0, 0), (cc.LEN / 2, 0, 0)),
                         ((0.3e-3, -cc.LEN / 2 + 0.3e-3, 2 * cc.R + 0.01e-3),
                          (0.3e-3, cc.LEN / 2 + 0.3e-3, 2 * cc.R + 0.01e-3))], fixed_rods=(0,))
    v0 = np.zeros((spec.n_nodes, 6))
    v0[spec.rod_nodes[1], 2] = -2.0
    o, g = _pair_run(spec, 4000, v0=v0, precision=precision)
    _compare_states(o, g, tol)
    assert g.error_word() == 0


def _fibre_case(n_rods, seed, speed):
    spec = lattices.fibre_network(n_rods=n_rods, seed=seed, plate_velocity=5.0)
    rng = np.random.default_rng(seed)
    v0 = np.zeros((spec.n_nodes, 6))
    per_rod = rng.normal(scale=speed, size=(n_rods, 3))
    v0[:, :3] = np.repeat(per_rod, 5, axis=0)
    return spec, v0


@pytest.mark.parametrize("precision,tol", [(DL_PLAIN_FP64, FP64_TOL), (DL_MIXED, MIXED_TOL)])
def test_fibre_network_random_velocities(gpu, precision, tol):
    """300 rods (same density as the 20 000-rod network), random rod
    velocities of 20 m/s and both plates: 3000 steps; closed pairs of the last
    step, contact energy, plate reactions and the state against the oracle."""
    spec, v0 = _fibre_case(300, 3, 20.0)
    o, g = _pair_run(spec, 3000, v0=v0, precision=precision)
    po, go = o.contact_pairs()
    pg, gg = g.contact_pairs()
    assert po.shape[0] > 0
    # identical sets, except pairs whose gap sits within EPS of the closing
    # threshold d = 2r (FP64: none at all)
    gap_o = {tuple(p): x for p, x in zip(po, go)}
    gap_g = {tuple(p): x for p, x in zip(pg, gg)}
    only_o = set(gap_o) - set(gap_g)
    only_g = set(gap_g) - set(gap_o)
    if precision == DL_PLAIN_FP64:
        assert not only_o and not only_g
    eps = CONTACT_EPS * cc.R
    assert all(-eps < gap_o[p] <= 0.0 for p in only_o), [gap_o[p] for p in only_o]
    assert all(-eps < gap_g[p] <= 0.0 for p in only_g), [gap_g[p] for p in only_g]
    _compare_states(o, g, tol)
    eo, eg = o.energies(), g.energies()
    assert eg["contact"] == pytest.approx(eo["contact"], rel=max(tol, 1e-9) * 100)
    ro, rg = o.plate_reaction(), g.plate_reaction()
    assert np.abs(rg - ro).max() <= max(tol, 1e-9) * 100 * max(np.abs(ro).max(), 1e-30)
    assert g.error_word() == 0


def test_fast_motion_short_chunks(gpu):
    """Rods at 500 m/s: the engine shortens its list chunks (margin / speed)
    and never lets the list go stale."""
    spec, v0 = _fibre_case(100, 5, 500.0)
    o, g = _pair_run(spec, 400, v0=v0)
    _compare_states(o, g, FP64_TOL)
    assert g.error_word() == 0


def test_blacklist_gpu(gpu):
    spec = cc.cross(gap0=-0.02e-3)
    o, g = _pair_run(spec, 20)
    assert o.blacklist_size() == 1
    pg, _ = g.contact_pairs()
    assert pg.shape[0] == 0
    _compare_states(o, g, FP64_TOL)


@pytest.mark.parametrize("precision", [DL_PLAIN_FP64, DL_MIXED])
def test_contact_runs_are_bitwise_repeatable(gpu, precision):
    """Contact forces are summed per node in a fixed order (pairs sorted by
    element indices, each node's pair ends in pair order), not by atomics:
    two identical runs with contact, list rebuilds and plates give the same
    bits."""
    spec, v0 = _fibre_case(300, 3, 20.0)
    states = []
    for _ in range(2):
        g = Lattice(spec, precision)
        g.set_state(v=v0)
        g.run(1500)
        g.synchronize()
        states.append(g.state())
        assert g.contact_stats()[1] > 1  # the list was rebuilt during the run
    for a, b in zip(states[0], states[1]):
        assert np.array_equal(a, b)
