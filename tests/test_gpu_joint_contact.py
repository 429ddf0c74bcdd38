"""GPU joint contact (JointContactModel) against the oracle.

The oracle tests every joint pair in every step (the reference's
findContacts_); the engine evaluates a candidate list of joint pairs built
on the device between chunks of steps (hash grid, 27-cell query).  Both apply
the same force in FP64, so the plain FP64 engine agrees with the oracle to
1e-9 relative on the state and the sets of joint pairs in contact are
identical; the mixed path (FP32 element force) to 1e-5.  The engine sums each
node's joint forces in the order of its sorted pair list, which differs from
the oracle's serial loop but is the same in every run."""
import numpy as np
import pytest

import joint_cases as jc
from dynlattice_b200.abi import DL_MIXED, DL_PLAIN_FP64, Integrator
from dynlattice_b200.engine import DLError, Lattice
from helpers import rel_err
from oracle_ffi import Oracle

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-9
MIXED_TOL = 1e-5


def _run(spec, steps, u0=None, v0=None, precision=DL_PLAIN_FP64):
    o = Oracle(spec, threads=4)
    g = Lattice(spec, precision)
    if u0 is not None or v0 is not None:
        o.set_state(u=u0, v=v0)
        g.set_state(u=u0, v=v0)
    o.run(steps)
    g.run(steps)
    g.synchronize()
    return o, g


def _compare(o, g, tol, v_floor=1e-3):
    uo, _, vo = o.state()
    ug, _, vg = g.state()
    assert rel_err(ug, uo) < tol
    assert rel_err(vg[:, :3], vo[:, :3], max(np.abs(vo[:, :3]).max(), v_floor)) < tol * 10


def test_tips_one_step(gpu):
    spec = jc.tips()
    u0 = jc.tips_closed_state(spec)
    o, g = _run(spec, 1, u0=u0)
    po, go = o.joint_contact_pairs()
    pg, gg = g.joint_contact_pairs()
    assert po.shape[0] == 1 and np.array_equal(po, pg)
    assert np.allclose(gg, go, rtol=1e-12, atol=0)
    _compare(o, g, FP64_TOL, v_floor=1e-6)
    assert g.energies()["contact"] == pytest.approx(o.energies()["contact"], rel=1e-12)
    assert g.error_word() == 0


def test_coincident_joints(gpu):
    spec = jc.tips()
    u0 = jc.tips_closed_state(spec, shift=(-jc.GAP, 0.0, 0.0))
    o, g = _run(spec, 1, u0=u0)
    pg, gg = g.joint_contact_pairs()
    assert len(pg) == 1 and gg[0] == -2 * jc.RJ
    _compare(o, g, FP64_TOL, v_floor=1e-6)
    assert np.isfinite(g.state()[2]).all()


@pytest.mark.parametrize("precision,tol", [(DL_PLAIN_FP64, FP64_TOL), (DL_MIXED, MIXED_TOL)])
def test_tips_thrown_together(gpu, precision, tol):
    """Rod B thrown at rod A at 30 m/s: 6000 steps of approach and attraction."""
    spec = jc.tips()
    v0 = np.zeros((spec.n_nodes, 6))
    v0[spec.rod_nodes[1], 0] = -30.0
    v0[spec.rod_nodes[1], 1] = 3.0
    o, g = _run(spec, 6000, v0=v0, precision=precision)
    assert o.joint_contact_pairs()[0].shape[0] == 1
    assert np.array_equal(o.joint_contact_pairs()[0], g.joint_contact_pairs()[0])
    _compare(o, g, tol)
    assert g.energies()["contact"] == pytest.approx(o.energies()["contact"], rel=max(tol, 1e-9) * 100)
    assert g.error_word() == 0


@pytest.mark.parametrize("precision,tol", [(DL_PLAIN_FP64, FP64_TOL), (DL_MIXED, MIXED_TOL)])
def test_fibre_network_joints(gpu, precision, tol):
    """300 random rods with random velocities of 20 m/s, rod--rod contact,
    both plates and joint contact of the 600 rod ends (r = 1 mm): 3000
    steps; joint pairs of the last step, contact energy and state."""
    spec = jc.fibre_joints(300, 3)
    rng = np.random.default_rng(3)
    v0 = np.zeros((spec.n_nodes, 6))
    v0[:, :3] = np.repeat(rng.normal(scale=20.0, size=(300, 3)), spec.n_nodes // 300, axis=0)
    o, g = _run(spec, 3000, v0=v0, precision=precision)
    po, _ = o.joint_contact_pairs()
    pg, _ = g.joint_contact_pairs()
    assert po.shape[0] > 5
    diff = {tuple(p) for p in po} ^ {tuple(p) for p in pg}
    assert len(diff) == 0 or precision == DL_MIXED
    _compare(o, g, tol)
    assert g.energies()["contact"] == pytest.approx(o.energies()["contact"], rel=max(tol, 1e-9) * 100)
    assert g.error_word() == 0


def test_candidate_list_matches_brute_force(gpu):
    """At the state where the pairs of the last step were evaluated, the
    engine's pairs equal an all-pairs search (hash-grid completeness)."""
    spec = jc.fibre_joints(300, 4, plates=False)
    rng = np.random.default_rng(4)
    v0 = np.zeros((spec.n_nodes, 6))
    v0[:, :3] = np.repeat(rng.normal(scale=20.0, size=(300, 3)), spec.n_nodes // 300, axis=0)
    g = Lattice(spec, DL_PLAIN_FP64)
    g.set_state(v=v0)
    g.run(1999)
    u_prev = g.state()[0]
    g.run(1)
    pg, _ = g.joint_contact_pairs()
    want = jc.brute_pairs(spec, u_prev)
    assert len(want) > 5 and [tuple(p) for p in pg] == want


def test_milne_refuses_joint_contact(gpu):
    g = Lattice(jc.tips(), DL_PLAIN_FP64)
    with pytest.raises(DLError, match="contact"):
        g.set_integrator(Integrator.milne(1e-6))


def test_joint_contact_runs_are_bitwise_repeatable(gpu):
    """Joint forces are summed per node in a fixed order (pairs sorted by
    node indices): two identical runs give the same bits."""
    spec = jc.fibre_joints(300, 4)
    rng = np.random.default_rng(4)
    v0 = np.zeros((spec.n_nodes, 6))
    v0[:, :3] = np.repeat(rng.normal(scale=20.0, size=(300, 3)), spec.n_nodes // 300, axis=0)
    states = []
    for _ in range(2):
        g = Lattice(spec, DL_MIXED)
        g.set_state(v=v0)
        g.run(800)
        g.synchronize()
        states.append(g.state())
    for a, b in zip(states[0], states[1]):
        assert np.array_equal(a, b)
