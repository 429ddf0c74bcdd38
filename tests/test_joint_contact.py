"""Joint contact (JointContactModel) in the oracle and the .pro input, on the CPU.

No reference test or input uses JointContactModel, so these cases restate
its two functions (findContacts_, JointContactModel.cpp:236-275;
computeContact_, :318-340) in numpy and hold the oracle to them: the pair set
(within 2r now, farther than 2r apart in the reference configuration), the
force -k (2r - d) n on joint A and +k (2r - d) n on joint B, and the "points"
element group of the mesh as the joint list."""
import copy

import numpy as np
import pytest

import joint_cases as jc
from dynlattice_b200.pro import ProModel
from oracle_ffi import Oracle


def _one_step(spec, u0):
    o = Oracle(spec)
    o.set_state(u=u0)
    o.run(1)
    return o


def test_pairs_and_force_one_step():
    spec = jc.tips()
    u0 = jc.tips_closed_state(spec)
    o = _one_step(spec, u0)
    a1, b0 = int(spec.rod_nodes[0][-1]), int(spec.rod_nodes[1][0])
    pairs, gaps = o.joint_contact_pairs()
    assert pairs.tolist() == [[a1, b0]] == [list(p) for p in jc.brute_pairs(spec, u0)]
    f, d = jc.joint_force(spec, u0, a1, b0)
    assert gaps[0] == pytest.approx(d - 2 * jc.RJ, rel=1e-12)
    # the same step without joint contact: the difference of the internal
    # forces at A's end and B's start is the contact force
    plain = copy.copy(spec)
    plain.joint_contact = None
    p = _one_step(plain, u0)
    ra, _ = o.group_sums([a1])
    rb, _ = o.group_sums([b0])
    pa, _ = p.group_sums([a1])
    pb, _ = p.group_sums([b0])
    assert np.allclose(ra[:3] - pa[:3], f, rtol=1e-9, atol=0)
    assert np.allclose(rb[:3] - pb[:3], -f, rtol=1e-9, atol=0)
    assert np.array_equal(ra[3:], pa[3:]) and np.array_equal(rb[3:], pb[3:])
    # B's end and C's start are RJ apart but were within 2r at the start
    c0, b1 = int(spec.rod_nodes[2][0]), int(spec.rod_nodes[1][-1])
    rc, _ = o.group_sums([c0, b1])
    pc, _ = p.group_sums([c0, b1])
    assert np.array_equal(rc, pc)
    assert o.energies()["contact"] == pytest.approx(-0.5 * jc.KJ * (2 * jc.RJ - d) ** 2, rel=1e-12)


def test_coincident_joints_get_no_force():
    """d = 0: the pair is in contact (gap -2r) but has no normal; the
    reference divides by d, the oracle and the engine add nothing."""
    spec = jc.tips()
    u0 = jc.tips_closed_state(spec, shift=(-jc.GAP, 0.0, 0.0))
    o = _one_step(spec, u0)
    pairs, gaps = o.joint_contact_pairs()
    assert len(pairs) == 1 and gaps[0] == -2 * jc.RJ
    u, th, v = o.state()
    assert np.isfinite(u).all() and np.isfinite(v).all()
    plain = copy.copy(spec)
    plain.joint_contact = None
    p = _one_step(plain, u0)
    assert np.array_equal(o.state()[2], p.state()[2])


def test_energy_balance_through_contact():
    """Rod B thrown at rod A: kinetic + strain + joint-contact energy stays
    constant while the tips come into reach and pull together."""
    spec = jc.tips()
    v0 = np.zeros((spec.n_nodes, 6))
    v0[spec.rod_nodes[1], 0] = -30.0
    v0[spec.rod_nodes[1], 1] = 3.0
    o = Oracle(spec)
    o.set_state(v=v0)
    o.set_sampling(50, [0])
    o.run(6000)
    steps, _, en = o.samples()
    tot = en[:, 0] + en[:, 1] + en[:, 4]
    assert (en[:, 4] < 0).any(), "the tips never came into reach"
    assert np.abs(tot - tot[0]).max() < 2e-4 * tot[0]


def test_pro_joint_contact(tmp_path):
    """`jointContact` of the Lattice model: the joints are the nodes of the
    mesh's point elements ("points"); .geo and .msh inputs agree."""
    (tmp_path / "frame.geo").write_text(
        "Point(1) = {0, 0, 0, 0.25};\nPoint(2) = {1, 0, 0, 0.25};\nPoint(3) = {1, 1, 0, 0.25};\n"
        "Line(1) = {1, 2};\nLine(2) = {2, 3};\n")
    (tmp_path / "case.pro").write_text(
        'control.runWhile = "i <= 10";\n'
        'Solver.modules = [ "integrator" ];\nSolver.integrator.type = "LeapFrog";\n'
        'Solver.integrator.deltaTime = 1e-6;\n'
        'Input.input.type = "GMSHInput";\nInput.input.file = "frame.geo";\n'
        'model.type = "Matrix";\nmodel.model.type = "Multi";\nmodel.model.models = [ "rods" ];\n'
        'model.model.rods.type = "Lattice";\nmodel.model.rods.prefix = "beam_";\n'
        'model.model.rods.child.type = "specialCosseratRod";\n'
        'model.model.rods.child.material = { type = "ElasticRod"; young = 1e9; shear_modulus = 4e8; '
        'area = 1e-4; area_moment = [1e-9, 1e-9]; density = 1000.; };\n'
        'model.model.rods.jointContact.type = "JointContact";\n'
        'model.model.rods.jointContact.penalty = 123.;\n'
        'model.model.rods.jointContact.radius = 0.01;\n')
    p = ProModel(tmp_path / "case.pro")
    d = p.desc().joint_contact
    assert d.enabled == 1 and d.penalty == 123.0 and d.radius == 0.01
    joints = [d.joints[i] for i in range(d.n_joints)]
    assert joints == [0, 1, 2] == p.group("points").tolist()
    assert p.group("point_2").tolist() == [1]
    assert np.allclose(p.coords[joints], [[0, 0, 0], [1, 0, 0], [1, 1, 0]])
    # the same mesh as a .msh 4.1 file with its point elements
    with open(tmp_path / "frame.msh", "w") as f:
        f.write("$MeshFormat\n4.1 0 8\n$EndMeshFormat\n")
        n = p.n_nodes
        f.write("$Nodes\n1 %d 1 %d\n1 1 0 %d\n" % (n, n, n))
        for i in range(n):
            f.write("%d\n" % (i + 1))
        for x in p.coords:
            f.write("%.17g %.17g %.17g\n" % tuple(x))
        E = p.n_elems
        f.write("$EndNodes\n$Elements\n2 %d 1 %d\n0 1 15 3\n" % (E + 3, E + 3))
        for k in range(3):
            f.write("%d %d\n" % (k + 1, k + 1))
        f.write("1 1 1 %d\n" % E)
        for k, (a, b) in enumerate(p.conn):
            f.write("%d %d %d\n" % (k + 4, a + 1, b + 1))
        f.write("$EndElements\n")
    (tmp_path / "case2.pro").write_text((tmp_path / "case.pro").read_text().replace("frame.geo", "frame.msh"))
    q = ProModel(tmp_path / "case2.pro")
    dq = q.desc().joint_contact
    assert [dq.joints[i] for i in range(dq.n_joints)] == joints


def test_pro_joint_contact_unknown_type(tmp_path):
    (tmp_path / "rod.geo").write_text("Point(1) = {0, 0, 0, 0.5};\nPoint(2) = {1, 0, 0, 0.5};\nLine(1) = {1, 2};\n")
    (tmp_path / "case.pro").write_text(
        'Solver.modules = [ "integrator" ];\nSolver.integrator.type = "LeapFrog";\n'
        'Solver.integrator.deltaTime = 1e-6;\n'
        'Input.input.type = "GMSHInput";\nInput.input.file = "rod.geo";\n'
        'model.type = "Matrix";\nmodel.model.type = "Multi";\nmodel.model.models = [ "rods" ];\n'
        'model.model.rods.type = "Lattice";\n'
        'model.model.rods.child.type = "specialCosseratRod";\n'
        'model.model.rods.child.material = { type = "ElasticRod"; young = 1e9; shear_modulus = 4e8; '
        'area = 1e-4; area_moment = [1e-9, 1e-9]; density = 1000.; };\n'
        'model.model.rods.jointContact.type = "Hinge";\n')
    with pytest.raises(Exception, match="jointContact"):
        ProModel(tmp_path / "case.pro")
