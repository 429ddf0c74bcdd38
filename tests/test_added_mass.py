"""Added point masses (MassModel, "Mass" in a .pro file) in the oracle, on the CPU.

MassModel adds totalMass / |group| to the diagonal of the mass matrix for
each listed DOF of each node of the group (MassModel.cpp:77-99); the explicit
module solves with the whole matrix and LatticeModel's kinetic energy uses it
too.  From rest the first step's velocities are dt * F / (m + m_add) per DOF,
which pins the oracle to that statement."""
import numpy as np
import pytest

from dynlattice_b200 import lattices
from dynlattice_b200.abi import BC, DL_BC_MASS, DL_BC_NEUMANN
from dynlattice_b200.pro import ProModel
from oracle_ffi import Oracle

M_ADD = [0.3, 0.5, 0.7, 2e-4, 3e-4, 4e-4]   # kg on dx, dy, dz; kg m^2 on rx, ry, rz


def tip_mass_rod(n_gauss=2):
    """Straight rod along x clamped at x = 0 with a ramped tip force along y,
    a tip moment about z and the masses M_ADD on the tip's six DOFs."""
    spec = lattices.straight_rod(n_elems=8, n_gauss=n_gauss)
    tip = np.array([spec.n_nodes - 1], np.int32)
    spec.bcs.append(BC(DL_BC_NEUMANN, 5, tip, 0.2, "min(i/500, 1)"))
    spec.bcs += [BC(DL_BC_MASS, d, tip, M_ADD[d]) for d in range(6)]
    spec.tip = int(tip[0])
    return spec


def test_first_step_from_rest():
    spec = tip_mass_rod()
    o = Oracle(spec)
    mt, mr = o.mass()
    o.run(1)
    _, _, v = o.state()
    t = spec.tip
    F, Mz = 1.0 / 500, 0.2 / 500
    assert v[t, 1] == pytest.approx(spec.dt * F / (mt[t] + M_ADD[1]), rel=1e-12)
    # the rod lies along x: its rotational block is diagonal in the spatial axes
    assert abs(mr[t, 2, 0]) < 1e-12 * mr[t, 2, 2] and abs(mr[t, 2, 1]) < 1e-12 * mr[t, 2, 2]
    assert v[t, 5] == pytest.approx(spec.dt * Mz / (mr[t, 2, 2] + M_ADD[5]), rel=1e-9)
    # kinetic energy with the added masses
    ek = 0.5 * (mt * (v[:, :3] ** 2).sum(1)).sum() + 0.5 * np.einsum("ni,nij,nj->", v[:, 3:], mr, v[:, 3:])
    ek += 0.5 * sum(M_ADD[d] * v[t, d] ** 2 for d in range(6))
    assert o.energies()["kinetic"] == pytest.approx(ek, rel=1e-12)


def test_gyroscopic_term_uses_added_rotational_mass():
    """The gyroscopic moment omega x (M omega) is formed with the explicit
    module's mass matrix (SpecialCosseratRodModel::assembleGyro_ multiplies
    by the MATRIX2 it is given), so the added rotational masses enter it."""
    spec = tip_mass_rod()
    t = spec.tip
    o = Oracle(spec)
    mt, mr = o.mass()
    v0 = np.zeros((spec.n_nodes, 6))
    w = np.array([0.0, 50.0, 30.0])
    v0[t, 3:] = w
    o.set_state(v=v0)
    o.run(1)
    _, _, v = o.state()
    M = mr[t] + np.diag(M_ADD[3:])
    moment = np.array([0.0, 0.0, 0.2 / 500]) - np.cross(w, M @ w)
    assert np.allclose(v[t, 3:], w + spec.dt * np.linalg.solve(M, moment), rtol=1e-12, atol=0)


def test_energy_balance_with_added_mass():
    """Tip load ramped then held: kinetic + strain energy equals the load's work."""
    spec = tip_mass_rod()
    o = Oracle(spec)
    o.run(3000)
    e = o.energies()
    assert e["external_work"] > 0
    assert e["kinetic"] + e["potential"] == pytest.approx(e["external_work"], rel=2e-3)


def test_pro_mass_model(tmp_path):
    (tmp_path / "rod.geo").write_text("Point(1) = {0, 0, 0, 0.25};\nPoint(2) = {1, 0, 0, 0.25};\nLine(1) = {1, 2};\n")
    (tmp_path / "case.pro").write_text(
        'Solver.modules = [ "integrator" ];\nSolver.integrator.type = "LeapFrog";\n'
        'Solver.integrator.deltaTime = 1e-6;\n'
        'Input.input.type = "GMSHInput";\nInput.input.file = "rod.geo";\n'
        'Input.groupInput.type = "GroupInput";\nInput.groupInput.nodeGroups = [ "right", "all2" ];\n'
        'Input.groupInput.right.xtype = "max";\nInput.groupInput.all2.ytype = "min";\n'
        'model.type = "Matrix";\nmodel.model.type = "Multi";\nmodel.model.models = [ "rods", "mass" ];\n'
        'model.model.rods.type = "Lattice";\n'
        'model.model.rods.child.type = "specialCosseratRod";\n'
        'model.model.rods.child.material = { type = "ElasticRod"; young = 1e9; shear_modulus = 4e8; '
        'area = 1e-4; area_moment = [1e-9, 1e-9]; density = 1000.; };\n'
        'model.model.mass.type = "Mass";\nmodel.model.mass.totalMass = [ 2.0, 5.0 ];\n'
        'model.model.mass.nodeGroups = [ "right", "all2" ];\nmodel.model.mass.dofs = [ "dx", "rz" ];\n')
    p = ProModel(tmp_path / "case.pro")
    d = p.desc()
    got = sorted((d.bcs[i].dof, d.bcs[i].n_nodes, round(d.bcs[i].factor, 12)) for i in range(d.n_bcs)
                 if d.bcs[i].kind == DL_BC_MASS)
    n_all = p.n_nodes
    assert got == sorted([(0, 1, 2.0), (5, 1, 2.0), (0, n_all, round(5.0 / n_all, 12)),
                          (5, n_all, round(5.0 / n_all, 12))])
    (tmp_path / "bad.pro").write_text((tmp_path / "case.pro").read_text().replace("[ 2.0, 5.0 ]", "[ 2.0 ]"))
    with pytest.raises(Exception, match="same length"):
        ProModel(tmp_path / "bad.pro")
