"""The .pro input surface on the reference's own benchmark inputs
(tests/golden/pro: copies of dynLattice's tests/transient and tests/contact
inputs made by tests/golden/make_pro_fixtures.py)."""
import shutil
from pathlib import Path

import numpy as np
import pytest

import transient_cases as tc
from dynlattice_b200.abi import DL_INTEG_MILNE
from dynlattice_b200.engine import DLError
from dynlattice_b200.pro import ProModel
from helpers import rel_err
from oracle_ffi import Oracle

PRO = Path(__file__).resolve().parent / "golden" / "pro"


def test_transient_inputs():
    p1 = ProModel(PRO / "transient" / "test1.pro")
    assert (p1.n_nodes, p1.n_elems, p1.nodes_per_elem, p1.n_gauss) == (9, 4, 3, 2)
    assert p1.dt == 5e-5 and p1.steps == 600000
    assert p1.group("fixed").tolist() == [0] and p1.group("free").tolist() == [1]
    d = p1.desc()
    m = d.materials[0]
    assert m.young == pytest.approx(5.6e10 / 12) and m.area == pytest.approx(12 / 2e3)
    assert m.area_moment[0] == pytest.approx((12 / 2e3) ** 2 / 12)
    # the LoadScale-wrapped Dirichlet on rz is the last constraint of the fixed node
    b = d.bcs[d.n_bcs - 1]
    assert (b.kind, b.dof, b.factor) == (0, 5, 1.0) and b"cos" in b.scale
    assert d.so3_update == 0        # no dofs_SO3: additive rotation update
    p2 = ProModel(PRO / "transient" / "test2.pro")
    assert (p2.n_nodes, p2.n_elems, p2.nodes_per_elem, p2.n_gauss) == (11, 10, 2, 1)
    assert p2.steps == 1000000
    # gmsh numbering: the two points first, then the interior nodes of the line
    assert np.allclose(p2.coords[:2, 0], [0.0, 1.0]) and np.allclose(p2.coords[2:, 0], np.arange(1, 10) / 10)
    # explicit module: MilneDevice (ExplicitModule.cpp:124-148); test1/test2
    # give no precision (the engine's default), test3 gives 1e-4
    assert p1.integrator.kind == DL_INTEG_MILNE and p1.integrator.precision == tc.MILNE_PRECISION
    assert p1.t_end == pytest.approx(30.0) and p2.t_end == pytest.approx(1.0)
    p3 = ProModel(PRO / "transient" / "test3.pro")
    assert p3.integrator.kind == DL_INTEG_MILNE and p3.integrator.precision == 1e-4
    assert (p3.n_nodes, p3.n_elems) == (41, 20) and p3.desc().so3_update == 1
    assert p3.group("elbow").tolist() == [1]
    assert p3.desc().materials[0].inertia_correct == 1e4


def test_static_input_rejected():
    with pytest.raises(DLError, match="explicit integrator"):
        ProModel(PRO / "contact" / "test1.pro")


def _perm(a_coords, b_coords):
    """index map i -> j with a_coords[i] == b_coords[j]"""
    out = []
    for x in a_coords:
        j = int(np.argmin(np.linalg.norm(b_coords - x, axis=1)))
        assert np.linalg.norm(b_coords[j] - x) < 1e-12
        out.append(j)
    return np.array(out)


def test_pro_model_equals_hand_built_model():
    """The swinging rod read from test2.pro steps exactly like the same model
    written by hand (tests/transient_cases.py), up to the node numbering."""
    p = ProModel(PRO / "transient" / "test2.pro")
    h = tc.swinging_rod()
    op, oh = Oracle(p), Oracle(h)
    op.run(3000)
    oh.run(3000)
    up, _, vp = op.state()
    uh, _, vh = oh.state()
    perm = _perm(p.coords, h.coords)
    assert rel_err(up, uh[perm]) < 1e-12 and rel_err(vp, vh[perm]) < 1e-12


def test_pro_spin_up_beam_literature():
    """test1.pro end to end (quadratic elements, oracle): within the reference
    test's 5 % of Simo & Vu-Quoc."""
    p = ProModel(PRO / "transient" / "test1.pro")
    o = Oracle(p)
    fixed, free = int(p.group("fixed")[0]), int(p.group("free")[0])
    o.set_sampling(20, [fixed, free])
    o.run(p.steps)
    steps, rows, _ = o.samples()
    errs = tc.spin_up_errors(steps * p.dt, rows[:, 0, 5], rows[:, 1, 0:3], rows[:, 1, 5], tc.literature())
    assert max(errs.values()) <= 0.05, errs


def _write_msh(path, coords, conn, version):
    with open(path, "w") as f:
        if version == 2:
            f.write("$MeshFormat\n2.2 0 8\n$EndMeshFormat\n$Nodes\n%d\n" % len(coords))
            for i, x in enumerate(coords):
                f.write("%d %.17g %.17g %.17g\n" % (i + 1, *x))
            f.write("$EndNodes\n$Elements\n%d\n" % len(conn))
            for k, (a, b) in enumerate(conn):
                f.write("%d 1 2 0 1 %d %d\n" % (k + 1, a + 1, b + 1))
            f.write("$EndElements\n")
        else:
            f.write("$MeshFormat\n4.1 0 8\n$EndMeshFormat\n")
            n = len(coords)
            f.write("$Nodes\n1 %d 1 %d\n1 1 0 %d\n" % (n, n, n))
            for i in range(n):
                f.write("%d\n" % (i + 1))
            for x in coords:
                f.write("%.17g %.17g %.17g\n" % tuple(x))
            f.write("$EndNodes\n$Elements\n1 %d 1 %d\n1 1 1 %d\n" % (len(conn), len(conn), len(conn)))
            for k, (a, b) in enumerate(conn):
                f.write("%d %d %d\n" % (k + 1, a + 1, b + 1))
            f.write("$EndElements\n")


@pytest.mark.parametrize("version", [2, 4])
def test_msh_input(tmp_path, version):
    """The same rod from a gmsh .msh file (formats 2.2 and 4.1)."""
    src = PRO / "transient"
    for n in ("test2.pro", "input.pro", "model.pro", "output.pro"):
        shutil.copyfile(src / n, tmp_path / n)
    g = ProModel(src / "test2.pro")
    _write_msh(tmp_path / "test2.msh", g.coords, g.conn, version)
    txt = (tmp_path / "input.pro").read_text().replace("$(CASE_NAME).geo", "$(CASE_NAME).msh")
    (tmp_path / "input.pro").write_text(txt)
    p = ProModel(tmp_path / "test2.pro")
    assert np.array_equal(p.coords, g.coords) and np.array_equal(p.conn, g.conn)
    assert p.group("free").tolist() == g.group("free").tolist()


def test_property_language(tmp_path):
    """includes, +=, references (leaves and subtrees), $(key) substitution,
    blocks and numeric expressions in strings."""
    (tmp_path / "rod.geo").write_text("L = 2;\nPoint(1) = {0, 0, 0, 0.5};\nPoint(2) = {L, 0, 0, 0.5};\n"
                                      "Line(1) = {1, 2};\n")
    (tmp_path / "inc.pro").write_text('params.mat = { type = "ElasticRod"; young = "2*1e9"; '
                                      'shear_modulus = 1e9; area = 1e-4; area_moment = [1e-9, 2e-9]; '
                                      'density = 1000.; };\n')
    (tmp_path / "case.pro").write_text(
        'include "inc.pro";\n'
        'control.runWhile = "i <= 7";\n'
        'Solver.modules = [ "integrator" ];\nSolver.integrator.type = "LeapFrog";\n'
        'Solver.integrator.deltaTime = 1e-6;\nSolver.integrator.dofs_SO3 = [ "rx", "ry", "rz" ];\n'
        'Input.input.type = "GMSHInput";\nInput.input.file = "rod.geo";\n'
        'Input.groupInput.type = "GroupInput";\nInput.groupInput.nodeGroups = [ "left" ];\n'
        'Input.groupInput.left.xtype = "min";\nInput.groupInput.nodeGroups += "right";\n'
        'Input.groupInput.right.xval = 2.;\n'
        'model.type = "Matrix";\nmodel.model.type = "Multi";\nmodel.model.models = [ "rods", "bc" ];\n'
        'model.model.rods.type = "Lattice";\nmodel.model.rods.prefix = "beam_";\n'
        'model.model.rods.child.type = "specialCosseratRod";\n'
        'model.model.rods.child.material = params.mat;\n'
        'params.load = 3.5;\n'
        'model.model.bc.type = "Neumann";\nmodel.model.bc.initLoad = "$(params.load) * 2";\n'
        'model.model.bc.loadIncr = 0.;\nmodel.model.bc.nodeGroups = [ "right" ];\n'
        'model.model.bc.dofs = [ "dy" ];\nmodel.model.bc.factors = [ -1. ];\n')
    p = ProModel(tmp_path / "case.pro")
    assert p.n_elems == 4 and p.steps == 7 and p.desc().so3_update == 1
    assert p.group("left").tolist() == [0] and p.group("right").tolist() == [1]
    m = p.desc().materials[0]
    assert m.area_moment[1] == 2e-9 and m.density == 1000.0
    b = p.desc().bcs[0]
    assert b.kind == 1 and b.dof == 1 and b.factor == -1.0 and b.scale.startswith(b"7 + i")


def test_unapplied_properties_are_noted():
    """The reference's test3 sets Solver.integrator.updateWhen = "i%20 < 1"
    (mass matrix rebuilt every 20 steps); the engine rebuilds it every step and
    says so in the file's notes.  test2 sets nothing the engine leaves out."""
    p3 = ProModel(PRO / "transient" / "test3.pro")
    assert any("updateWhen" in n for n in p3.notes)
    p2 = ProModel(PRO / "transient" / "test2.pro")
    assert not any("updateWhen" in n for n in p2.notes)


def test_rod_hinges_from_pro(tmp_path):
    """A rod model's "hinges" properties (type rigidHinge) split every rod as
    HingeModel::createHinges_ does and tie each copy to its original; the
    hinged swinging rod of test2.pro follows the unhinged one."""
    for f in (PRO / "transient").iterdir():
        shutil.copy(f, tmp_path / f.name)
    pro = tmp_path / "test2.pro"
    pro.write_text(pro.read_text() + '\nmodel.model.rodMesh.child.hinges.type = "rigidHinge";\n'
                                      'model.model.rodMesh.child.hinges.yieldCond = "abs(rx) - 1";\n')
    ph = ProModel(pro)
    p = ProModel(PRO / "transient" / "test2.pro")
    assert ph.n_elems == p.n_elems and ph.n_nodes == p.n_nodes + p.n_elems + 1
    d = ph.desc()
    assert d.n_ties == p.n_elems + 1
    assert any("hinges" in n for n in ph.notes)
    oh, op = Oracle(ph), Oracle(p)
    oh.run(2000)
    op.run(2000)
    uh, _, vh = oh.state()
    up, _, vp = op.state()
    N = p.n_nodes
    assert rel_err(uh[:N], up) < 1e-10 and rel_err(vh[:N], vp) < 1e-9
