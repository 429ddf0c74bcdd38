"""The explicit module's LUMPED mass mode on the GPU against the oracle:
diagonal of each node's mass block, a = M^-1 r per DOF, no gyroscopic moment
(ExplicitModule.cpp:154-172, 339-357; SpecialCosseratRodModel.cpp:351-355)."""
import numpy as np
import pytest

from dynlattice_b200 import lattices
from dynlattice_b200.abi import DL_MIXED, DL_PLAIN_FP64
from dynlattice_b200.engine import DLError, Lattice
from helpers import quat_angle_between, rel_err
from oracle_ffi import Oracle

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision,tol", [(DL_PLAIN_FP64, 1e-9), (DL_MIXED, 1e-5)])
def test_lumped_impact_against_oracle(gpu, precision, tol):
    spec = lattices.lattice_impact("bcc", n=3, velocity=20.0, dt=5e-8, plastic=True, seed=7)
    spec.lumped_mass = True
    o = Oracle(spec, threads=4)
    g = Lattice(spec, precision)
    o.run(600)
    g.run(600)
    uo, tho, vo = o.state()
    ug, thg, vg = g.state()
    assert rel_err(ug, uo) < tol
    assert quat_angle_between(thg, tho).max() / max(np.abs(tho).max(), 1e-30) < 10 * tol
    assert rel_err(vg, vo) < 10 * tol
    eo, eg = o.energies(), g.energies()
    for k in ("kinetic", "potential", "dissipated"):
        assert eg[k] == pytest.approx(eo[k], rel=10 * tol), k
    assert eo["dissipated"] > 0.0
    assert g.error_word() == 0


def test_lumped_spinning_rod_against_oracle(gpu):
    """A free rod spinning about a non-principal axis: no gyroscopic moment,
    rotations large enough that the lumped diagonal changes each step."""
    spec = lattices.straight_rod(n_elems=8, tip_force=0.0, dt=1e-5)
    spec.bcs = []
    spec.lumped_mass = True
    w0 = np.array([30.0, 10.0, 5.0])
    v = np.zeros((spec.n_nodes, 6))
    v[:, 3:] = w0
    v[:, :3] = np.cross(w0, spec.coords)
    o = Oracle(spec)
    o.set_state(v=v)
    g = Lattice(spec, DL_PLAIN_FP64)
    g.set_state(v=v)
    o.run(2000)
    g.run(2000)
    uo, tho, vo = o.state()
    ug, thg, vg = g.state()
    assert rel_err(ug, uo) < 1e-9 and rel_err(vg, vo) < 1e-9
    assert quat_angle_between(thg, tho).max() < 1e-9
    assert g.energies()["kinetic"] == pytest.approx(o.energies()["kinetic"], rel=1e-9)


def test_lumped_mode_refused_by_the_adjoint(gpu):
    spec = lattices.lattice_impact("bcc", n=1, velocity=5.0, plastic=False)
    spec.lumped_mass = True
    g = Lattice(spec, DL_PLAIN_FP64)
    with pytest.raises(DLError) as ei:
        g.adjoint_radius(10, 5, elem_param=spec.elem_rod)
    assert ei.value.code == 8  # DL_ERR_UNSUPPORTED
