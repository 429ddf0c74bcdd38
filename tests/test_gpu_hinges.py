"""Rigid hinges (HingeModel ties, condensed) on the GPU against the oracle:
every member of a tie group sums the group's end forces in one fixed order
and carries the group's mass, so the members stay bitwise equal."""
import numpy as np
import pytest

from dynlattice_b200 import lattices
from dynlattice_b200.abi import DL_MIXED, DL_PLAIN_FP64
from dynlattice_b200.engine import DLError, Lattice
from helpers import quat_angle_between, rel_err
from oracle_ffi import Oracle

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision,tol", [(DL_PLAIN_FP64, 1e-9), (DL_MIXED, 1e-5)])
def test_hinged_impact_against_oracle(gpu, precision, tol):
    spec = lattices.with_hinges(lattices.lattice_impact("bcc", n=3, velocity=20.0, dt=5e-8, plastic=True, seed=5))
    o = Oracle(spec, threads=4)
    g = Lattice(spec, precision)
    o.run(600)
    g.run(600)
    uo, tho, vo = o.state()
    ug, thg, vg = g.state()
    assert rel_err(ug, uo) < tol
    assert rel_err(vg, vo) < 10 * tol
    assert quat_angle_between(thg, tho).max() / max(np.abs(tho).max(), 1e-30) < 10 * tol
    m, s = spec.ties[:, 0], spec.ties[:, 1]
    assert np.array_equal(ug[s], ug[m]) and np.array_equal(vg[s], vg[m])
    eo, eg = o.energies(), g.energies()
    for k in ("kinetic", "potential", "dissipated"):
        assert eg[k] == pytest.approx(eo[k], rel=10 * tol), k
    assert eo["dissipated"] > 0.0
    assert g.error_word() == 0


def test_hinged_equals_unhinged_on_the_gpu(gpu):
    base = lattices.lattice_impact("bcc", n=3, velocity=20.0, dt=5e-8, plastic=True, seed=5)
    a = Lattice(base, DL_PLAIN_FP64)
    b = Lattice(lattices.with_hinges(base), DL_PLAIN_FP64)
    a.run(500)
    b.run(500)
    ua, _, va = a.state()
    ub, _, vb = b.state()
    N = base.n_nodes
    assert rel_err(ub[:N], ua) < 1e-10 and rel_err(vb[:N], va) < 1e-9


def test_hinges_refused_where_not_provided(gpu):
    spec = lattices.with_hinges(lattices.lattice_impact("bcc", n=1, velocity=5.0, plastic=False))
    g = Lattice(spec, DL_PLAIN_FP64)
    with pytest.raises(DLError) as ei:
        g.adjoint_radius(10, 5, elem_param=spec.elem_rod)
    assert ei.value.code == 8
    spec.lumped_mass = True
    with pytest.raises(DLError) as ei:
        Lattice(spec, DL_PLAIN_FP64)
    assert ei.value.code == 8
