"""GPU added point masses (MassModel) against the oracle: a cantilever with
masses on the tip's six DOFs, and a node whose rotation is partly prescribed
(the masked solve) with added masses, over 2000 steps of a ramped tip load."""
import numpy as np
import pytest

from dynlattice_b200.abi import BC, DL_BC_DIRICHLET, DL_BC_MASS, DL_MIXED, DL_PLAIN_FP64, Integrator
from dynlattice_b200.engine import DLError, Lattice
from helpers import rel_err
from oracle_ffi import Oracle
from test_added_mass import tip_mass_rod

pytestmark = pytest.mark.gpu


def _spec(masked):
    spec = tip_mass_rod()
    if masked:
        mid = np.array([spec.n_nodes // 2], np.int32)
        spec.bcs += [BC(DL_BC_DIRICHLET, 3, mid, 0.0), BC(DL_BC_MASS, 4, mid, 1e-4),
                     BC(DL_BC_MASS, 5, mid, 2e-4), BC(DL_BC_MASS, 1, mid, 0.2)]
    return spec


@pytest.mark.parametrize("masked", [False, True])
@pytest.mark.parametrize("precision,tol", [(DL_PLAIN_FP64, 1e-9), (DL_MIXED, 1e-5)])
def test_added_mass_matches_oracle(gpu, masked, precision, tol):
    spec = _spec(masked)
    o = Oracle(spec)
    g = Lattice(spec, precision)
    o.run(2000)
    g.run(2000)
    g.synchronize()
    uo, to, vo = o.state()
    ug, tg, vg = g.state()
    assert rel_err(ug, uo) < tol
    assert rel_err(tg, to) < tol
    assert rel_err(vg, vo) < tol * 10
    assert g.energies()["kinetic"] == pytest.approx(o.energies()["kinetic"], rel=tol * 10)
    assert g.error_word() == 0


def test_milne_refuses_added_mass(gpu):
    g = Lattice(_spec(False), DL_PLAIN_FP64)
    with pytest.raises(DLError, match="added masses"):
        g.set_integrator(Integrator.milne(1e-6))
