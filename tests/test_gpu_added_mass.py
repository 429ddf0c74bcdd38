"""GPU added point masses (MassModel) against the oracle: a cantilever with
masses on the tip's six DOFs, and a node whose rotation is partly prescribed
(the masked solve) with added masses, over 2000 steps of a ramped tip load.

Plain FP64 only: the added masses enter the node update, which is FP64 in
both precisions.  Positions and rotations agree to 1e-9.  Velocities are held
to 1e-6 of their largest value: the loads are about 1e-11 of the rod's axial
stiffness, and the round-off of the unloaded rod's internal force (exactly
zero in the oracle's axis-aligned matrix arithmetic, about 1e-15 relative in
the engine's quaternion path) drives an out-of-plane angular velocity near
1e-8 of the in-plane one, with or without added masses."""
import numpy as np
import pytest

from dynlattice_b200.abi import BC, DL_BC_DIRICHLET, DL_BC_MASS, DL_PLAIN_FP64, Integrator
from dynlattice_b200.engine import DLError, Lattice
from helpers import rel_err
from oracle_ffi import Oracle
from test_added_mass import tip_mass_rod

pytestmark = pytest.mark.gpu


def _spec(masked, with_mass=True):
    spec = tip_mass_rod()
    if masked:
        mid = np.array([spec.n_nodes // 2], np.int32)
        spec.bcs += [BC(DL_BC_DIRICHLET, 3, mid, 0.0), BC(DL_BC_MASS, 4, mid, 1e-4),
                     BC(DL_BC_MASS, 5, mid, 2e-4), BC(DL_BC_MASS, 1, mid, 0.2)]
    if not with_mass:
        spec.bcs = [b for b in spec.bcs if b.kind != DL_BC_MASS]
    return spec


@pytest.mark.parametrize("spin", [False, True])
@pytest.mark.parametrize("masked", [False, True])
def test_added_mass_matches_oracle(gpu, masked, spin):
    """spin: the tip starts spinning about an oblique axis, so the
    gyroscopic moment with the added rotational masses is exercised."""
    spec = _spec(masked)
    o = Oracle(spec)
    g = Lattice(spec, DL_PLAIN_FP64)
    if spin:
        v0 = np.zeros((spec.n_nodes, 6))
        v0[spec.tip, 3:] = (0.0, 50.0, 30.0)
        o.set_state(v=v0)
        g.set_state(v=v0)
    o.run(2000)
    g.run(2000)
    g.synchronize()
    uo, to, vo = o.state()
    ug, tg, vg = g.state()
    assert rel_err(ug, uo) < 1e-9
    assert rel_err(tg, to) < 1e-9
    assert rel_err(vg, vo) < 1e-6
    assert g.energies()["kinetic"] == pytest.approx(o.energies()["kinetic"], rel=1e-8)
    assert g.error_word() == 0
    # the added masses change the motion far beyond these bounds
    h = Lattice(_spec(masked, with_mass=False), DL_PLAIN_FP64)
    if spin:
        h.set_state(v=v0)
    h.run(2000)
    assert rel_err(h.state()[2], vo) > 1e-2


def test_milne_refuses_added_mass(gpu):
    g = Lattice(_spec(False), DL_PLAIN_FP64)
    with pytest.raises(DLError, match="added masses"):
        g.set_integrator(Integrator.milne(1e-6))
