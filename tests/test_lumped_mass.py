"""The explicit module's LUMPED mass mode in the oracle (ExplicitModule.cpp:
154-172, 339-357, 445-453): the model's MATRIX2 assembled into a diagonal
matrix, a = M^-1 r per DOF, and no gyroscopic moment (the rod model adds it
only when given the consistent matrix, SpecialCosseratRodModel.cpp:351-355)."""
import copy

import numpy as np

from dynlattice_b200 import lattices
from oracle_ffi import Oracle


def _spinning_rod(lumped):
    spec = lattices.straight_rod(n_elems=8, tip_force=0.0)
    spec.bcs = []
    spec.lumped_mass = lumped
    return spec


def test_lumped_mass_is_the_diagonal_of_the_node_block():
    spec = _spinning_rod(False)
    rng = np.random.default_rng(0)
    th = rng.normal(scale=0.4, size=(spec.n_nodes, 3))
    mt_c, mr_c = Oracle(spec).mass(th)
    mt_l, mr_l = Oracle(_spinning_rod(True)).mass(th)
    assert np.array_equal(mt_c, mt_l)
    for n in range(spec.n_nodes):
        assert np.allclose(np.diag(mr_l[n]), np.diag(mr_c[n]), rtol=1e-15, atol=0)
        assert np.count_nonzero(mr_l[n] - np.diag(np.diag(mr_l[n]))) == 0
        assert np.abs(mr_c[n] - np.diag(np.diag(mr_c[n]))).max() > 0  # the rotated block is full


def test_lumped_step_has_no_gyroscopic_moment():
    """One step of a rigidly spinning rod about an axis that is not principal:
    with the lumped matrix the angular acceleration is (f_ext - f_int)/diag(M)
    only (here f_int = 0: rigid motion), so omega does not change; the
    consistent mode turns omega by the gyroscopic moment."""
    w0 = np.array([3.0, 1.0, 0.5])
    out = {}
    for lumped in (False, True):
        spec = _spinning_rod(lumped)
        o = Oracle(spec)
        v = np.zeros((spec.n_nodes, 6))
        v[:, 3:] = w0
        # rigid rotation about the origin: v = w x x
        v[:, :3] = np.cross(w0, spec.coords)
        o.set_state(v=v)
        o.run(1)
        _, _, v1 = o.state()
        out[lumped] = v1
    dw_l = np.abs(out[True][:, 3:] - w0).max()
    dw_c = np.abs(out[False][:, 3:] - w0).max()
    assert dw_l < 1e-9 * np.abs(w0).max() < dw_c


def test_lumped_energy_from_diagonal():
    spec = _spinning_rod(True)
    o = Oracle(spec)
    rng = np.random.default_rng(1)
    v = rng.normal(size=(spec.n_nodes, 6)) * 1e-3
    o.set_state(v=v)
    o.run(1)
    _, th, v1 = o.state()
    # E_kin of the step: 1/2 v^T M v with M of the step's start (identity rotations)
    mt, mr = Oracle(spec).mass(np.zeros((spec.n_nodes, 3)))
    ek = 0.5 * (mt * (v1[:, :3] ** 2).sum(1)).sum() + 0.5 * sum(
        v1[n, 3:] @ mr[n] @ v1[n, 3:] for n in range(spec.n_nodes))
    assert abs(o.energies()["kinetic"] - ek) <= 1e-12 * ek
