"""Element tables (GET_TABLE strain/stress/mat_strain/mat_stress/plast_strain,
as ParaViewModule writes them) in the oracle, on the CPU: closed forms for a
uniformly stretched straight rod, the frames (material axis e3 along the rod,
spatial along x), the Gauss-point sum scaled by the point count, and the
linear relation mat_stress = C (mat_strain - plast_strain) per element."""
import numpy as np
import pytest

from dynlattice_b200 import lattices
from oracle_ffi import Oracle


@pytest.mark.parametrize("n_gauss", [1, 2])
def test_stretched_rod_closed_form(n_gauss):
    spec = lattices.straight_rod(n_elems=4, n_gauss=n_gauss)
    s = 1e-3
    u = np.zeros((spec.n_nodes, 3))
    u[:, 0] = s * spec.coords[:, 0]
    o = Oracle(spec)
    o.set_state(u=u)
    G = n_gauss
    m = spec.materials[0]
    EA = m.young * m.area
    want_mat = np.zeros(6)
    want_mat[2] = s * G * G          # sum over G points, times G
    want_sp = np.zeros(6)
    want_sp[0] = s * G * G
    assert np.allclose(o.element_table("mat_strain"), want_mat, rtol=1e-9, atol=1e-15)
    assert np.allclose(o.element_table("strain"), want_sp, rtol=1e-9, atol=1e-15)
    assert np.allclose(o.element_table("mat_stress"), EA * want_mat, rtol=1e-9, atol=1e-6)
    assert np.allclose(o.element_table("stress"), EA * want_sp, rtol=1e-9, atol=1e-6)
    assert not o.element_table("plast_strain").any()
    with pytest.raises(RuntimeError, match="unknown element table"):
        o.element_table("hard_params")


def test_plastic_lattice_tables_are_consistent():
    """2^3 BCC elastoplastic impact after 1500 steps: plastic strain present
    and, per element, mat_stress = C (mat_strain - plast_strain)."""
    spec = lattices.lattice_impact(n=2)
    o = Oracle(spec, threads=4)
    o.run(1500)
    ms, me, mp = o.element_table("mat_stress"), o.element_table("mat_strain"), o.element_table("plast_strain")
    assert np.abs(mp).max() > 0.0, "the lattice must yield"
    m = spec.materials[0]
    r = spec.elem_radius
    A, I = np.pi * r ** 2, np.pi * r ** 4 / 4
    Gs = m.shear_modulus
    C = np.stack([Gs * 0.9 * A, Gs * 0.9 * A, m.young * A, m.young * I, m.young * I, Gs * 2 * I], axis=1)
    assert np.allclose(ms, C * (me - mp), rtol=1e-9, atol=1e-9 * np.abs(ms).max())
