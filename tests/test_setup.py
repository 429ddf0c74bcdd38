"""Host-side set-up of the engine (frames, reference strains, lumped masses)
against the oracle's restatement of initRotation_/initStrain_/assembleM_."""
import ctypes as C

import numpy as np
import pytest

from dynlattice_b200 import lattices
from dynlattice_b200.abi import DL_MIXED, DL_PLAIN_FP64, dl_model_desc
from dynlattice_b200.engine import load_library
from oracle_ffi import Oracle
import transient_cases as tc


def quat2mat(q):
    w, x, y, z = q
    return np.array([[w*w+x*x-y*y-z*z, 2*(x*y-w*z), 2*(x*z+w*y)],
                     [2*(x*y+w*z), w*w-x*x+y*y-z*z, 2*(y*z-w*x)],
                     [2*(x*z-w*y), 2*(y*z+w*x), w*w-x*x-y*y+z*z]])


def inspect(spec, precision=DL_PLAIN_FP64):
    lib = load_library()
    dp = C.POINTER(C.c_double)
    lib.dl_inspect_setup.argtypes = [C.POINTER(dl_model_desc), C.c_int, dp, dp, dp, dp]
    E, N, G, nen = spec.n_elems, spec.n_nodes, spec.n_gauss, spec.conn.shape[1]
    fr = np.zeros((E, nen, 4)); st = np.zeros((E, G, 6)); m = np.zeros(N); ri = np.zeros((N, 3, 3))
    d = spec.desc()
    p = lambda a: a.ctypes.data_as(dp)
    assert lib.dl_inspect_setup(C.byref(d), precision, p(fr), p(st), p(m), p(ri)) == 0, lib.dl_last_error()
    return fr, st, m, ri


@pytest.mark.parametrize("make", [
    lambda: lattices.straight_rod(),
    lambda: lattices.lattice_impact("bcc", n=2),
    lambda: lattices.lattice_impact("sc", n=2),
    lambda: lattices.lattice_impact("octet", n=1),
    lambda: lattices.helix_rod(nodes_per_elem=2),
    lambda: lattices.helix_rod(nodes_per_elem=3),
    lambda: lattices.helix_rod(nodes_per_elem=4),
    lambda: tc.spin_up_beam(order=2),
])
def test_setup_matches_oracle(make):
    """Frames, reference strains and node masses; the helices (curvature and
    torsion in the reference state, 2/3/4-node elements) take the reference
    curvature through Line3D's interpolated rotation and its derivative."""
    spec = make()
    fr, st, m, ri = inspect(spec)
    o = Oracle(spec)
    LN, s0 = o.frames()
    mt, mr = o.mass()
    nen = spec.conn.shape[1]
    Rm = np.array([[quat2mat(fr[e, a]) for a in range(nen)] for e in range(spec.n_elems)])
    assert np.abs(Rm - LN).max() < 1e-13
    assert np.abs(st - s0).max() < 1e-11 * max(1.0, np.abs(s0).max())
    assert np.abs(m - mt).max() < 1e-13 * mt.max()
    assert np.abs(ri - mr).max() < 1e-12 * np.abs(mr).max()


def test_mixed_frames_are_rounded_but_consistent():
    """Mixed precision rounds the end frames to FP32 and forms the reference
    strains from the rounded frames, so an undeformed rod stays strain free."""
    spec = lattices.lattice_impact("bcc", n=2)
    fr64, st64, _, _ = inspect(spec, DL_PLAIN_FP64)
    fr32, st32, _, _ = inspect(spec, DL_MIXED)
    assert np.abs(fr32 - fr64).max() < 1e-7
    assert np.array_equal(fr32, fr32.astype(np.float32).astype(np.float64))
    assert np.abs(st32 - st64).max() < 1e-6


def test_bcc_lattice_counts():
    spec = lattices.lattice_impact("bcc", n=20)
    assert spec.n_elems == 128000
    assert spec.n_nodes == 21 ** 3 + 20 ** 3 + 64000
    assert spec.groups["top"].size == 21 * 21 and spec.groups["bottom"].size == 21 * 21
    r = spec.strut_radius
    assert r.min() >= 0.5e-3 * 0.95 and r.max() <= 0.5e-3 * 1.05


def test_nnode_contact_refused():
    """Contact runs on two-node elements (segments between the element end
    nodes); a model of 3-node elements with contact is refused at set-up."""
    from dynlattice_b200.abi import Contact
    spec = lattices.helix_rod(nodes_per_elem=3)
    spec.contact = Contact(radius=0.005, penalty=1e5)
    lib = load_library()
    dp = C.POINTER(C.c_double)
    lib.dl_inspect_setup.argtypes = [C.POINTER(dl_model_desc), C.c_int, dp, dp, dp, dp]
    d = spec.desc()
    assert lib.dl_inspect_setup(C.byref(d), DL_PLAIN_FP64, None, None, None, None) != 0
    assert b"two-node" in lib.dl_last_error()
