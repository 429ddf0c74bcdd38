"""Small rod--rod contact configurations shared by the CPU (oracle) and GPU
contact tests.  Each case is a set of straight rods; rod ids follow list
order, so the first rod is the reference's "A" side of every pair."""
from __future__ import annotations

import numpy as np

from dynlattice_b200.abi import BC, DL_BC_DIRICHLET, Contact, Material, ModelSpec

R = 0.1e-3          # contact radius
KPEN = 1e4          # penalty (STS and NTS)
LEN = 10e-3


def rods_spec(rods, elems=4, radius=R, penalty=KPEN, dt=1e-8, fixed_rods=(), plates=(), margin=None,
              n_gauss=1):
    """rods: list of (start[3], end[3]).  Rods in ``fixed_rods`` are clamped at both ends."""
    coords, conn, erod = [], [], []
    ends = []
    for r, (a, b) in enumerate(rods):
        a, b = np.asarray(a, float), np.asarray(b, float)
        n0 = len(coords)
        for i in range(elems + 1):
            coords.append(a + (b - a) * i / elems)
        for e in range(elems):
            conn.append((n0 + e, n0 + e + 1))
            erod.append(r)
        ends.append((n0, n0 + elems))
    coords = np.array(coords)
    conn = np.array(conn, np.int32)
    erod = np.array(erod, np.int32)
    mat = Material.circle_section(radius, young=3e9, poisson_ratio=0.35, density=1200.0)
    bcs = []
    fixed = np.array([n for r in fixed_rods for n in ends[r]], np.int32)
    if fixed.size:
        bcs = [BC(DL_BC_DIRICHLET, d, fixed, 0.0) for d in range(6)]
    contact = Contact(radius=radius, penalty=penalty, plates=list(plates),
                      margin=(2.0 * radius if margin is None else margin))
    spec = ModelSpec(coords=coords, conn=conn, elem_rod=erod, materials=[mat], n_gauss=n_gauss, dt=dt,
                     bcs=bcs, contact=contact, name="rods")
    spec.rod_nodes = [np.arange(e0, e1 + 1) for e0, e1 in ends]
    return spec


def shift_rod(spec, rod, delta):
    """Displacement field [N, 3] that translates one rod by delta."""
    u = np.zeros((spec.coords.shape[0], 3))
    u[spec.rod_nodes[rod]] = np.asarray(delta, float)
    return u


def cross(gap0=0.05e-3):
    """STS: rod 0 along x, rod 1 along y above it (crossing inside elements
    of both rods), surface gap gap0."""
    z = 2 * R + gap0
    return rods_spec([((-LEN / 2, 0, 0), (LEN / 2, 0, 0)),
                      ((0.3e-3, -LEN / 2 + 0.3e-3, z), (0.3e-3, LEN / 2 + 0.3e-3, z))])


def tee_b_end(gap0=0.05e-3):
    """One-sided NTS: the lower end of rod 1 (B, vertical) sits above the
    middle of rod 0 (A, along x)."""
    z = 2 * R + gap0
    return rods_spec([((-LEN / 2, 0, 0), (LEN / 2, 0, 0)), ((0.7e-3, 0, z), (0.7e-3, 0, z + LEN))])


def tee_a_end(gap0=0.05e-3):
    """Mirror of tee_b_end with the rod order swapped: the end of rod 0 (A)
    sits above the middle of rod 1 (B).  The reference's one-sided branch
    projects node iA of element B here (RodContactModel.cpp:575)."""
    z = 2 * R + gap0
    return rods_spec([((0.7e-3, 0, z), (0.7e-3, 0, z + LEN)), ((-LEN / 2, 0, 0), (LEN / 2, 0, 0))])


# dyadic coordinates keep the two parallel directions bitwise equal, so the
# line--line closest-point system is exactly singular (0/0) on every host
PLEN = 2.0 ** -7
POFF = 2.0 ** -10
PZ = 2.0 ** -12


def parallel():
    """Speculative NTS: two parallel rods along x, rod 1 shifted by POFF along
    x and PZ above rod 0 (surface gap PZ - 2R)."""
    return rods_spec([((0, 0, 0), (PLEN, 0, 0)), ((POFF, 0, PZ), (PLEN + POFF, 0, PZ))])
