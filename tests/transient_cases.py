"""The reference's transient benchmark models (tests/transient of dynLattice),
restated as plain-array model descriptions, and the comparison metrics its
test scripts apply against digitised literature curves (tolerance 5 %)."""
from __future__ import annotations

import math
from pathlib import Path

import numpy as np

from dynlattice_b200.abi import BC, DL_BC_DIRICHLET, DL_BC_NEUMANN, Material, ModelSpec

GOLDEN = Path(__file__).resolve().parent / "golden" / "transient_literature.npz"


def literature():
    return np.load(GOLDEN)


def _line_mesh(p0, p1, n_elems, order):
    """Straight line split into n_elems elements of `order` (1: 2 nodes, 2: 3
    nodes, natural order along the line as GMSHInputModule stores them)."""
    p0, p1 = np.asarray(p0, float), np.asarray(p1, float)
    n_nodes = n_elems * order + 1
    s = np.linspace(0.0, 1.0, n_nodes)
    coords = p0[None, :] + s[:, None] * (p1 - p0)[None, :]
    conn = np.array([[e * order + a for a in range(order + 1)] for e in range(n_elems)], np.int32)
    return coords, conn


def spin_up_beam(dt=5e-5, n_elems=4, order=2):
    """test1.pro: Simo & Vu-Quoc 1988 example 5.1.  10 m beam along x (4
    quadratic elements: lc 2.5), square section side sqrt(12/2e3), E = 5.6e10/12,
    G = 2e9, rho = 200; node at x = 0 clamped except rz, whose angular
    acceleration follows LoadScale "if (t<15, 6/15 * (1 - cos(2*PI/15 * t)), 0)".
    order=1 gives the same beam with two-node elements (the GPU engine's)."""
    coords, conn = _line_mesh((0, 0, 0), (10, 0, 0), n_elems, order)
    s = math.sqrt(12 / 2e3)
    A, I = s * s, s ** 4 / 12.0
    mat = Material(young=5.6e10 / 12, shear_modulus=2e9, area=A, area_moment=(I, I), polar_moment=2 * I,
                   density=200.0, shear_correction=5.0 / 6.0)
    fixed = np.array([0], np.int32)
    free = np.array([coords.shape[0] - 1], np.int32)
    bcs = [BC(DL_BC_DIRICHLET, d, fixed, 0.0) for d in range(6)]
    bcs.append(BC(DL_BC_DIRICHLET, 5, fixed, 1.0, "if (t<15, 6/15 * (1 - cos(2*PI/15 * t)), 0)"))
    # Line3D's default scheme for 3 nodes is Gauss2 (reduced integration)
    return ModelSpec(coords=coords, conn=conn, elem_rod=np.zeros(conn.shape[0], np.int32), materials=[mat],
                     n_gauss=2, dt=dt, bcs=bcs, groups={"fixed": fixed, "free": free}, name="spin_up_beam")


def swinging_rod(dt=1e-6):
    """test2.pro: Lang et al. 2011 example 1.  1 m rod along x (10 linear
    elements: lc 0.1), circular r = 5 mm, E = 5e6, nu = 0.4999999, shear
    correction 1, rho = 1100, translations of x = 0 fixed, gravity as nodal
    loads (one element's weight per node, half at the ends)."""
    coords, conn = _line_mesh((0, 0, 0), (1, 0, 0), 10, 1)
    mat = Material.circle_section(5e-3, young=5e6, poisson_ratio=0.4999999, density=1.1e3,
                                  shear_correction=1.0)
    n = coords.shape[0]
    fixed = np.array([0], np.int32)
    free = np.array([n - 1], np.int32)
    allg = np.arange(n, dtype=np.int32)
    w = math.pi * (5e-3) ** 2 * 0.1 * 1.1e3 * 9.81
    bcs = [BC(DL_BC_DIRICHLET, d, fixed, 0.0) for d in range(3)]
    bcs += [BC(DL_BC_NEUMANN, 2, allg, -w), BC(DL_BC_NEUMANN, 2, free, 0.5 * w), BC(DL_BC_NEUMANN, 2, fixed, 0.5 * w)]
    return ModelSpec(coords=coords, conn=conn, elem_rod=np.zeros(conn.shape[0], np.int32), materials=[mat],
                     n_gauss=1, dt=dt, bcs=bcs, groups={"fixed": fixed, "free": free}, name="swinging_rod")


# --- metrics of the reference's test scripts (tests/metrics.py), restated ---

def interp_on_reference(x_sim, y_sim, x_ref):
    order = np.argsort(x_sim)
    return np.interp(x_ref, np.asarray(x_sim)[order], np.asarray(y_sim)[order])


def relative_l2(y_sim, y_ref):
    den = np.linalg.norm(y_ref)
    if den < 1e-12:
        den = max(np.abs(y_ref).max(), 1e-12)
    return float(np.linalg.norm(np.asarray(y_sim) - y_ref) / den)


def curve_distance_2d(sim_xy, ref_xy):
    """Mean distance from each reference point to the nearest simulated point,
    over the diagonal of the reference bounding box."""
    dist = np.sqrt(((sim_xy[:, None, :] - ref_xy[None, :, :]) ** 2).sum(axis=2))
    bbox = ref_xy.max(axis=0) - ref_xy.min(axis=0)
    return float(dist.min(axis=0).mean() / max(np.linalg.norm(bbox), 1e-12))


def spin_up_errors(t, psi, free_u, free_rz, lit):
    """test1.py's four relative-L2 errors: the prescribed angle psi, and the
    free end's rotation lag and axial / radial deviation in the rotating frame."""
    psi = np.unwrap(psi)
    rz = np.unwrap(free_rz)
    px, py = 10.0 + free_u[:, 0], free_u[:, 1]
    dvec = np.stack([px - 10 * np.cos(psi), py - 10 * np.sin(psi)], -1)
    outv = np.stack([np.cos(psi), np.sin(psi)], -1)
    tanv = np.stack([-np.sin(psi), np.cos(psi)], -1)
    dev_rz = np.rad2deg(psi - rz)
    dev_u1 = (dvec * outv).sum(1)
    dev_u2 = (dvec * tanv).sum(1)
    bc, ang, u1, u2 = lit["test1_bc"], lit["test1_angle"], lit["test1_u1"], lit["test1_u2"]
    return {
        "psi": relative_l2(interp_on_reference(t, psi, bc[:, 0]), bc[:, 1]),
        "rz": relative_l2(interp_on_reference(t, dev_rz, ang[:, 0]), ang[:, 1]),
        "u1": relative_l2(interp_on_reference(t, dev_u1, u1[:, 0]), u1[:, 1]),
        "u2": relative_l2(interp_on_reference(t, dev_u2, u2[:, 0]), u2[:, 1]),
    }


def swinging_errors(times, shapes, lit):
    """test2.py: rod shape (x, z) at t = 0.0, 0.1, ..., 1.0 against Lang et al."""
    out = {}
    for t, xz in zip(times, shapes):
        out[round(float(t), 1)] = curve_distance_2d(xz, lit[f"test2_t{t:.1f}"])
    return out


# MilneDevice tolerance of the transient .pro files that set none (the
# engine's default for the reference's jive::solver::Solver::PRECISION)
MILNE_PRECISION = 1e-6
