"""The reference's quasi-static benchmarks as oracle models (test
infrastructure): the inputs of dynLattice tests/plastic/test1.pro, test2a.pro,
test2b.pro, test3.pro and tests/contact/test1.pro (copies under
tests/golden/pro/plastic and tests/golden/pro/contact), restated as model
descriptions with their load-step schedules, plus the comparison metrics of
tests/metrics.py.

Meshes follow the .geo files with gmsh's 1D rule (segments =
floor(L / lc + 0.99), equidistant nodes), linear elements with the reference's
default one-point Gauss rule for 2-node lines (Line3D.cpp:72-73), and the node
groups of tests/plastic/input.pro and tests/contact/input.pro.
"""
from __future__ import annotations

import math
from pathlib import Path

import numpy as np

from dynlattice_b200.abi import Contact, Material, ModelSpec
from static_driver import Prescribed, increment, loadscale

GOLDEN = Path(__file__).resolve().parent / "golden"


def literature():
    return dict(np.load(GOLDEN / "static_literature.npz"))


def _line(p0, p1, lc):
    p0, p1 = np.asarray(p0, float), np.asarray(p1, float)
    n = max(1, int(math.floor(np.linalg.norm(p1 - p0) / lc + 0.99)))
    t = np.linspace(0.0, 1.0, n + 1)[:, None]
    return p0 + t * (p1 - p0), n


def _rod_y(length, lc):
    x, n = _line((0, 0, 0), (0, length, 0), lc)
    conn = np.stack([np.arange(n), np.arange(1, n + 1)], 1)
    return x, conn, n


# ---------------------------------------------------------------------------
# tests/plastic/test1, test2a, test2b: one rod along y (0..1, lc 0.2), E = 1e6,
# nu = 0.4, circle r = 0.05, shear factor (6*1.4)/(7+9*0.4),
# isotropicCoefficient 1, kinematicTensor = I6 (test1.pro:19-31,
# test2a.pro:19-26, test2b.pro:19-26)
# ---------------------------------------------------------------------------

def _ramp(i, a, b, rate):
    """if(i>a, rate*(i-a), 0) - if(i>b, rate*(i-b), 0)"""
    return (rate * (i - a) if i > a else 0.0) - (rate * (i - b) if i > b else 0.0)


def stretch_test1(i):
    """scaleFunc of test1.pro:42-46."""
    return (_ramp(i, 1, 101, 0.031) + _ramp(i, 101, 201, -0.059) + _ramp(i, 201, 301, 0.071)
            + _ramp(i, 301, 401, -0.084) + _ramp(i, 401, 501, 0.056))


def stretch_test2(i):
    """scaleFunc of test2a.pro / test2b.pro:34-40."""
    return (_ramp(i, 1, 101, 0.031) + _ramp(i, 101, 201, -0.059) + _ramp(i, 201, 301, 0.071)
            + _ramp(i, 301, 401, -0.084) + _ramp(i, 401, 501, 0.098) + _ramp(i, 501, 601, -0.114)
            + _ramp(i, 601, 701, 0.093))


YIELD_TEST1 = ("abs(dx) + abs(dy) + abs(dz+0*h_dz) + abs(rx/0.12) + abs(ry/0.12) + abs(rz/0.12) "
               "- 10 * (1+0*h_0)")
YIELD_TEST2A = "abs(dz+0*h_dz) - 10 * (1+1*h_0)"
YIELD_TEST2B = "abs(dz+20*h_dz) - 10 * (1+0*h_0)"


def smriti_rod(yield_cond: str, twist: float, stretch, steps: int):
    """Model, prescribed DOFs and step count of plastic test 1/2a/2b.

    Groups (input.pro): fixed_left = fixed_right = the node at y = 0, free =
    the node at y = 1.  Constraints (model.pro diriFixed, test*.pro:56-62):
    translations of y = 0 fixed, its rotations fixed (fixed_right);
    free: dx, dz, rx, rz = 0; ry = twist (Dirichlet initDisp, dispIncr 0);
    dy = 1e-3 * scaleFunc(i) (LoadScale of a Dirichlet).  The rod stays
    straight under axial stretch and twist, so the transverse displacements
    and bending rotations of the inner nodes are zero by symmetry and are
    held there (the Newton iterates of the reference keep them at zero too)."""
    mat = Material.circle_section(0.05, young=1e6, poisson_ratio=0.4, density=1.0,
                                  shear_correction=(6 * 1.4) / (7 + 9 * 0.4), yield_cond=yield_cond,
                                  isotropic_coefficient=1.0, kinematic_tensor=list(np.eye(6).ravel()),
                                  max_iter=20, precision=1e-5)
    coords, conn, n = _rod_y(1.0, 0.2)
    spec = ModelSpec(coords=coords, conn=conn, elem_rod=np.zeros(n, np.int32), materials=[mat], n_gauss=1,
                     dt=1.0)
    zero = lambda i: 0.0
    pres = [Prescribed([0], d, zero) for d in range(6)]
    pres += [Prescribed([n], d, zero) for d in (0, 2, 3, 5)]
    pres += [Prescribed([n], 4, increment(1.0, 0.0, twist)), Prescribed([n], 1, loadscale(1e-3, stretch))]
    pres += [Prescribed(list(range(1, n)), d, zero) for d in (0, 2, 3, 5)]
    return spec, pres, steps, n


def plastic_test1():
    return smriti_rod(YIELD_TEST1, 0.18, stretch_test1, 500)    # runWhile i<501


def plastic_test2a():
    return smriti_rod(YIELD_TEST2A, 0.0, stretch_test2, 700)    # runWhile i<701


def plastic_test2b():
    return smriti_rod(YIELD_TEST2B, 0.0, stretch_test2, 700)


# ---------------------------------------------------------------------------
# tests/plastic/test3: rod along y (0..0.1, lc 3e-3), G = 80.193 GPa,
# E = 9 K G / (3 K + G) with K = 164.21 GPa, circle r = 1e-3, the
# Herrnboeck et al. yield surface with its yieldDeriv and a full kinematic
# tensor (test3.pro:19-48)
# ---------------------------------------------------------------------------

_T3 = [("dx", "700", "2.04"), ("dy", "700", "2.04"), ("dz", "1470", "1.76"),
       ("rx", "0.62", "2.09"), ("ry", "0.62", "2.09"), ("rz", "0.56", "1.73")]
KIN_TEST3 = [19014e+0, 17547e+0, 33121e+0, 16069e-3, 16743e-3, 15552e-3,
             17547e+0, 19014e+0, 33121e+0, 16743e-3, 16069e-3, 15556e-3,
             33121e+0, 33121e+0, 56864e+0, 24578e-3, 24578e-3, 26757e-3,
             16069e-3, 16743e-3, 24578e-3, 15015e-6, 15009e-6, 12715e-6,
             16743e-3, 16069e-3, 24578e-3, 15009e-6, 16015e-6, 12715e-6,
             15552e-3, 15556e-3, 26757e-3, 12715e-6, 12715e-6, 10434e-6]


def plastic_test3():
    """Model, prescribed DOFs and load factors of plastic test 3: y = 0 node
    translations fixed, rx = rz = 0, ry = pi/2 * lambda (fixed_right);
    y = 0.1 node dz = rx = ry = rz = 0, dx = 0.04 * lambda (free); lambda =
    (i - 1) * 0.01 (Dirichlet dispIncr 0.01) while lambda <= 1."""
    yc = " + ".join(f"abs({v}/({c}-h_{v}))^{p}" for v, c, p in _T3) + " - 1"

    def sgn(a):
        return f"if({a}>0, 1, if({a}<0, -1, 0))"

    yd = [f"{p} * abs({v}/({c}-h_{v}))^{float(p) - 1:g} * {sgn(f'{v}/({c}-h_{v})')} / ({c}-h_{v})"
          for v, c, p in _T3]
    yd += [f"{p} * abs({v}/({c}-h_{v}))^{float(p) - 1:g} * {sgn(f'{v}/({c}-h_{v})')} * {v}/(({c}-h_{v})^2)"
           for v, c, p in _T3]
    G = 80.193e9
    E = 9 * 164.210e9 * G / (3 * 164.210e9 + G)
    mat = Material.circle_section(1e-3, young=E, shear_modulus=G, density=1.0, yield_cond=yc, yield_deriv=yd,
                                  kinematic_tensor=KIN_TEST3, max_iter=20, precision=1e-5)
    coords, conn, n = _rod_y(100e-3, 3e-3)
    spec = ModelSpec(coords=coords, conn=conn, elem_rod=np.zeros(n, np.int32), materials=[mat], n_gauss=1,
                     dt=1.0)
    zero = lambda i: 0.0
    pres = [Prescribed([0], d, zero) for d in (0, 1, 2, 3, 5)] + [Prescribed([0], 4, increment(math.pi / 2, 0.01))]
    pres += [Prescribed([n], d, zero) for d in (2, 3, 4, 5)] + [Prescribed([n], 0, increment(0.04, 0.01))]
    factors = [(i - 1) * 0.01 for i in range(1, 102) if (i - 1) * 0.01 <= 1 + 1e-12]
    return spec, pres, factors, n


# ---------------------------------------------------------------------------
# tests/contact/test1: two crossed rods (test1.geo: (4,0,1)-(4,10,1) and
# (0,5,0)-(14,5,0), lc 0.5), E = 1e8, nu = 0, A = 4e-2, I = 2e-4, shear
# factor 1; RodContact penaltySTS = penaltyNTS = 1e4, radius 0.2
# (test1.pro:17-45, model.pro)
# ---------------------------------------------------------------------------

def contact_test1():
    """Model, prescribed DOFs, step count and the moving node: rod 1 clamped
    at both ends (fixed_left: y min, fixed_right: y max), rod 2's end at
    x max (moving_right) moved by (0.1, 0, 1) * 0.3 (i - 1) with its
    rotations held (Dirichlet dispIncr 0.3), its other end free;
    control.runWhile "i<=6" makes seven load steps."""
    x1, n1 = _line((4, 0, 1), (4, 10, 1), 0.5)
    x2, n2 = _line((0, 5, 0), (14, 5, 0), 0.5)
    coords = np.vstack([x1, x2])
    conn = np.vstack([np.stack([np.arange(n1), np.arange(1, n1 + 1)], 1),
                      n1 + 1 + np.stack([np.arange(n2), np.arange(1, n2 + 1)], 1)])
    rod = np.r_[np.zeros(n1, np.int32), np.ones(n2, np.int32)]
    mat = Material(young=1e8, shear_modulus=1e8 / 2.0, area=4e-2, area_moment=(2e-4, 2e-4), polar_moment=4e-4,
                   density=1.0, shear_correction=1.0)
    spec = ModelSpec(coords=coords, conn=conn, elem_rod=rod, materials=[mat], n_gauss=1, dt=1.0,
                     contact=Contact(radius=0.2, penalty=1e4, penalty_nts=1e4))
    fixed_left, fixed_right, moving_right = 0, n1, n1 + 1 + n2
    zero = lambda i: 0.0
    pres = [Prescribed([fixed_left], d, zero) for d in range(6)]
    pres += [Prescribed([fixed_right], d, zero) for d in range(6)]
    fac = (0.1, 0.0, 1.0, 0.0, 0.0, 0.0)
    pres += [Prescribed([moving_right], d, increment(fac[d], 0.3)) for d in range(6)]
    # element pairs of the two rods within reach of each other: coupled in the
    # column-compressed tangent
    ea, eb = np.arange(n1), n1 + np.arange(n2)
    mid = lambda e: coords[conn[e]].mean(axis=1)
    dist = np.linalg.norm(mid(ea)[:, None, :] - mid(eb)[None, :, :], axis=2)
    pa, pb = np.nonzero(dist < 3.0)
    coupling = np.concatenate([conn[ea[pa]], conn[eb[pb]]], axis=1)
    return spec, pres, 7, moving_right, coupling


# ---------------------------------------------------------------------------
# comparison metrics (tests/metrics.py:30-60)
# ---------------------------------------------------------------------------

def envelope_error(sim, ref):
    """Worst relative error of the maximum and of the minimum of two signals."""
    peak = abs(np.max(sim) - np.max(ref)) / max(abs(np.max(ref)), 1e-12)
    valley = abs(np.min(sim) - np.min(ref)) / max(abs(np.min(ref)), 1e-12)
    return float(max(peak, valley))


def curve_distance_2d(sim_xy, ref_xy):
    """Mean distance of each reference point to its nearest simulation point,
    over the diagonal of the reference's bounding box."""
    delta = sim_xy[:, None, :] - ref_xy[None, :, :]
    dist = np.sqrt((delta * delta).sum(axis=2))
    bbox = ref_xy.max(axis=0) - ref_xy.min(axis=0)
    return float(dist.min(axis=0).mean() / max(np.linalg.norm(bbox), 1e-12))
