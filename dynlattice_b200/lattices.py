"""Seeded synthetic workloads: a straight rod and strut lattices of rods.

Each strut of a lattice is one rod ("beam_k" element group in the reference's
GMSH input, src/modules/GMSHInputModule.cpp:336-394) split into
``elems_per_strut`` two-node elements; nodes are merged at shared lattice
points.  These generators produce the engine's plain-array model description
(:class:`dynlattice_b200.abi.ModelSpec`).
"""
from __future__ import annotations

import math
from typing import Optional, Tuple

import numpy as np

from .abi import (BC, DL_BC_DIRICHLET, DL_BC_INIT_VELO, DL_BC_NEUMANN, Contact, Material,
                  ModelSpec)

# ---------------------------------------------------------------------------
# materials
# ---------------------------------------------------------------------------

SIGMA_Y_AL = 300e6
HARDENING_AL = 1e9


def aluminium_elastoplastic(radius: float = 0.5e-3, sigma_y: float = SIGMA_Y_AL,
                            hardening: float = HARDENING_AL) -> Material:
    """Elastoplastic aluminium strut material (E=70 GPa, nu=0.33, rho=2700).

    Yield surface in stress-resultant space, written as a reference-style
    ``yieldCond`` expression with its ``yieldDeriv`` list.  Capacities use the
    element's own section through the ``area``/``radius`` element variables:
    N_p = sy A, V_p = sy/sqrt(3) A, M_p = sy 4 r^3/3, T_p = sy/sqrt(3) 2 pi r^3/3;
      s = sqrt((dx/Vp)^2 + (dy/Vp)^2 + (dz/Np)^2 + (rx/Mp)^2 + (ry/Mp)^2 + (rz/Tp)^2)
      f = s - 1 + h_0 / (sy sqrt(area))
    With isotropicCoefficient H = hardening, uniaxial loading gives
    sigma = sy + H eps_p (linear isotropic hardening modulus H).
    """
    sy = float(sigma_y)
    Np = f"({sy!r}*area)"
    Vp = f"({sy / math.sqrt(3.0)!r}*area)"
    Mp = f"({sy * 4.0 / 3.0!r}*radius^3)"
    Tp = f"({sy / math.sqrt(3.0) * 2.0 / 3.0 * math.pi!r}*radius^3)"
    s = (f"sqrt((dx/{Vp})^2 + (dy/{Vp})^2 + (dz/{Np})^2 + (rx/{Mp})^2 + (ry/{Mp})^2"
         f" + (rz/{Tp})^2)")
    f = f"{s} - 1 + h_0/({sy!r}*sqrt(area))"
    deriv = [f"dx/({Vp}^2)/{s}", f"dy/({Vp}^2)/{s}", f"dz/({Np}^2)/{s}",
             f"rx/({Mp}^2)/{s}", f"ry/({Mp}^2)/{s}", f"rz/({Tp}^2)/{s}",
             f"1/({sy!r}*sqrt(area))"]
    return Material.circle_section(radius, young=70e9, poisson_ratio=0.33, density=2700.0,
                                   yield_cond=f, yield_deriv=deriv,
                                   isotropic_coefficient=float(hardening), max_iter=20,
                                   precision=1e-5)


def aluminium_elastic(radius: float = 0.5e-3) -> Material:
    return Material.circle_section(radius, young=70e9, poisson_ratio=0.33, density=2700.0)


# ---------------------------------------------------------------------------
# straight rod (single clamped cantilever)
# ---------------------------------------------------------------------------

def straight_rod(n_elems: int = 32, length: float = 1.0, radius: float = 0.01,
                 young: float = 210e9, poisson: float = 0.3, density: float = 7850.0,
                 tip_force: float = 1.0, ramp_steps: int = 500, dt: float = 2e-6,
                 n_gauss: int = 2) -> ModelSpec:
    """Single straight elastic rod along x, clamped at x = 0, tip force along y
    ramped linearly over ``ramp_steps`` steps then held (LoadScale
    ``min(i/ramp, 1)`` on a Neumann load)."""
    x = np.linspace(0.0, length, n_elems + 1)
    coords = np.stack([x, np.zeros_like(x), np.zeros_like(x)], axis=1)
    conn = np.stack([np.arange(n_elems), np.arange(1, n_elems + 1)], axis=1)
    mat = Material.circle_section(radius, young=young, poisson_ratio=poisson, density=density)
    clamp = np.array([0], dtype=np.int32)
    tip = np.array([n_elems], dtype=np.int32)
    bcs = [BC(DL_BC_DIRICHLET, d, clamp, 0.0) for d in range(6)]
    bcs.append(BC(DL_BC_NEUMANN, 1, tip, tip_force, f"min(i/{ramp_steps}, 1)"))
    return ModelSpec(coords=coords, conn=conn, elem_rod=np.zeros(n_elems, np.int32),
                     materials=[mat], n_gauss=n_gauss, dt=dt, bcs=bcs,
                     groups={"fixed": clamp, "free": tip}, name="straight_rod")


def helix_rod(n_elems: int = 8, nodes_per_elem: int = 3, turns: float = 0.75, helix_radius: float = 0.1,
              pitch: float = 0.05, radius: float = 0.005, young: float = 70e9, poisson: float = 0.33,
              density: float = 2700.0, tip_force: float = 5.0, ramp_steps: int = 200, dt: float = 5e-7,
              n_gauss: int = 0, plastic: bool = False) -> ModelSpec:
    """One helical rod (curvature and torsion in the reference state) of
    ``n_elems`` elements with 2, 3 or 4 nodes each (Line2/Line3/Line4, nodes
    along the line), clamped at its first node; a tip force along -z ramped
    over ``ramp_steps`` steps.  ``n_gauss`` 0 takes Line3D's default
    Gauss(n-1) rule (Line3D.cpp:72-73); ``plastic`` takes the elastoplastic
    aluminium law (yielding under larger tip forces)."""
    nen = int(nodes_per_elem)
    n_nodes = n_elems * (nen - 1) + 1
    t = np.linspace(0.0, 2.0 * np.pi * turns, n_nodes)
    coords = np.stack([helix_radius * np.cos(t), helix_radius * np.sin(t), pitch * t / (2.0 * np.pi)], axis=1)
    conn = np.array([[e * (nen - 1) + a for a in range(nen)] for e in range(n_elems)], np.int32)
    mat = (aluminium_elastoplastic(radius) if plastic else
           Material.circle_section(radius, young=young, poisson_ratio=poisson, density=density))
    clamp = np.array([0], dtype=np.int32)
    tip = np.array([n_nodes - 1], dtype=np.int32)
    bcs = [BC(DL_BC_DIRICHLET, d, clamp, 0.0) for d in range(6)]
    bcs.append(BC(DL_BC_NEUMANN, 2, tip, -tip_force, f"min(i/{ramp_steps}, 1)"))
    return ModelSpec(coords=coords, conn=conn, elem_rod=np.zeros(n_elems, np.int32), materials=[mat],
                     n_gauss=n_gauss if n_gauss > 0 else nen - 1, dt=dt, bcs=bcs,
                     groups={"fixed": clamp, "free": tip}, name=f"helix_rod_{nen}")


# ---------------------------------------------------------------------------
# lattices
# ---------------------------------------------------------------------------

def _grid_points(n: int, cell: float) -> np.ndarray:
    g = np.arange(n + 1, dtype=np.float64) * cell
    X, Y, Z = np.meshgrid(g, g, g, indexing="ij")
    return np.stack([X.ravel(order="F"), Y.ravel(order="F"), Z.ravel(order="F")], axis=1)


def _corner_index(i, j, k, n):
    return i + (n + 1) * (j + (n + 1) * k)


def lattice_struts(topology: str, n: int, cell: float) -> Tuple[np.ndarray, np.ndarray]:
    """Lattice points and strut list for an n^3 block of unit cells.

    bcc: corners + cell centres, 8 corner-to-centre struts per cell;
    sc: corners, struts along the three axes between neighbouring corners;
    octet: corners + face centres (FCC points), struts between nearest
    neighbours at distance cell/sqrt(2).
    """
    corners = _grid_points(n, cell)
    idx = np.arange(n)
    I, J, K = np.meshgrid(idx, idx, idx, indexing="ij")
    I, J, K = I.ravel(order="F"), J.ravel(order="F"), K.ravel(order="F")
    if topology == "bcc":
        centres = np.stack([(I + 0.5) * cell, (J + 0.5) * cell, (K + 0.5) * cell], axis=1)
        ncorner = corners.shape[0]
        cidx = ncorner + np.arange(centres.shape[0])
        struts = []
        for di in (0, 1):
            for dj in (0, 1):
                for dk in (0, 1):
                    struts.append(np.stack([_corner_index(I + di, J + dj, K + dk, n), cidx], 1))
        # order struts cell by cell
        struts = np.stack(struts, axis=1).reshape(-1, 2)
        return np.concatenate([corners, centres]), struts.astype(np.int64)
    if topology == "sc":
        g = np.arange(n + 1)
        A, B, Cc = np.meshgrid(g, g, g, indexing="ij")
        A, B, Cc = A.ravel(order="F"), B.ravel(order="F"), Cc.ravel(order="F")
        s = []
        m = A < n
        s.append(np.stack([_corner_index(A[m], B[m], Cc[m], n), _corner_index(A[m] + 1, B[m], Cc[m], n)], 1))
        m = B < n
        s.append(np.stack([_corner_index(A[m], B[m], Cc[m], n), _corner_index(A[m], B[m] + 1, Cc[m], n)], 1))
        m = Cc < n
        s.append(np.stack([_corner_index(A[m], B[m], Cc[m], n), _corner_index(A[m], B[m], Cc[m] + 1, n)], 1))
        return corners, np.concatenate(s).astype(np.int64)
    if topology == "octet":
        # FCC points on a half-cell grid: integer coords (2i,2j,2k) with even sum
        h = 2 * n
        g = np.arange(h + 1)
        A, B, Cc = np.meshgrid(g, g, g, indexing="ij")
        A, B, Cc = A.ravel(order="F"), B.ravel(order="F"), Cc.ravel(order="F")
        keep = ((A + B + Cc) % 2) == 0
        pts = np.stack([A[keep], B[keep], Cc[keep]], 1)
        lut = -np.ones((h + 1,) * 3, dtype=np.int64)
        lut[pts[:, 0], pts[:, 1], pts[:, 2]] = np.arange(pts.shape[0])
        s = []
        for d in [(1, 1, 0), (1, -1, 0), (1, 0, 1), (1, 0, -1), (0, 1, 1), (0, 1, -1)]:
            q = pts + np.array(d)
            ok = np.all((q >= 0) & (q <= h), axis=1)
            a = np.nonzero(ok)[0]
            b = lut[q[ok, 0], q[ok, 1], q[ok, 2]]
            good = b >= 0
            s.append(np.stack([a[good], b[good]], 1))
        return pts.astype(np.float64) * (cell / 2.0), np.concatenate(s).astype(np.int64)
    raise ValueError(f"unknown topology {topology!r}")


def subdivide(points: np.ndarray, struts: np.ndarray, elems_per_strut: int):
    """Split each strut into elements with interior nodes appended after the
    lattice points.  Returns coords, conn [E,2], elem_rod [E]."""
    m = int(elems_per_strut)
    S = struts.shape[0]
    P = points.shape[0]
    a = points[struts[:, 0]]
    b = points[struts[:, 1]]
    if m > 1:
        t = np.arange(1, m, dtype=np.float64) / m
        inner = a[:, None, :] + (b - a)[:, None, :] * t[None, :, None]   # [S, m-1, 3]
        inner_idx = P + np.arange(S * (m - 1)).reshape(S, m - 1)
        coords = np.concatenate([points, inner.reshape(-1, 3)])
        chain = np.concatenate([struts[:, :1], inner_idx, struts[:, 1:]], axis=1)  # [S, m+1]
    else:
        coords = points.copy()
        chain = struts
    conn = np.stack([chain[:, :-1], chain[:, 1:]], axis=2).reshape(-1, 2)
    elem_rod = np.repeat(np.arange(S), m)
    return coords, conn.astype(np.int32), elem_rod.astype(np.int32)


def lattice_impact(topology: str = "bcc", n: int = 20, cell: float = 10e-3, elems_per_strut: int = 2,
                   radius: float = 0.5e-3, radius_jitter: float = 0.05, seed: int = 0,
                   velocity: float = 10.0, dt: float = 5e-8, plastic: bool = True,
                   n_gauss: int = 2, radius_range: Optional[Tuple[float, float]] = None) -> ModelSpec:
    """Strut-lattice impact: bottom face (min z) fixed in all six DOFs, top face
    (max z) moving down at ``velocity`` (InitLoad velocity + Dirichlet a_z = 0).

    Strut radii: radius * (1 + U[-jitter, jitter]) per strut from ``seed``, or
    U(radius_range) when given."""
    pts, struts = lattice_struts(topology, n, cell)
    coords, conn, elem_rod = subdivide(pts, struts, elems_per_strut)
    rng = np.random.default_rng(seed)
    S = struts.shape[0]
    if radius_range is not None:
        r_strut = rng.uniform(radius_range[0], radius_range[1], size=S)
    else:
        r_strut = radius * (1.0 + rng.uniform(-radius_jitter, radius_jitter, size=S))
    elem_radius = np.repeat(r_strut, elems_per_strut)
    mat = aluminium_elastoplastic(radius) if plastic else aluminium_elastic(radius)
    z = coords[:, 2]
    zmin, zmax = z.min(), z.max()
    tol = 1e-9 * max(1.0, abs(zmax))
    bottom = np.nonzero(np.abs(z - zmin) <= tol)[0].astype(np.int32)
    top = np.nonzero(np.abs(z - zmax) <= tol)[0].astype(np.int32)
    bcs = [BC(DL_BC_DIRICHLET, d, bottom, 0.0) for d in range(6)]
    bcs.append(BC(DL_BC_DIRICHLET, 2, top, 0.0))
    bcs.append(BC(DL_BC_INIT_VELO, 2, top, -float(velocity)))
    spec = ModelSpec(coords=coords, conn=conn, elem_rod=elem_rod, materials=[mat],
                     elem_radius=elem_radius, n_gauss=n_gauss, dt=dt, bcs=bcs,
                     groups={"bottom": bottom, "top": top},
                     name=f"{topology}{n}^3")
    spec.strut_radius = r_strut
    return spec


def critical_dt(spec: ModelSpec, safety: float = 0.5) -> float:
    """dt_k = safety * min_e(L_e / c) with c = sqrt(E / rho) (bar wave speed)."""
    m = spec.materials[0]
    c = math.sqrt(m.young / m.density)
    d = spec.coords[spec.conn[:, 1]] - spec.coords[spec.conn[:, 0]]
    L = np.sqrt((d * d).sum(1)).min()
    return safety * L / c


def batch_lattices(n_lattices: int = 256, seed: int = 0, n_range=(4, 12), cell: float = 10e-3,
                   elems_per_strut: int = 2, radius_range=(0.3e-3, 0.7e-3), velocity_range=(1.0, 50.0),
                   topologies=("bcc", "sc", "octet"), safety: float = 0.5):
    """Uneven batch of impact lattices: per lattice a topology drawn uniformly from
    ``topologies``, n^3 cells with n ~ U{n_range}, one strut radius ~ U(radius_range),
    impact velocity log-uniform in ``velocity_range`` and its own time step
    dt = safety * min_e(L_e / c) (c = sqrt(E/rho)).  Elastoplastic aluminium."""
    rng = np.random.default_rng(seed)
    specs = []
    for k in range(n_lattices):
        topo = topologies[int(rng.integers(len(topologies)))]
        n = int(rng.integers(n_range[0], n_range[1] + 1))
        r = float(rng.uniform(*radius_range))
        v = float(np.exp(rng.uniform(np.log(velocity_range[0]), np.log(velocity_range[1]))))
        spec = lattice_impact(topo, n=n, cell=cell, elems_per_strut=elems_per_strut, radius=r,
                              radius_jitter=0.0, seed=seed * 100003 + k, velocity=v, dt=1.0, plastic=True)
        # every strut of this lattice has radius r; one material per lattice
        spec.materials = [aluminium_elastoplastic(r)]
        spec.dt = critical_dt(spec, safety)
        spec.name = f"{topo}{n}^3#{k}"
        specs.append(spec)
    return specs


# ---------------------------------------------------------------------------
# random fibre network with rod--rod contact
# ---------------------------------------------------------------------------

def generate_fibres(n_rods: int, length: float = 10e-3, elems_per_rod: int = 4, radius: float = 0.1e-3,
                    box: float = 50e-3, seed: int = 0, max_tries: int = 0):
    """Random sequential addition of straight rods (``dl_generate_fibres``):
    returns (coords [N, 3], conn [E, 2], elem_rod [E], tries)."""
    import ctypes as C

    from .engine import DLError, load_library
    lib = load_library()
    f = lib.dl_generate_fibres
    f.argtypes = [C.c_int32, C.c_double, C.c_int32, C.c_double, C.c_double, C.c_uint64, C.c_int64,
                  C.POINTER(C.c_double), C.POINTER(C.c_int32), C.POINTER(C.c_int32), C.POINTER(C.c_int64)]
    E = n_rods * elems_per_rod
    coords = np.zeros((n_rods * (elems_per_rod + 1), 3))
    conn = np.zeros((E, 2), np.int32)
    elem_rod = np.zeros(E, np.int32)
    tries = C.c_int64()
    rc = f(n_rods, length, elems_per_rod, radius, box, seed, max_tries,
           coords.ctypes.data_as(C.POINTER(C.c_double)), conn.ctypes.data_as(C.POINTER(C.c_int32)),
           elem_rod.ctypes.data_as(C.POINTER(C.c_int32)), C.byref(tries))
    if rc != 0:
        raise DLError(rc, "dl_generate_fibres failed (bad argument or max_tries reached)")
    return coords, conn, elem_rod, tries.value


def fibre_network(n_rods: int = 20000, length: float = 10e-3, elems_per_rod: int = 4,
                  radius: float = 0.1e-3, box: Optional[float] = None, seed: int = 0,
                  plate_velocity: float = 5.0, penalty: float = 1e4, dt: float = 1e-8,
                  margin: Optional[float] = None) -> ModelSpec:
    """Random fibre network compressed between two rigid plates.

    Rods: elastic (E = 3 GPa, nu = 0.35, rho = 1200), circular radius
    ``radius``, centres uniform in a cube, directions uniform on the sphere,
    rods closer than 2r at t = 0 resampled.  ``box`` defaults to 50 mm for
    20 000 rods and scales with n_rods^(1/3) so that smaller networks keep the
    same rod density.  Rod--rod penalty contact with stiffness ``penalty``
    (N/m per unit overlap, both segment-to-segment and node-to-segment).
    Plates: the bottom one (normal +z) touches the lowest node and stays; the
    top one (normal -z) touches the highest node and moves down at
    ``plate_velocity``; node--plate penalty ``penalty`` with the rod radius."""
    if box is None:
        box = 50e-3 * (n_rods / 20000.0) ** (1.0 / 3.0)
    coords, conn, elem_rod, tries = generate_fibres(n_rods, length, elems_per_rod, radius, box, seed)
    mat = Material.circle_section(radius, young=3e9, poisson_ratio=0.35, density=1200.0)
    z = coords[:, 2]
    zmin, zmax = float(z.min()), float(z.max())
    plates = [
        {"normal": (0.0, 0.0, 1.0), "point0": (0.0, 0.0, zmin - radius), "velocity": (0.0, 0.0, 0.0),
         "penalty": penalty},
        {"normal": (0.0, 0.0, -1.0), "point0": (0.0, 0.0, zmax + radius),
         "velocity": (0.0, 0.0, -float(plate_velocity)), "penalty": penalty},
    ]
    contact = Contact(radius=radius, penalty=penalty, margin=(2.0 * radius if margin is None else margin),
                      plates=plates)
    spec = ModelSpec(coords=coords, conn=conn, elem_rod=elem_rod, materials=[mat], n_gauss=1, dt=dt,
                     bcs=[], contact=contact, name=f"fibres{n_rods}")
    spec.generator_tries = tries
    return spec


# ---------------------------------------------------------------------------
# rigid hinges
# ---------------------------------------------------------------------------

def with_hinges(spec: ModelSpec, rods=None) -> ModelSpec:
    """The hinges a rod model's ``hinges`` property creates
    (HingeModel::createHinges_, HingeModel.cpp:268-358): along each rod, in
    element order, the first node of every element is duplicated and the
    element takes the copy, and finally the last node of the rod's last
    element; each copy is tied to the node it was made from (the copy is the
    slave, HingeModel.cpp:172-199).  ``rods``: the rod indices to hinge (all
    by default).  Returns a new spec with the extra nodes and the ties."""
    import copy as _copy
    coords = [tuple(x) for x in spec.coords]
    conn = spec.conn.copy()
    ties = []
    rod_ids = np.unique(spec.elem_rod) if rods is None else np.asarray(rods)
    for r in rod_ids:
        elems = np.flatnonzero(spec.elem_rod == r)
        for e in elems:
            orig = int(conn[e, 0])
            coords.append(coords[orig])
            new = len(coords) - 1
            conn[e, 0] = new
            ties.append((orig, new))
        e = elems[-1]
        orig = int(conn[e, 1])
        coords.append(coords[orig])
        new = len(coords) - 1
        conn[e, 1] = new
        ties.append((orig, new))
    out = _copy.copy(spec)
    out.coords = np.asarray(coords, dtype=np.float64)
    out.conn = np.ascontiguousarray(conn, dtype=np.int32)
    out.ties = np.asarray(ties, dtype=np.int32)
    out.name = spec.name + "+hinges"
    return out
