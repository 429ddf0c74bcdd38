"""Finite-difference checks of the adjoint building blocks on the CPU.

tests/cpp/adjoint_check.cpp compiles the engine's adjoint header
(dynlattice_b200/csrc/adjoint.cuh) for the host together with the yield
policy the engine generates (dl_yield_source, reverse-mode product included).
Each vector-Jacobian product is compared with central differences of the
matching pure forward function: the element (elastic and elastoplastic, all
inputs: node positions and rotations, section constants, history), the node
update (all inputs, with and without constraints) and the yield policy.
"""
import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np
import pytest

from dynlattice_b200 import lattices
from dynlattice_b200.engine import load_library

ROOT = Path(__file__).resolve().parent.parent
NAMES = ["dx", "dy", "dz", "rx", "ry", "rz", "h_0", "radius", "area"]


def yield_source(mat, fp32=False, adjoint=True, host=True):
    lib = load_library()
    f = lib.dl_yield_source
    f.argtypes = [C.c_char_p, C.c_int32, C.POINTER(C.c_char_p), C.c_int32, C.POINTER(C.c_char_p), C.c_int32,
                  C.c_int32, C.c_int32, C.c_char_p, C.c_int64, C.POINTER(C.c_int64)]
    derivs = (C.c_char_p * len(mat.yield_deriv))(*[d.encode() for d in mat.yield_deriv])
    names = (C.c_char_p * len(NAMES))(*[n.encode() for n in NAMES])
    need = C.c_int64()
    rc = f(mat.yield_cond.encode(), len(mat.yield_deriv), derivs, len(NAMES), names, int(fp32), int(adjoint),
           int(host), None, 0, C.byref(need))
    assert rc == 0
    buf = C.create_string_buffer(need.value)
    assert f(mat.yield_cond.encode(), len(mat.yield_deriv), derivs, len(NAMES), names, int(fp32), int(adjoint),
             int(host), buf, need.value, C.byref(need)) == 0
    return buf.value.decode()


@pytest.fixture(scope="module")
def ac(tmp_path_factory):
    d = tmp_path_factory.mktemp("adjcheck")
    mat = lattices.aluminium_elastoplastic(0.5e-3)
    (d / "yield_policy.inc").write_text(yield_source(mat))
    so = d / "libac.so"
    cmd = ["g++", "-O1", "-std=c++17", "-shared", "-fPIC", f"-I{ROOT / 'dynlattice_b200' / 'csrc'}", f"-I{d}",
           str(ROOT / "tests" / "cpp" / "adjoint_check.cpp"), "-o", str(so)]
    subprocess.run(cmd, check=True, capture_output=True)
    lib = C.CDLL(str(so))
    dp = C.POINTER(C.c_double)
    lib.ac_setup.argtypes = [dp, dp, C.c_double, C.c_double, dp, dp, C.c_int, C.c_int, C.c_int, dp, C.c_int,
                             C.c_double]
    lib.ac_elem_forward.argtypes = [dp, dp, dp]
    lib.ac_elem_vjp.argtypes = [dp, dp, dp, dp]
    lib.ac_node_forward.argtypes = [dp, dp, dp, C.c_int, C.c_int, C.c_double, dp]
    lib.ac_node_vjp.argtypes = [dp, dp, dp, C.c_int, C.c_int, C.c_double, dp, dp]
    lib.ac_yield.argtypes = [dp, C.c_int, C.c_int, dp, dp, C.c_double, dp, dp]
    lib.mat = mat
    return lib


def P(a):
    return np.ascontiguousarray(a, dtype=np.float64).ctypes.data_as(C.POINTER(C.c_double))


# --- quaternion helpers (w, x, y, z) ---
def qmul(a, b):
    w1, x1, y1, z1 = a
    w2, x2, y2, z2 = b
    return np.array([w1 * w2 - x1 * x2 - y1 * y2 - z1 * z2, w1 * x2 + x1 * w2 + y1 * z2 - z1 * y2,
                     w1 * y2 - x1 * z2 + y1 * w2 + z1 * x2, w1 * z2 + x1 * y2 - y1 * x2 + z1 * w2])


def qexp(v):
    t = np.linalg.norm(v)
    if t < 1e-300:
        return np.array([1.0, *(0.5 * v)])
    return np.array([np.cos(t / 2), *(np.sin(t / 2) / t * v)])


def rand_quat(rng, scale=1.0):
    return qexp(rng.normal(scale=scale, size=3))


def qmat(q):
    w, x, y, z = q
    return np.array([[w * w + x * x - y * y - z * z, 2 * (x * y - w * z), 2 * (x * z + w * y)],
                     [2 * (x * y + w * z), w * w - x * x + y * y - z * z, 2 * (y * z - w * x)],
                     [2 * (x * z - w * y), 2 * (y * z + w * x), w * w - x * x - y * y + z * z]])


def mat_quat(R):
    tr = np.trace(R)
    if tr > 0:
        s = np.sqrt(tr + 1.0) * 2
        return np.array([0.25 * s, (R[2, 1] - R[1, 2]) / s, (R[0, 2] - R[2, 0]) / s, (R[1, 0] - R[0, 1]) / s])
    i = int(np.argmax(np.diag(R)))
    j, k = (i + 1) % 3, (i + 2) % 3
    s = np.sqrt(1.0 + R[i, i] - R[j, j] - R[k, k]) * 2
    q = np.zeros(4)
    q[0] = (R[k, j] - R[j, k]) / s
    q[1 + i] = 0.25 * s
    q[1 + j] = (R[j, i] + R[i, j]) / s
    q[1 + k] = (R[k, i] + R[i, k]) / s
    return q


# --- element -------------------------------------------------------------

def _element_case(ac, rng, plastic, G=2, stretch=0.012):
    L0 = 5e-3
    qNi, qNj = rand_quat(rng, 0.3), rand_quat(rng, 0.3)
    g0 = rng.normal(scale=1e-3, size=(G, 3))
    k0 = rng.normal(scale=1e-1, size=(G, 3))
    H = np.zeros((7, 7))
    H[0, 0] = 1e9
    ac.ac_setup(P(qNi), P(qNj), 1.0 / L0, L0, P(g0.ravel()), P(k0.ravel()), G, 1, int(plastic), P(H.ravel()), 20,
                1e-5)
    r = 0.5e-3
    A, I = np.pi * r * r, np.pi * r ** 4 / 4
    E, Gm = 70e9, 70e9 / 2 / 1.33
    Cd = [Gm * 0.9 * A, Gm * 0.9 * A, E * A, E * I, E * I, Gm * 2 * I]
    t = qmat(qNi) @ np.array([0, 0, 1.0])
    xi = rng.normal(scale=1e-3, size=3)
    xj = xi + L0 * (1 + stretch) * t + rng.normal(scale=2e-5, size=3)
    Ri, Rj = rand_quat(rng, 0.05), rand_quat(rng, 0.05)
    ep = rng.normal(scale=1e-4, size=(G, 6))
    al = np.abs(rng.normal(scale=1e-4, size=(G, 1)))
    epsc = rng.normal(scale=1e-3, size=(G, 6))
    p = np.concatenate([xi, xj, Ri, Rj, Cd, [r, A], ep.ravel(), al.ravel(), epsc.ravel()])
    return p, G


def _elem_J(ac, p, lf, lh, G):
    f = np.zeros(12)
    h = np.zeros(G * 6 + G * 1 + G * 6 + G)
    ac.ac_elem_forward(P(p), P(f), P(h))
    return lf @ f + lh @ h


def _perturb(p, idx, eps, rot_slot=None):
    q = p.copy()
    if rot_slot is None:
        q[idx] += eps
    else:
        off, k = rot_slot
        v = np.zeros(3)
        v[k] = eps
        q[off:off + 4] = qmul(qexp(v), p[off:off + 4])
    return q


@pytest.mark.parametrize("plastic", [False, True])
def test_element_vjp_matches_finite_differences(ac, plastic):
    rng = np.random.default_rng(7 if plastic else 3)
    p, G = _element_case(ac, rng, plastic)
    nh = 1
    lf = rng.normal(size=12)
    lh = rng.normal(size=G * 6 + G * nh + G * 6 + G) * (1.0 if plastic else 0.0)
    lh[-G:] = [1.3, 0.7][:G] if plastic else 0.0
    out = np.zeros(3 * 4 + 6 + 2 + G * 6 + G * nh + G * 6)
    ac.ac_elem_vjp(P(p), P(lf), P(lh), P(out))
    # check the return map was active in the plastic case
    f = np.zeros(12)
    h = np.zeros(G * 6 + G * nh + G * 6 + G)
    ac.ac_elem_forward(P(p), P(f), P(h))
    if plastic:
        assert np.abs(h[-G:]).max() > 0, "plastic flow expected"
    checks = []
    # translations
    for k in range(6):
        sc = 1e-8   # metres (L0 = 5 mm); the return map needs small steps
        num = (_elem_J(ac, _perturb(p, k, sc), lf, lh, G) - _elem_J(ac, _perturb(p, k, -sc), lf, lh, G)) / (2 * sc)
        checks.append((f"x{k}", out[k], num))
    # rotations (spatial tangent)
    for n, off in enumerate((6, 10)):
        for k in range(3):
            e = 1e-7
            num = (_elem_J(ac, _perturb(p, None, e, (off, k)), lf, lh, G) -
                   _elem_J(ac, _perturb(p, None, -e, (off, k)), lf, lh, G)) / (2 * e)
            checks.append((f"th{n}{k}", out[6 + 3 * n + k], num))
    # section constants, yield variables and history
    names = [f"C{k}" for k in range(6)] + ["radius", "area"]
    idx_p = list(range(14, 22))
    idx_o = list(range(12, 20))
    if plastic:
        for g in range(G):
            names += [f"ep{g}{k}" for k in range(6)]
        names += [f"al{g}" for g in range(G)]
        for g in range(G):
            names += [f"epsc{g}{k}" for k in range(6)]
        idx_p += list(range(22, 22 + G * 13))
        idx_o += list(range(20, 20 + G * 13))
    for nm, ip, io in zip(names, idx_p, idx_o):
        # constants: relative steps of 1e-5 keep the difference well above the
        # rounding of J
        sc = 1e-5 * abs(p[ip]) if nm[0] in "Cra" else 1e-8   # history: strain units
        num = (_elem_J(ac, _perturb(p, ip, sc), lf, lh, G) - _elem_J(ac, _perturb(p, ip, -sc), lf, lh, G)) / (2 * sc)
        checks.append((nm, out[io], num))
    bad = [(n, a, b) for n, a, b in checks if abs(a - b) > 1e-5 * max(abs(b), 1e-30) + 1e-7 * _scale(checks, n)]
    assert not bad, bad


def _scale(checks, name):
    """magnitude of the gradient entries of the same group (absolute floor)"""
    grp = name.rstrip("0123456789")
    vals = [abs(b) for n, _, b in checks if n.rstrip("0123456789") == grp]
    return max(vals) if vals else 1.0


# --- node ----------------------------------------------------------------

def _node_case(rng, gyro=1):
    x = rng.normal(size=3)
    R = rand_quat(rng, 1.0)
    v = rng.normal(size=6) * np.array([1, 1, 1, 50, 50, 50])
    fint = rng.normal(size=6) * np.array([1, 1, 1, 1e-3, 1e-3, 1e-3])
    mass = 2e-6
    S = rng.normal(size=(3, 3)) * 1e-12
    S = S @ S.T + np.eye(3) * 3e-12
    return x, R, v, fint, mass, S


def _pd_from_S(S):
    w, V = np.linalg.eigh(S)
    if np.linalg.det(V) < 0:
        V[:, 0] *= -1
    return mat_quat(V), w


def _node_pack(x, R, v, fint, mass, S):
    Pq, D = _pd_from_S(S)
    return np.concatenate([x, R, v, fint, [mass], Pq, D])


@pytest.mark.parametrize("mask,gyro", [(0, 1), (0, 0), (0b000111, 1), (0b101000, 1), (0b111111, 1),
                                       (0b010111, 1)])
def test_node_vjp_matches_finite_differences(ac, mask, gyro):
    rng = np.random.default_rng(11 + mask)
    x, R, v, fint, mass, S = _node_case(rng, gyro)
    aPre = rng.normal(size=6) * np.array([1, 1, 1, 10, 10, 10])
    fx = rng.normal(size=6) * np.array([1, 1, 1, 1e-3, 1e-3, 1e-3])
    dt = 1e-6
    lq = rng.normal(size=4)
    lx1, lv1, lfseed = rng.normal(size=3), rng.normal(size=6), rng.normal(size=6)

    def fwd(x, R, v, fint, mass, S):
        out = np.zeros(13)
        ac.ac_node_forward(P(_node_pack(x, R, v, fint, mass, S)), P(aPre), P(fx), mask, gyro, dt, P(out))
        return out

    def J(x, R, v, fint, mass, S):
        o = fwd(x, R, v, fint, mass, S)
        return lx1 @ o[0:3] + lq @ o[3:7] + lv1 @ o[7:13] + lfseed @ fint

    o = fwd(x, R, v, fint, mass, S)
    R1 = o[3:7]
    u = R1[1:]
    lth1 = 0.5 * (-lq[0] * u + R1[0] * lq[1:] + np.cross(u, lq[1:]))
    adj = np.concatenate([lx1, lth1, lv1, lfseed])
    out = np.zeros(25)
    ac.ac_node_vjp(P(_node_pack(x, R, v, fint, mass, S)), P(aPre), P(fx), mask, gyro, dt, P(adj), P(out))
    checks = []
    for k in range(3):
        e = 1e-6
        xp, xm = x.copy(), x.copy()
        xp[k] += e
        xm[k] -= e
        checks.append((f"x{k}", out[k], (J(xp, R, v, fint, mass, S) - J(xm, R, v, fint, mass, S)) / (2 * e)))
    for k in range(3):
        e = 1e-4   # J is smooth in R; larger steps keep rounding out of the difference
        d = np.zeros(3)
        d[k] = e
        Rp, Rm = qmul(qexp(d), R), qmul(qexp(-d), R)
        checks.append((f"th{k}", out[3 + k], (J(x, Rp, v, fint, mass, S) - J(x, Rm, v, fint, mass, S)) / (2 * e)))
    for k in range(6):
        e = 1e-4 * max(1.0, abs(v[k]))
        vp, vm = v.copy(), v.copy()
        vp[k] += e
        vm[k] -= e
        checks.append((f"v{k}", out[6 + k], (J(x, R, vp, fint, mass, S) - J(x, R, vm, fint, mass, S)) / (2 * e)))
    for k in range(6):
        e = 1e-4 * max(1e-3, abs(fint[k]))
        fp, fm = fint.copy(), fint.copy()
        fp[k] += e
        fm[k] -= e
        checks.append((f"f{k}", out[12 + k], (J(x, R, v, fp, mass, S) - J(x, R, v, fm, mass, S)) / (2 * e)))
    e = 1e-4 * mass
    checks.append(("mass", out[18], (J(x, R, v, fint, mass + e, S) - J(x, R, v, fint, mass - e, S)) / (2 * e)))
    dS = rng.normal(size=(3, 3))
    dS = dS + dS.T
    e = 1e-4 * np.abs(S).max()
    num = (J(x, R, v, fint, mass, S + e * dS) - J(x, R, v, fint, mass, S - e * dS)) / (2 * e)
    lS = out[19:25]
    ana = (lS[0] * dS[0, 0] + lS[1] * dS[1, 1] + lS[2] * dS[2, 2] +
           2 * (lS[3] * dS[0, 1] + lS[4] * dS[0, 2] + lS[5] * dS[1, 2]))
    checks.append(("S", ana, num))
    bad = [(n, a, b) for n, a, b in checks if abs(a - b) > 1e-6 * max(abs(b), 1e-30) + 1e-9 * _scale(checks, n)]
    assert not bad, bad


# --- yield policy --------------------------------------------------------

def test_yield_vjp_matches_finite_differences(ac):
    rng = np.random.default_rng(5)
    r = 0.5e-3
    A = np.pi * r * r
    args = np.array([30.0, -20.0, 200.0, 0.03, -0.02, 0.01, -5e6, r, A])
    lg = rng.normal(size=7)
    lf = 0.7
    fv, g, la = np.zeros(1), np.zeros(7), np.zeros(9)
    ac.ac_yield(P(args), 9, 7, P(fv), P(g), lf, P(lg), P(la))

    def J(a):
        f1, g1, l1 = np.zeros(1), np.zeros(7), np.zeros(9)
        ac.ac_yield(P(a), 9, 7, P(f1), P(g1), 0.0, P(lg), P(l1))
        return lf * f1[0] + lg @ g1

    for i in range(9):
        e = 1e-6 * max(abs(args[i]), 1e-9)
        ap, am = args.copy(), args.copy()
        ap[i] += e
        am[i] -= e
        num = (J(ap) - J(am)) / (2 * e)
        assert abs(la[i] - num) <= 1e-5 * abs(num) + 1e-9 * np.abs(la).max(), (i, la[i], num)
    # the gradient expressions are the derivatives of f
    for i in range(7):
        e = 1e-6 * max(abs(args[i]), 1e-9)
        ap, am = args.copy(), args.copy()
        ap[i] += e
        am[i] -= e
        f1, f2, gg, ll = np.zeros(1), np.zeros(1), np.zeros(7), np.zeros(9)
        ac.ac_yield(P(ap), 9, 7, P(f1), P(gg), 0.0, P(lg), P(ll))
        ac.ac_yield(P(am), 9, 7, P(f2), P(gg), 0.0, P(lg), P(ll))
        assert abs((f1[0] - f2[0]) / (2 * e) - g[i]) <= 1e-5 * abs(g[i]) + 1e-12
