"""MilneDevice predictor-corrector with error-controlled dt in the oracle
(oracle/oracle.cpp, milneAttempt), pinned two ways:
  * against a numpy restatement of MilneDeviceModule::solve
    (MilneDeviceModule.cpp:41-118) with ExplicitModule::getQuality (:494-501),
    ::commit and ::cancel (:277-334), driven only by the oracle's internal
    force and mass evaluations, including rejected steps;
  * against the reference's transient benchmark that runs MilneDevice
    (tests/transient/test2: Lang et al. 2011, 5 % on the digitised curves).
"""
import numpy as np
import pytest
from scipy.spatial.transform import Rotation

import transient_cases as tc
from dynlattice_b200 import lattices
from dynlattice_b200.abi import DL_BC_DIRICHLET, DL_BC_NEUMANN, Integrator
from oracle_ffi import Oracle


def _loads(spec):
    N = spec.coords.shape[0]
    fext = np.zeros((N, 6))
    mask = np.zeros((N, 6), bool)
    apre = np.zeros((N, 6))
    for b in spec.bcs:
        if b.kind == DL_BC_NEUMANN:
            assert b.scale is None
            np.add.at(fext[:, b.dof], b.nodes, b.factor)
        elif b.kind == DL_BC_DIRICHLET:
            assert b.scale is None
            mask[b.nodes, b.dof] = True
            apre[b.nodes, b.dof] = b.factor
    return fext, mask, apre


def _accel(o, u, th, v, mT, mR, fext, mask, apre):
    f = o.internal_force(u, th)
    w = v[:, 3:]
    f[:, 3:] += np.cross(w, np.einsum("nij,nj->ni", mR, w))  # gyroscopic term
    r = fext - f
    a = apre.copy()
    free_t = ~mask[:, :3]
    a[:, :3][free_t] = (r[:, :3] / mT[:, None])[free_t]
    for n in range(u.shape[0]):
        fr = ~mask[n, 3:]
        if fr.any():
            b = r[n, 3:][fr] - mR[n][np.ix_(fr, ~fr)] @ a[n, 3:][~fr]
            a[n, 3:][fr] = np.linalg.solve(mR[n][np.ix_(fr, fr)], b)
    return a


def _rot_update(th, dr):
    return (Rotation.from_rotvec(dr) * Rotation.from_rotvec(th)).as_rotvec()


def _quality(a, b, L):
    d = (a - b).copy()
    d[:, :3] /= L
    return np.linalg.norm(d) / np.sqrt(d.size)


def milne_numpy(o, spec, nsteps, prec, L=1e-3, safety=0.9, incr=1.2, decr=0.8):
    """Reference MilneDevice + ExplicitModule step control (order 1)."""
    dt = spec.dt
    min_dt, max_dt = dt / 100, dt * 100
    u, th, v = o.state()
    fext, mask, apre = _loads(spec)
    t, step, rejected, dts = 0.0, 0, 0, []
    while step < nsteps:
        mT, mR = o.mass(th)
        a_cur = _accel(o, u, th, v, mT, mR, fext, mask, apre)
        v_pre = v + dt * a_cur
        u_pre = u + dt * v[:, :3]
        th_pre = _rot_update(th, dt * v[:, 3:])
        a_pre = _accel(o, u_pre, th_pre, v_pre, mT, mR, fext, mask, apre)
        v_new = v + dt * a_pre
        u_new = u + dt * v_pre[:, :3]
        th_new = _rot_update(th, dt * v_pre[:, 3:])
        err = 0.5 * (_quality(np.hstack([u_pre, th_pre]), np.hstack([u_new, th_new]), L)
                     + _quality(v_pre, v_new, L) * dt)
        dt_opt = dt * np.sqrt(prec / err)
        if err <= prec or dt <= min_dt:
            t += dt
            step += 1
            dts.append(dt)
            u, th, v = u_new, th_new, v_new
            dt = max(min(safety * dt_opt, incr * dt, max_dt), decr * dt, min_dt)
        else:
            dt = max(safety * dt_opt, decr * dt, min_dt)
            rejected += 1
    return (u, th, v), (t, dt, step, rejected), np.array(dts)


def _case(name, dt0):
    if name == "rod":
        return tc.swinging_rod(dt=dt0)
    # initial velocity on the top face (an InitLoad value, not a constraint),
    # acceleration constraints, two Gauss points
    return lattices.lattice_impact("bcc", n=1, velocity=20.0, dt=dt0, plastic=False, seed=4)


@pytest.mark.parametrize("case,dt0,prec", [("rod", 1e-6, 1e-6), ("rod", 2e-4, 1e-7), ("lattice", 5e-7, 1e-6)])
def test_milne_oracle_matches_numpy_restatement(case, dt0, prec):
    """Accepted and (with the large first dt) rejected attempts: the same
    time, dt, counts and state as the numpy restatement."""
    spec = _case(case, dt0)
    ref = Oracle(spec)
    (u, th, v), (t, dt, step, rej), _ = milne_numpy(ref, spec, 120, prec)
    o = Oracle(spec)
    o.set_integrator(Integrator.milne(prec))
    o.run(120)
    to, dto, so, ro = o.time()
    assert so == step == 120 and ro == rej
    if dt0 > 1e-5 or case == "lattice":
        assert rej > 0  # the rejection branch ran
    assert to == pytest.approx(t, rel=1e-12) and dto == pytest.approx(dt, rel=1e-9)
    uo, tho, vo = o.state()
    scale = np.abs(u).max() + 1e-30
    assert np.abs(uo - u).max() <= 1e-9 * scale
    assert np.abs(tho - th).max() <= 1e-9 * (np.abs(th).max() + 1e-30)
    assert np.abs(vo - v).max() <= 1e-9 * (np.abs(v).max() + 1e-30)


def test_milne_step_control_bounds():
    """dt stays in [dt0/100, 100 dt0], never grows by more than x1.2 per
    accepted step, and sample times are the accumulated accepted dts."""
    spec = tc.swinging_rod(dt=1e-6)
    o = Oracle(spec)
    o.set_integrator(Integrator.milne(1e-6))
    o.set_sampling(1, [spec.coords.shape[0] - 1])
    o.run(400)
    steps, _, _ = o.samples()
    ts = o.sample_times(len(steps))
    dts = np.diff(np.concatenate([[0.0], ts]))
    assert (dts >= 1e-8 * (1 - 1e-12)).all() and (dts <= 1e-4 * (1 + 1e-12)).all()
    assert (dts[1:] <= 1.2 * dts[:-1] * (1 + 1e-12)).all()
    assert np.array_equal(steps, np.arange(1, 401))


def test_milne_swinging_rod_lang():
    """tests/transient/test2 with its own integrator (MilneDevice, deltaTime
    1e-6): rod shapes at t = 0.0 ... 1.0 within 5 % of Lang et al."""
    lit = tc.literature()
    spec = tc.swinging_rod()
    o = Oracle(spec)
    o.set_integrator(Integrator.milne(tc.MILNE_PRECISION))
    shapes = []
    for target in lit["test2_times"]:
        while o.time()[0] < target - 1e-12:
            o.run(1)
        u, _, _ = o.state()
        x = spec.coords + u
        shapes.append(np.stack([x[:, 0], x[:, 2]], 1))
    errs = tc.swinging_errors(lit["test2_times"], shapes, lit)
    assert max(errs.values()) <= 0.05, errs
