"""MilneDevice predictor-corrector with error-controlled dt on the GPU (the
persistent k_milne launch) against the oracle's MilneDevice: accepted and
rejected attempts, time-dependent load scales evaluated on the device,
plastic history committed from the corrector's force evaluation, samples
and energies."""
import numpy as np
import pytest

import transient_cases as tc
from dynlattice_b200 import lattices
from dynlattice_b200.abi import BC, DL_BC_NEUMANN, DL_MIXED, DL_PLAIN_FP64, Integrator
from dynlattice_b200.engine import DLError, Lattice
from helpers import rel_err
from oracle_ffi import Oracle

pytestmark = pytest.mark.gpu


def _pair(spec, integ, precision, threads=2):
    o = Oracle(spec, threads=threads)
    o.set_integrator(integ)
    g = Lattice(spec, precision)
    g.set_integrator(integ)
    return o, g


@pytest.mark.parametrize("dt0,prec", [(1e-6, 1e-6), (2e-4, 1e-7)])
def test_swinging_rod_fp64(gpu, dt0, prec):
    spec = tc.swinging_rod(dt=dt0)
    o, g = _pair(spec, Integrator.milne(prec), DL_PLAIN_FP64)
    for _ in range(3):
        o.run(150)
        g.run(150)
        to, dto, so, ro = o.time()
        tg, dtg, sg, rg = g.time()
        assert (sg, rg) == (so, ro)
        assert tg == pytest.approx(to, rel=1e-12) and dtg == pytest.approx(dto, rel=1e-10)
        ug, thg, vg = g.state()
        uo, tho, vo = o.state()
        assert rel_err(ug, uo) < 1e-10 and rel_err(thg, tho) < 1e-10 and rel_err(vg, vo) < 1e-9
    if dt0 > 1e-5:
        assert ro > 0


def test_swinging_rod_mixed(gpu):
    spec = tc.swinging_rod(dt=1e-6)
    o, g = _pair(spec, Integrator.milne(1e-6), DL_MIXED)
    o.run(2000)
    g.run(2000)
    to, _, _, _ = o.time()
    tg, _, _, _ = g.time()
    assert tg == pytest.approx(to, rel=1e-5)
    ug, _, _ = g.state()
    uo, _, _ = o.state()
    assert rel_err(ug, uo) < 1e-4


@pytest.mark.parametrize("case", ["dirichlet", "neumann"])
def test_load_scales_on_device(gpu, case):
    """Time-dependent LoadScale functions evaluated by the device program at
    the adapted times: a scaled rotational acceleration (the spin-up beam
    with 8 two-node elements) and scaled gravity loads (the swinging rod).
    The scales are nonzero from t = 0, so the motion is never at the
    rounding level of the positions (a ramp from zero, as in test1, is:
    the first hundred steps then compare rounding noise)."""
    if case == "dirichlet":
        spec = tc.spin_up_beam(n_elems=8, order=1)
        spec.bcs = [b if b.scale is None else BC(b.kind, b.dof, b.nodes, 0.4, "1 + sin(40 * t)") for b in spec.bcs]
        n = 1500
    else:
        spec = tc.swinging_rod(dt=1e-6)
        spec.bcs = [BC(b.kind, b.dof, b.nodes, b.factor, "1 + 0.5 * sin(20 * t)") if b.kind == DL_BC_NEUMANN else b
                    for b in spec.bcs]
        n = 3000
    o, g = _pair(spec, Integrator.milne(tc.MILNE_PRECISION), DL_PLAIN_FP64)
    free = spec.coords.shape[0] - 1
    o.set_sampling(10, [0, free])
    g.set_sampling(10, [0, free], capacity=n // 10 + 1)
    o.run(n)
    g.run(n)
    to, dto, _, ro_ = o.time()
    tg, dtg, _, rg_ = g.time()
    assert rg_ == ro_ and tg == pytest.approx(to, rel=1e-10) and dtg == pytest.approx(dto, rel=1e-9)
    so, ro, eo = o.samples()
    sg, rg, eg = g.samples()
    assert np.array_equal(so, sg)
    assert np.allclose(g.sample_times(), o.sample_times(len(so)), rtol=1e-10, atol=0)
    assert rel_err(rg[:, 1, :3], ro[:, 1, :3]) < 1e-8     # free-end displacement
    assert rel_err(rg[:, 1, 6:], ro[:, 1, 6:]) < 1e-7     # free-end velocity
    assert rel_err(eg[:, :2], eo[:, :2]) < 1e-7


@pytest.mark.parametrize("precision,tol", [(DL_PLAIN_FP64, 1e-9), (DL_MIXED, 1e-4)])
def test_plastic_lattice_with_rejections(gpu, precision, tol):
    """An elastoplastic impact started at 10x the stable dt: rejected
    attempts first, then accepted steps whose history comes from the
    corrector's force evaluation."""
    spec = lattices.lattice_impact("bcc", n=2, velocity=20.0, dt=5e-7, plastic=True, seed=4)
    o, g = _pair(spec, Integrator.milne(1e-6), precision)
    o.run(200)
    g.run(200)
    to, dto, so, ro = o.time()
    tg, dtg, sg, rg = g.time()
    assert ro > 0 and sg == so
    if precision == DL_PLAIN_FP64:
        assert rg == ro
    assert tg == pytest.approx(to, rel=tol)
    ug, _, vg = g.state()
    uo, _, vo = o.state()
    assert rel_err(ug, uo) < tol and rel_err(vg, vo) < 10 * tol
    eo, eg = o.energies(), g.energies()
    for k in ("kinetic", "potential", "dissipated"):
        assert eg[k] == pytest.approx(eo[k], rel=10 * tol), k
    _, _, edo = o.history()
    _, _, edg = g.history()
    assert rel_err(edg, edo) < 10 * tol


def test_leapfrog_after_milne_and_refusals(gpu):
    """Back to LeapFrog continues from the Milne state at the adapted time;
    batches and contact are refused with DL_ERR_UNSUPPORTED."""
    spec = tc.swinging_rod(dt=1e-6)
    g = Lattice(spec, DL_PLAIN_FP64)
    g.set_integrator(Integrator.milne(1e-6))
    g.run(100)
    t1 = g.time()[0]
    g.set_integrator(Integrator())
    g.run(10)
    t2, dt2, s2, _ = g.time()
    assert s2 == 110 and dt2 == spec.dt and t2 == pytest.approx(t1 + 10 * spec.dt, rel=1e-12)
    import contact_cases as cc
    c = Lattice(cc.cross(), DL_PLAIN_FP64)
    with pytest.raises(DLError):
        c.set_integrator(Integrator.milne(1e-6))
