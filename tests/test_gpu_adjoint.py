"""Adjoint of the explicit impact dynamics (dl_adjoint_radius) on the GPU.

Objective (the config of the differentiation workload, reduced size):
J = E_diss(T) - 0.1 * max_k |R(k)|, R(k) the summed internal force z of the
top face at step k (its peak magnitude is the peak reaction force), with respect to the strut radii (each strut's elements
share one parameter).  The gradient is checked against central finite
differences of J (relative step 1e-6) along seeded random directions, with
the forward computed by the same engine in FP64; the mixed-precision adjoint
is checked against the FP64 finite-difference gradient."""
import copy

import numpy as np
import pytest

from dynlattice_b200 import lattices
from dynlattice_b200.abi import DL_MIXED, DL_PLAIN_FP64
from dynlattice_b200.engine import Lattice
from helpers import rel_err

pytestmark = pytest.mark.gpu

REACT_W = -0.1


def _impact(plastic=True, n=2, v=20.0):
    return lattices.lattice_impact("bcc", n=n, velocity=v, dt=5e-8, plastic=plastic, seed=4)


def _with_radii(spec, r_strut):
    s = copy.copy(spec)
    s.elem_radius = np.repeat(np.asarray(r_strut, float), 2)
    return s


def _run(spec, r_strut, steps, K, prec):
    g = Lattice(_with_radii(spec, r_strut), prec)
    J, grad = g.adjoint_radius(steps, K, elem_param=spec.elem_rod, react_nodes=spec.groups["top"], react_dof=2,
                               react_weight=REACT_W)
    g.synchronize()
    return J, grad, g


def _fd_directional(spec, r0, d, steps, K, h_rel=1e-6):
    h = h_rel * np.abs(r0).mean()
    Jp, _, _ = _run(spec, r0 + h * d, steps, 0, DL_PLAIN_FP64)   # objective only
    Jm, _, _ = _run(spec, r0 - h * d, steps, 0, DL_PLAIN_FP64)
    return (Jp - Jm) / (2 * h)


@pytest.mark.parametrize("plastic,steps,K", [(False, 300, 64), (True, 400, 100)])
def test_adjoint_matches_finite_differences_fp64(gpu, plastic, steps, K):
    spec = _impact(plastic)
    r0 = spec.strut_radius.copy()
    J, grad, _ = _run(spec, r0, steps, K, DL_PLAIN_FP64)
    assert np.isfinite(grad).all() and np.abs(grad).max() > 0
    rng = np.random.default_rng(1)
    for _ in range(4):
        d = rng.normal(size=r0.size)
        fd = _fd_directional(spec, r0, d, steps, K)
        ad = grad @ d
        assert abs(ad - fd) <= 1e-4 * max(abs(fd), 1e-3 * np.abs(grad).sum() * np.abs(d).mean()), (ad, fd)


def test_adjoint_mixed_against_fp64_fd(gpu):
    spec = _impact(True)
    r0 = spec.strut_radius.copy()
    steps, K = 400, 100
    J64, g64, _ = _run(spec, r0, steps, K, DL_PLAIN_FP64)
    J32, g32, _ = _run(spec, r0, steps, K, DL_MIXED)
    assert abs(J32 - J64) <= 1e-4 * abs(J64)
    rng = np.random.default_rng(2)
    for _ in range(3):
        d = rng.normal(size=r0.size)
        fd = _fd_directional(spec, r0, d, steps, K)
        assert abs(g32 @ d - fd) <= 2e-2 * abs(fd) + 1e-3 * np.abs(g64).sum() * np.abs(d).mean() / d.size, (g32 @ d, fd)
    assert rel_err(g32, g64) < 5e-2


@pytest.mark.parametrize("steps", [250, 120, 61])
def test_checkpoint_mode_equals_full_tape(gpu, steps):
    """Checkpoints every 60 steps with recomputation (tape budget 0) give the
    same gradient as the full tape: the recomputed segments are bitwise the
    forward run's steps.  Odd, even and a single-step last segment: the
    recomputation alternates between two tape sets while the reverse sweep
    over the previous segment runs on its own stream."""
    spec = _impact(True)
    r0 = spec.strut_radius.copy()
    out = []
    for budget in (-1, 0):
        g = Lattice(_with_radii(spec, r0), DL_PLAIN_FP64)
        g.set_tape_budget(budget)
        out.append(g.adjoint_radius(steps, 60, elem_param=spec.elem_rod, react_nodes=spec.groups["top"],
                                    react_dof=2, react_weight=REACT_W))
    assert out[0][0] == out[1][0]
    assert rel_err(out[1][1], out[0][1]) < 1e-13


def test_retained_tape_pool(gpu):
    """Gradients on successive handles (the tape memory of the first one
    reused from the retained pool) and after trimming the pool are equal."""
    from dynlattice_b200.engine import trim_retained_memory
    spec = _impact(True)
    r0 = spec.strut_radius.copy()
    res = []
    for trim in (False, False, True):
        if trim:
            trim_retained_memory()
        res.append(_run(spec, r0, 200, 50, DL_MIXED)[:2])
    for J, g in res[1:]:
        assert J == res[0][0]
        assert np.array_equal(g, res[0][1])


@pytest.mark.parametrize("budget", [-1, 0])
def test_adjoint_leaves_final_state(gpu, budget):
    spec = _impact(True)
    r0 = spec.strut_radius.copy()
    g = Lattice(_with_radii(spec, r0), DL_PLAIN_FP64)
    g.set_tape_budget(budget)
    g.adjoint_radius(250, 60, elem_param=spec.elem_rod, react_nodes=spec.groups["top"], react_dof=2,
                     react_weight=REACT_W)
    g.synchronize()
    ref = Lattice(_with_radii(spec, r0), DL_PLAIN_FP64)
    ref.run(250)
    ua, ta, va = g.state()
    ub, tb, vb = ref.state()
    assert rel_err(ua, ub) < 1e-12 and rel_err(va, vb) < 1e-12
    ea, eb = g.energies(), ref.energies()
    assert abs(ea["dissipated"] - eb["dissipated"]) <= 1e-12 * abs(eb["dissipated"])
    assert g.step == 250


def test_objective_value(gpu):
    """J of the adjoint call = E_diss(T) + w * max_k |R(k)|, with R(k) rebuilt
    from plain single steps (dl_group_sums: the internal force of the last
    step)."""
    spec = _impact(True)
    r0 = spec.strut_radius.copy()
    steps = 200
    J, _, _ = _run(spec, r0, steps, 100, DL_PLAIN_FP64)
    ref = Lattice(_with_radii(spec, r0), DL_PLAIN_FP64)
    ref.set_group_output(True)
    top = spec.groups["top"]
    R = []
    for _ in range(steps):
        ref.run(1)
        resp, _ = ref.group_sums(top)
        R.append(resp[2])
    e = ref.energies()
    assert J == pytest.approx(e["dissipated"] + REACT_W * max(abs(x) for x in R), rel=1e-9, abs=1e-12)


def test_torch_autograd_wrapper(gpu):
    """impact_objective: the gradient torch back-propagates is the engine's,
    and torch.autograd.gradcheck passes on an elastic lattice (smooth J)."""
    import torch

    from dynlattice_b200.autograd import impact_objective
    spec = _impact(True)
    r = torch.tensor(spec.strut_radius, dtype=torch.float64, requires_grad=True)
    J = impact_objective(r, spec, 200, checkpoint_every=50, react_weight=REACT_W, precision=DL_PLAIN_FP64)
    J.backward()
    J2, g2, _ = _run(spec, spec.strut_radius.copy(), 200, 50, DL_PLAIN_FP64)
    assert float(J.detach()) == pytest.approx(J2, rel=1e-14)
    assert rel_err(r.grad.numpy(), g2) < 1e-14
    el = lattices.lattice_impact("bcc", n=1, velocity=5.0, dt=5e-8, plastic=False, seed=2)
    re = torch.tensor(el.strut_radius, dtype=torch.float64, requires_grad=True)
    f = lambda x: impact_objective(x, el, 150, checkpoint_every=40, react_weight=REACT_W,
                                   precision=DL_PLAIN_FP64) * 1e3
    # central differences with eps = 2e-4 relative to the radius: J is
    # dominated by the peak reaction, to which some struts contribute only
    # 1e-14 of J per unit relative change, so a smaller step would measure
    # J's rounding; truncation stays near 1e-7 of the entries
    assert torch.autograd.gradcheck(f, (re,), eps=1e-7, atol=1e-2, rtol=1e-3)


def _objective_imposed(spec, r, steps, tape, peak_step, peak_sign):
    g = Lattice(_with_radii(spec, r), DL_PLAIN_FP64)
    g.set_branch_mode(2)
    g.set_branch_tape(tape, peak_step, peak_sign)
    J, _ = g.adjoint_radius(steps, 0, elem_param=spec.elem_rod, react_nodes=spec.groups["top"], react_dof=2,
                            react_weight=REACT_W)
    g.synchronize()
    return J


def test_adjoint_is_the_derivative_of_its_branch(gpu):
    """J is piecewise smooth: Gauss points that start or stop yielding, the
    cutting plane's iteration count and the peak step switch branches.  The
    recorded branch (the iteration count of every Gauss point in every step
    and the peak step) is imposed on the finite-difference runs, which then
    differentiate the same function the adjoint does: agreement to 1e-4 at
    the protocol's relative step 1e-6, on an impact that yields."""
    spec = _impact(True, n=3, v=20.0)
    r0 = spec.strut_radius.copy()
    steps = 800
    g = Lattice(_with_radii(spec, r0), DL_PLAIN_FP64)
    g.set_branch_mode(1)
    J, grad = g.adjoint_radius(steps, 100, elem_param=spec.elem_rod, react_nodes=spec.groups["top"], react_dof=2,
                               react_weight=REACT_W)
    g.synchronize()
    tape, peak_step, peak_sign = g.branch_tape()
    assert tape.size == steps * spec.n_gauss * spec.n_elems
    assert (tape > 0).sum() > 100, "the impact must yield"
    assert 1 <= peak_step <= steps and peak_sign in (-1.0, 1.0)
    # the imposed branch reproduces the recorded run's objective
    assert abs(_objective_imposed(spec, r0, steps, tape, peak_step, peak_sign) - J) <= 1e-12 * abs(J)
    rng = np.random.default_rng(5)
    h = 1e-6 * np.abs(r0).mean()
    for _ in range(6):
        d = rng.normal(size=r0.size)
        fd = (_objective_imposed(spec, r0 + h * d, steps, tape, peak_step, peak_sign)
              - _objective_imposed(spec, r0 - h * d, steps, tape, peak_step, peak_sign)) / (2 * h)
        assert abs(grad @ d - fd) <= 1e-4 * abs(fd), (grad @ d, fd)


def test_peak_term_is_the_reaction_magnitude(gpu):
    """max_k |R(k)|: the top face's summed internal force is compressive
    during the impact, and the peak term follows its magnitude."""
    spec = _impact(True, n=2, v=20.0)
    r0 = spec.strut_radius.copy()
    J0, _, _ = _run_w(spec, r0, 300, 0.0)
    J1, _, _ = _run_w(spec, r0, 300, 1.0)
    assert J1 - J0 > 0.0  # a nonzero peak magnitude, whatever R's sign


def _run_w(spec, r, steps, w):
    g = Lattice(_with_radii(spec, r), DL_PLAIN_FP64)
    J, grad = g.adjoint_radius(steps, 0, elem_param=spec.elem_rod, react_nodes=spec.groups["top"], react_dof=2,
                               react_weight=w)
    g.synchronize()
    return J, grad, g
