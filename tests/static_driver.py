"""Quasi-static equilibrium driver on the oracle (test infrastructure only).

The reference runs its plastic benchmarks (tests/plastic/test1-3) and its
contact benchmark (tests/contact/test1) with JIVE's Nonlin solver: per load
step the prescribed DOFs take their new values, Newton iterations drive the
internal force of the free DOFs to zero with the return map run from the
committed history, and the converged step is committed.  This module restates
that loop around the oracle's force (orc_static_force) and commit
(orc_static_commit), with a finite-difference tangent (column-compressed by a
distance-2 colouring of the element graph when the model has no contact), so
that the oracle's return map and contact force are checked against the
reference's own benchmark data.

Load-step semantics of the BC models (restated from the reference):
  * DirichletModel INCREMENT (dispIncr given): the scale starts at
    initDisp - dispIncr and each ADVANCE adds dispIncr, so step i (1-based)
    prescribes factor * (initDisp + (i - 1) dispIncr)
    (src/models/DirichletModel.cpp:187-194, 312-319, 351);
  * DirichletModel LOADSCALE (neither dispIncr nor dispRate): factor times the
    load scale of the enclosing LoadScale model, scaleFunc evaluated at step i
    (DirichletModel.cpp:103-119, 196-199, 351).
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import Callable, List, Optional, Sequence

import numpy as np


@dataclass
class Prescribed:
    """One prescribed DOF set: value(i) on DOF `dof` of `nodes` at load step i."""
    nodes: Sequence[int]
    dof: int
    value: Callable[[int], float]


def increment(factor: float, disp_incr: float, init_disp: float = 0.0) -> Callable[[int], float]:
    """DirichletModel INCREMENT: factor * (initDisp + (i - 1) dispIncr)."""
    return lambda i: factor * (init_disp + (i - 1) * disp_incr)


def loadscale(factor: float, scale: Callable[[int], float]) -> Callable[[int], float]:
    """DirichletModel LOADSCALE under a LoadScale model: factor * scaleFunc(i)."""
    return lambda i: factor * scale(i)


def jem_if(c, a, b):
    return a if c else b


def node_colouring(conn, n_nodes: int) -> List[np.ndarray]:
    """Greedy distance-2 colouring of the node graph: nodes of one colour share
    no element and no element neighbour, so perturbing all of them at once
    leaves every residual row depending on at most one of them."""
    nbr = [set() for _ in range(n_nodes)]
    for row in conn:
        for a in row:
            nbr[a].update(int(b) for b in row)
    colour = -np.ones(n_nodes, dtype=np.int64)
    for n in range(n_nodes):
        taken = set()
        for a in nbr[n]:
            for b in nbr[a]:
                if colour[b] >= 0:
                    taken.add(int(colour[b]))
        c = 0
        while c in taken:
            c += 1
        colour[n] = c
    return [np.flatnonzero(colour == c) for c in range(int(colour.max()) + 1)]


class StaticDriver:
    """Load-step loop of a Nonlin solver on an oracle model.

    prescribed: list of Prescribed (constant zero values included); every DOF
    not prescribed is solved for.  `coloured` compresses the finite-difference
    tangent (contact couplings must then be listed in `coupling`: rows of
    nodes treated like the nodes of one element).  tangent="trial" differentiates the
    residual itself (return map and contact included: Newton with the
    consistent tangent); "elastic" differentiates the force with the stresses
    taken elastically from the committed plastic strain (the material's
    elastic stiffness: a modified Newton method); "auto" uses the trial
    tangent and falls back to the elastic one where a perturbed state's
    return map fails (maxIter)."""

    def __init__(self, orc, spec, prescribed: List[Prescribed], coloured: bool = True,
                 fd_step: float = 1e-7, length_scale: float = 1.0, tangent: str = "auto", rot_step: float = 1e-5,
                 extrapolate: bool = False, coupling: Optional[np.ndarray] = None):
        self.orc = orc
        self.N = spec.n_nodes
        self.pres = prescribed
        mask = np.zeros((self.N, 6), dtype=bool)
        for p in prescribed:
            mask[np.asarray(p.nodes), p.dof] = True
        self.free = ~mask
        self.free_idx = np.flatnonzero(self.free.ravel())
        self.x = np.zeros((self.N, 6))   # [u | theta]
        self.h_u = fd_step * length_scale
        # rotations: a larger step, since the reference's logMat (acos of the
        # trace) resolves an angle a near identity only to about 1e-16 / a
        self.h_r = rot_step
        self.coloured = coloured
        # node sets whose forces depend on each other: the elements, plus the
        # caller's extra rows (e.g. the four nodes of each element pair that
        # may come into contact)
        rows = [list(r) for r in spec.conn] + ([list(r) for r in coupling] if coupling is not None else [])
        self.colours = node_colouring(rows, self.N) if coloured else [np.array([n]) for n in range(self.N)]
        nbr = [set() for _ in range(self.N)]
        for row in rows:
            for a in row:
                nbr[a].update(int(b) for b in row)
        self.nbr = [np.array(sorted(s)) for s in nbr]
        self.newton_iters = []
        self.residuals = []
        self.tangent = tangent
        # predictor of the free DOFs: the previous step's increment repeated
        self.extrapolate = extrapolate
        self.x_prev = None

    def force(self, x):
        return self.orc.static_force(x[:, :3], x[:, 3:])

    def tangent_force(self, x, elastic=False):
        if elastic:
            return self.orc.internal_force(x[:, :3], x[:, 3:])
        return self.force(x)

    def jacobian(self, x):
        """d fint[free] / d x[free] by central differences (compressed columns)."""
        if self.tangent == "elastic":
            return self._jacobian(x, True)
        try:
            return self._jacobian(x, False)
        except RuntimeError:
            if self.tangent == "trial":
                raise
            return self._jacobian(x, True)

    def _jacobian(self, x, elastic):
        nf = self.free_idx.size
        pos = -np.ones(self.N * 6, dtype=np.int64)
        pos[self.free_idx] = np.arange(nf)
        J = np.zeros((nf, nf))
        for group in self.colours:
            for d in range(6):
                nodes = group[self.free[group, d]]
                if nodes.size == 0:
                    continue
                h = self.h_u if d < 3 else self.h_r
                xp = x.copy(); xp[nodes, d] += h
                xm = x.copy(); xm[nodes, d] -= h
                df = ((self.tangent_force(xp, elastic) - self.tangent_force(xm, elastic)) / (2 * h)).ravel()
                if not self.coloured:
                    J[:, pos[nodes[0] * 6 + d]] = df[self.free_idx]
                    continue
                for n in nodes:
                    rows = (self.nbr[n][:, None] * 6 + np.arange(6)[None, :]).ravel()
                    keep = pos[rows] >= 0
                    J[pos[rows[keep]], pos[n * 6 + d]] = df[rows[keep]]
        return J

    def step(self, i: int, rtol: float = 1e-8, max_newton: int = 40, stall: int = 4, substeps: int = 1) -> int:
        """Load step i: prescribe, Newton to equilibrium, commit.  Returns the
        Newton iterations taken.  The return map stops at f < precision, so
        the residual has a floor of about that precision relative to the
        forces; iterations end at rtol or after `stall` iterations without
        a new lowest residual (the residual reached is kept in `residual`).
        substeps > 1 reaches the step's prescribed values through that many
        intermediate equilibria (a continuation of the solver only: the
        history is committed once, at the end, and every force is evaluated
        from the committed history, so the result does not depend on it)."""
        x_last = self.x.copy()
        if self.extrapolate and self.x_prev is not None:
            self.x.ravel()[self.free_idx] += (self.x - self.x_prev).ravel()[self.free_idx]
        target = self.x.copy()
        for p in self.pres:
            target[np.asarray(p.nodes), p.dof] = p.value(i)
        pmask = ~self.free
        it_total = 0
        for sub in range(1, substeps + 1):
            self.x[pmask] = x_last[pmask] + (target[pmask] - x_last[pmask]) * (sub / substeps)
            it_total += self._newton(rtol, max_newton, stall)
        self.x_prev = x_last
        self.orc.static_commit(self.x[:, :3], self.x[:, 3:])
        self.newton_iters.append(it_total)
        self.residuals.append(self.residual)
        return it_total

    def _newton(self, rtol, max_newton, stall):
        f = self.force(self.x)
        r = f.ravel()[self.free_idx]
        best_x, best = self.x.copy(), np.abs(r).max()
        # residual scale: the first residual or the largest force
        scale = max(best, np.abs(f).max(), 1e-300)
        it = since = 0
        J = None
        while best > rtol * scale and it < max_newton and since < stall:
            if J is None or self.tangent != "elastic":
                J = self.jacobian(self.x)
            dx = np.linalg.lstsq(J, -r, rcond=None)[0]
            # backtracking on the residual norm (the return map makes the
            # force only piecewise smooth)
            lam = 1.0
            x0 = self.x.copy()
            while True:
                xt = x0.copy()
                xt.ravel()[self.free_idx] += lam * dx
                ft = self.force(xt)
                rt = ft.ravel()[self.free_idx]
                if np.abs(rt).max() < best or lam < 1e-3:
                    break
                lam *= 0.5
            self.x, f, r = xt, ft, rt
            it += 1
            since += 1
            if np.abs(r).max() < best:
                best_x, best = self.x.copy(), np.abs(r).max()
                since = 0
        self.x = best_x
        self.residual = best / scale
        return it

    def resp(self, nodes: Sequence[int]) -> np.ndarray:
        """GroupOutput "resp" of a node group: the summed internal force of the
        last committed step (GroupOutputModule.cpp:70-166)."""
        f = self.force(self.x)
        return f[np.asarray(nodes)].sum(axis=0)
