"""Batched lattices (one launch over many independent lattices of uneven size
and time step) against the oracle run lattice by lattice."""
import numpy as np
import pytest

from dynlattice_b200 import lattices
from dynlattice_b200.abi import DL_MIXED, DL_PLAIN_FP64
from dynlattice_b200.engine import Batch, Lattice
from helpers import quat_angle_between, rel_err
from oracle_ffi import Oracle

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision,tol", [(DL_PLAIN_FP64, 1e-9), (DL_MIXED, 1e-5)])
def test_batch_matches_per_lattice_oracle(gpu, precision, tol):
    specs = lattices.batch_lattices(n_lattices=5, seed=3, n_range=(1, 3))
    assert len({s.dt for s in specs}) > 1, "the batch must mix time steps"
    b = Batch(specs, precision)
    steps = 600
    b.run(steps)
    b.synchronize()
    for k, spec in enumerate(specs):
        o = Oracle(spec, threads=2)
        o.run(steps)
        uo, to, vo = o.state()
        ug, tg, vg = b.lattice_state(k)
        assert rel_err(ug, uo) < tol, spec.name
        ang = quat_angle_between(tg, to)
        # rotation scale: the larger of the largest rotation and the largest
        # displacement over the shortest element (FP32 rounding of the axial
        # forces of an axially loaded lattice leaks into its small rotations)
        d = spec.coords[spec.conn[:, 1]] - spec.coords[spec.conn[:, 0]]
        rot_scale = max(np.abs(to).max(), np.abs(uo).max() / np.sqrt((d * d).sum(1)).min(), 1e-12)
        assert ang.max() <= tol * rot_scale, spec.name
        if precision == DL_PLAIN_FP64:
            assert rel_err(vg, vo) < tol, spec.name
        eo = o.energies()
        eg = b.lattice_energies(k)
        scale = max(abs(eo["kinetic"]), abs(eo["potential"]))
        for key in ("kinetic", "potential", "dissipated"):
            assert abs(eg[key] - eo[key]) <= tol * scale + 1e-300, (spec.name, key)
    assert b.error_word() == 0


def test_batch_equals_separate_lattices(gpu):
    """A lattice evolves identically alone and inside a batch."""
    specs = lattices.batch_lattices(n_lattices=3, seed=5, n_range=(2, 3))
    b = Batch(specs, DL_PLAIN_FP64)
    b.run(300)
    for k, spec in enumerate(specs):
        g = Lattice(spec, DL_PLAIN_FP64)
        g.run(300)
        u1, _, v1 = g.state()
        u2, _, v2 = b.lattice_state(k)
        assert rel_err(u2, u1) < 1e-12 and rel_err(v2, v1) < 1e-12


def test_graph_mode_equals_persistent(gpu):
    """Exec mode 2 (CUDA graph captured for the first block, replayed with
    new arguments for the next ones) steps exactly like the persistent launch,
    for a batch and for a single lattice with a time-dependent load."""
    specs = lattices.batch_lattices(n_lattices=3, seed=7, n_range=(1, 2))
    a = Batch(specs, DL_PLAIN_FP64)
    b = Batch(specs, DL_PLAIN_FP64)
    b.set_exec_mode(2)
    for _ in range(4):
        a.run(50)
        b.run(50)
    b.synchronize()
    for k in range(len(specs)):
        ua, _, va = a.lattice_state(k)
        ub, _, vb = b.lattice_state(k)
        assert rel_err(ub, ua) < 1e-13 and rel_err(vb, va) < 1e-13
    rod = lattices.straight_rod()
    r1, r2 = Lattice(rod), Lattice(rod)
    r2.set_exec_mode(2)
    for n in (100, 100, 100, 37, 100):
        r1.run(n)
        r2.run(n)
    r2.synchronize()
    assert rel_err(r2.state()[0], r1.state()[0]) < 1e-13
    assert r2.energies()["external_work"] == pytest.approx(r1.energies()["external_work"], rel=1e-13)


def test_autotune(gpu):
    specs = lattices.batch_lattices(n_lattices=4, seed=9, n_range=(2, 3))
    b = Batch(specs, DL_MIXED)
    mode, tpb, ms = b.autotune(50)
    assert mode in (0, 1) and tpb in (0, 32, 64, 128, 256) and ms > 0
    ref = Batch(specs, DL_MIXED)
    b.run(100)
    ref.run(100)
    b.synchronize()
    u1, _, _ = b.lattice_state(0)
    u2, _, _ = ref.lattice_state(0)
    assert rel_err(u1, u2) < 1e-6
