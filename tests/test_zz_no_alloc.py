"""dl_internal_force_static: the allocation-free internal force.

Callers that may not allocate device memory when they need the force (a
real-time loop with a fixed memory budget, where a cudaMalloc may synchronise
the device; a host framework that owns every device allocation) use this
entry point; its scratch lives in a static device array.  Its output must equal the ordinary
dl_internal_force on the same configuration, for two calls in a row (the
shared scratch keeps the previous call's contents).  This file is collected
last on purpose.
"""
import ctypes as C

import numpy as np
import pytest

from dynlattice_b200 import lattices
from dynlattice_b200.abi import DL_MIXED, DL_PLAIN_FP64
from dynlattice_b200.engine import Lattice

pytestmark = pytest.mark.gpu


def static_force(g, u, th):
    import torch
    lib = g.lib
    dp = C.POINTER(C.c_double)
    lib.dl_internal_force_static.argtypes = [C.c_void_p, dp, dp, dp]
    ud = torch.from_numpy(np.ascontiguousarray(u)).cuda()
    td = torch.from_numpy(np.ascontiguousarray(th)).cuda()
    fd = torch.full((g.N, 6), float("nan"), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    cast = lambda t: C.cast(C.c_void_p(t.data_ptr()), dp)
    rc = lib.dl_internal_force_static(g.h, cast(ud), cast(td), cast(fd))
    assert rc == 0, lib.dl_last_error().decode()
    g.synchronize()
    return fd.cpu().numpy()


@pytest.mark.parametrize("precision,tol", [(DL_PLAIN_FP64, 1e-9), (DL_MIXED, 1e-5)])
def test_static_scratch_force_matches_internal_force(gpu, precision, tol):
    spec = lattices.lattice_impact(n=3)
    g = Lattice(spec, precision)
    rng = np.random.default_rng(11)
    for call in range(2):
        u = rng.normal(scale=1e-6 * (call + 1), size=(spec.n_nodes, 3))
        th = rng.normal(scale=1e-3 * (call + 1), size=(spec.n_nodes, 3))
        ref = g.internal_force(u, th)
        got = static_force(g, u, th)
        assert np.isfinite(got).all()
        assert np.abs(got - ref).max() <= tol * np.abs(ref).max()


def test_static_scratch_rejects_oversized_lattice(gpu):
    spec = lattices.straight_rod(n_elems=600_000, length=600.0)
    g = Lattice(spec, DL_PLAIN_FP64)
    lib = g.lib
    dp = C.POINTER(C.c_double)
    lib.dl_internal_force_static.argtypes = [C.c_void_p, dp, dp, dp]
    import torch
    z = torch.zeros((g.N, 6), dtype=torch.float64, device="cuda")
    cast = lambda t: C.cast(C.c_void_p(t.data_ptr()), dp)
    rc = lib.dl_internal_force_static(g.h, cast(z), cast(z), cast(z))
    assert rc == 1  # DL_ERR_INVALID
    assert b"too large" in lib.dl_last_error()
