"""Every failure the engine reports, made to happen on the GPU in safe forms:
no fault, no trap, no unbounded wait.  Each status is asserted through the C
ABI (dl_synchronize) and the handle stays usable afterwards.

* DL_ERR_RETURN_MAP: maxIter = 1 on a lattice that yields (the reference's
  JEM_PRECHECK2 "Too many iterations in plasticity loop",
  ElastoPlasticRodMaterial.cpp:234);
* DL_ERR_NONFINITE: a NaN velocity written from the host (dl_set_state);
* DL_ERR_MASS: a node without mass, refused at creation (ExplicitModule.cpp:
  450-453 throws for zero lumped masses);
* DL_ERR_CONTACT: a contact candidate list with a tiny margin and a node
  pushed beyond half of it;
* DL_ERR_TIMEOUT: the grid barrier made to expect one block that never
  arrives (dl_set_barrier_test), with a 2 ms bound: every block's wait runs
  out and the kernel returns.
"""
import copy

import numpy as np
import pytest

import contact_cases as cc
from dynlattice_b200 import lattices
from dynlattice_b200.abi import BC, DL_BC_NEUMANN, DL_MIXED, DL_PLAIN_FP64
from dynlattice_b200.engine import DLError, Lattice

pytestmark = pytest.mark.gpu

DL_ERR_RETURN_MAP, DL_ERR_NONFINITE, DL_ERR_MASS, DL_ERR_TIMEOUT, DL_ERR_CONTACT = 4, 5, 6, 7, 12


def _code(fn):
    with pytest.raises(DLError) as ei:
        fn()
    return ei.value.code


@pytest.mark.parametrize("precision", [DL_PLAIN_FP64, DL_MIXED])
def test_return_map_iteration_limit(gpu, precision):
    spec = lattices.lattice_impact("bcc", n=2, velocity=40.0, dt=5e-8, plastic=True, seed=3)
    spec.materials = [copy.copy(spec.materials[0])]
    spec.materials[0].max_iter = 1
    g = Lattice(spec, precision)
    g.run(400)
    assert _code(g.synchronize) == DL_ERR_RETURN_MAP
    # the same lattice with the default limit runs clean
    ok = Lattice(lattices.lattice_impact("bcc", n=2, velocity=40.0, dt=5e-8, plastic=True, seed=3), precision)
    ok.run(400)
    ok.synchronize()


def test_nonfinite_state(gpu):
    spec = lattices.lattice_impact("bcc", n=2, velocity=10.0, plastic=False)
    g = Lattice(spec, DL_PLAIN_FP64)
    u, th, v = g.state()
    v[3, 1] = np.nan
    g.set_state(u, th, v)
    g.run(2)
    assert _code(g.synchronize) == DL_ERR_NONFINITE
    # cleared and given a finite state, the handle runs again
    g.clear_error()
    v[3, 1] = 0.0
    g.set_state(u, th, v)
    g.run(2)
    g.synchronize()


def test_node_without_mass_is_refused(gpu):
    spec = lattices.lattice_impact("bcc", n=1, velocity=10.0, plastic=False)
    spec.materials = [copy.copy(spec.materials[0])]
    spec.materials[0].density = 0.0
    assert _code(lambda: Lattice(spec, DL_PLAIN_FP64)) == DL_ERR_MASS


def test_stale_contact_list(gpu):
    """A node pushed by a load moves beyond half the candidate list's margin
    (1 nm here) before the list is rebuilt (it was built at rest, so its
    lifetime is unbounded): the step kernel flags it.  The same push, about
    20 nm in 200 steps, stays well inside the default margin (2r)."""
    spec = cc.cross(gap0=0.05e-3)
    spec.contact.margin = 1e-9
    push = np.array([2], np.int32)  # the middle node of rod 0
    spec.bcs = list(spec.bcs) + [BC(DL_BC_NEUMANN, 2, push, 1e-3)]
    g = Lattice(spec, DL_MIXED)
    g.run(200)
    assert _code(g.synchronize) == DL_ERR_CONTACT
    # with a margin that the motion stays inside, the same run is clean
    spec2 = cc.cross(gap0=0.05e-3)
    spec2.bcs = list(spec2.bcs) + [BC(DL_BC_NEUMANN, 2, push, 1e-3)]
    ok = Lattice(spec2, DL_MIXED)
    ok.run(200)
    ok.synchronize()


@pytest.mark.parametrize("precision", [DL_PLAIN_FP64, DL_MIXED])
def test_barrier_wait_runs_out(gpu, precision):
    spec = lattices.lattice_impact("bcc", n=3, velocity=10.0, plastic=False)
    ref = Lattice(spec, precision)
    ref.run(30)
    ref.synchronize()
    g = Lattice(spec, precision)
    g.set_barrier_test(2000, 1)
    g.run(5)
    assert _code(g.synchronize) == DL_ERR_TIMEOUT
    # back to a normal barrier and a clean error word: the handle runs again
    # from the state the aborted launch left (an elastic lattice has no
    # history, and the node phase never ran), and matches the reference run
    g.set_barrier_test(0, 0)
    g.clear_error()
    g.run(30)
    g.synchronize()
    ua, ta, va = g.state()
    ub, tb, vb = ref.state()
    assert np.abs(ua - ub).max() <= 1e-12 * max(np.abs(ub).max(), 1e-30)
    assert np.abs(va - vb).max() <= 1e-12 * max(np.abs(vb).max(), 1e-30)
