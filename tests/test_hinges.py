"""Rigid hinges (HingeModel, "rigidHinge") in an explicit run, in the oracle.

HingeModel::createHinges_ (HingeModel.cpp:268-358) splits every node of a
rod and ties each copy to its original through constraints
(HingeModel.cpp:172-199) whose plastic offset changes only in CHECK_COMMIT,
which the explicit modules never issue: in an explicit run each tie is rigid,
and the consistent solve condenses it, so a tie group moves as one node with
the summed mass and forces of its members.  A hinged lattice then follows the
same trajectory as the unhinged one (to rounding: the sums are ordered
differently), which is what these tests check; the GPU engine against this
oracle is in tests/test_gpu_hinges.py."""
import numpy as np
import pytest

from dynlattice_b200 import lattices
from helpers import rel_err
from oracle_ffi import Oracle


def test_hinge_creation_splits_every_rod_node():
    spec = lattices.lattice_impact("bcc", n=1, velocity=10.0, plastic=False)
    h = lattices.with_hinges(spec)
    n_rods = np.unique(spec.elem_rod).size
    assert h.n_nodes == spec.n_nodes + spec.n_elems + n_rods
    assert h.ties.shape == (spec.n_elems + n_rods, 2)
    # every element owns its nodes now, apart from the originals it kept
    assert np.array_equal(h.coords[h.ties[:, 0]], h.coords[h.ties[:, 1]])
    assert set(h.ties[:, 1]) == set(range(spec.n_nodes, h.n_nodes))


@pytest.mark.parametrize("plastic", [False, True])
def test_hinged_lattice_follows_the_unhinged_one(plastic):
    spec = lattices.lattice_impact("bcc", n=2, velocity=20.0, dt=5e-8, plastic=plastic, seed=2)
    hinged = lattices.with_hinges(spec)
    a, b = Oracle(spec, threads=4), Oracle(hinged, threads=4)
    a.run(400)
    b.run(400)
    ua, ta, va = a.state()
    ub, tb, vb = b.state()
    N = spec.n_nodes
    assert rel_err(ub[:N], ua) < 1e-10
    assert rel_err(vb[:N], va) < 1e-9
    # the slaves move with their masters
    m, s = hinged.ties[:, 0], hinged.ties[:, 1]
    assert np.array_equal(ub[s], ub[m]) and np.array_equal(vb[s], vb[m])
    ea, eb = a.energies(), b.energies()
    for k in ("kinetic", "potential", "dissipated"):
        assert eb[k] == pytest.approx(ea[k], rel=1e-9, abs=1e-300), k
    if plastic:
        assert ea["dissipated"] > 0.0


def test_ties_are_validated():
    spec = lattices.lattice_impact("bcc", n=1, velocity=10.0, plastic=False)
    h = lattices.with_hinges(spec)
    bad = h.ties.copy()
    bad[1, 1] = bad[0, 1]  # one slave, two masters
    h.ties = bad
    with pytest.raises(RuntimeError):
        Oracle(h)
