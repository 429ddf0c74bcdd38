"""Rod--rod contact in the oracle (CPU): known answers of each branch of the
reference's pair evaluation, the blacklist of pairs closed at t = 0, rigid
plates, and the fibre-network generator."""
import numpy as np
import pytest

import contact_cases as cc
from oracle_ffi import Oracle


def _closed_after(spec, rod, delta):
    """Move one rod by delta (set_state), take one step, return the oracle."""
    o = Oracle(spec)
    o.set_state(u=cc.shift_rod(spec, rod, delta))
    o.run(1)
    return o


def test_cross_sts_force():
    d = 0.02e-3
    spec = cc.cross(gap0=0.05e-3)
    o = _closed_after(spec, 1, (0, 0, -(0.05e-3 + d)))
    pairs, gaps = o.contact_pairs()
    # rod 0: elements 0..3, crossing at x = 0.3 mm -> element 2;
    # rod 1: elements 4..7, crossing at y = 0 -> element 5
    assert pairs.tolist() == [[2, 5]]
    assert gaps[0] == pytest.approx(-d, rel=1e-9)
    # rigid translation: no elastic force, fint = contact force only
    rb, _ = o.group_sums(spec.rod_nodes[1])
    ra, _ = o.group_sums(spec.rod_nodes[0])
    assert rb[2] == pytest.approx(cc.KPEN * (-d), rel=1e-9)
    assert ra[2] == pytest.approx(-cc.KPEN * (-d), rel=1e-9)
    assert abs(rb[0]) + abs(rb[1]) < 1e-12
    assert o.energies()["contact"] == pytest.approx(0.5 * cc.KPEN * d * d, rel=1e-9)


def test_cross_open_gap_no_force():
    spec = cc.cross(gap0=0.05e-3)
    o = _closed_after(spec, 1, (0, 0, -0.04e-3))
    pairs, _ = o.contact_pairs()
    assert pairs.shape[0] == 0
    rb, _ = o.group_sums(spec.rod_nodes[1])
    assert np.abs(rb).max() < 1e-15


def test_tee_node_to_segment():
    d = 0.03e-3
    spec = cc.tee_b_end(gap0=0.05e-3)
    o = _closed_after(spec, 1, (0, 0, -(0.05e-3 + d)))
    pairs, gaps = o.contact_pairs()
    assert pairs.tolist() == [[2, 4]]
    assert gaps[0] == pytest.approx(-d, rel=1e-9)
    rb, _ = o.group_sums(spec.rod_nodes[1])
    assert rb[2] == pytest.approx(cc.KPEN * (-d), rel=1e-9)
    # the force acts on the end node of rod 1 only
    end = int(spec.rod_nodes[1][0])
    rend, _ = o.group_sums(np.array([end]))
    assert rend[2] == pytest.approx(cc.KPEN * (-d), rel=1e-9)


def test_tee_reference_projection_quirk():
    """With the rod order swapped the reference projects node iA of element B
    onto element A (RodContactModel.cpp:575); for a tee that parameter lies
    outside A, so the contact never closes."""
    spec = cc.tee_a_end(gap0=0.05e-3)
    o = _closed_after(spec, 0, (0, 0, -(0.05e-3 + 0.03e-3)))
    pairs, _ = o.contact_pairs()
    assert pairs.shape[0] == 0


def test_parallel_speculative_nts():
    d = 0.01e-3
    spec = cc.parallel()
    gap0 = cc.PZ - 2 * cc.R
    o = _closed_after(spec, 1, (0, 0, -(gap0 + d)))
    pairs, gaps = o.contact_pairs()
    assert pairs.shape[0] > 0
    assert np.allclose(gaps, -d, rtol=1e-6)
    rb, _ = o.group_sums(spec.rod_nodes[1])
    ra, _ = o.group_sums(spec.rod_nodes[0])
    assert rb[2] < 0 and ra[2] == pytest.approx(-rb[2], rel=1e-12)
    # every node-to-segment evaluation closes with the same overlap d
    n_eval = -rb[2] / (cc.KPEN * d)
    assert n_eval == pytest.approx(round(n_eval), abs=1e-6)


def test_blacklist_initial_overlap():
    spec = cc.cross(gap0=-0.02e-3)
    o = Oracle(spec)
    assert o.blacklist_size() == 1
    o.run(5)
    pairs, _ = o.contact_pairs()
    assert pairs.shape[0] == 0


def test_plate_penalty():
    d = 0.01e-3
    spec = cc.rods_spec([((-cc.LEN / 2, 0, 0), (cc.LEN / 2, 0, 0))],
                        plates=[{"normal": (0, 0, 1), "point0": (0, 0, -cc.R + d), "velocity": (0, 0, 0),
                                 "penalty": cc.KPEN}])
    spec.contact.penalty = 0.0      # plates only
    o = Oracle(spec)
    o.run(1)
    react = o.plate_reaction()
    n_nodes = spec.coords.shape[0]
    assert react[0, 2] == pytest.approx(n_nodes * cc.KPEN * (-d), rel=1e-9)
    r, _ = o.group_sums(np.arange(n_nodes))
    assert r[2] == pytest.approx(react[0, 2], rel=1e-12)


def test_moving_plate_time():
    """The plate position at step k uses t_k = k dt."""
    dt = 1e-8
    v = -5.0
    spec = cc.rods_spec([((-cc.LEN / 2, 0, 0), (cc.LEN / 2, 0, 0))], dt=dt,
                        plates=[{"normal": (0, 0, -1), "point0": (0, 0, cc.R), "velocity": (0, 0, v),
                                 "penalty": cc.KPEN}])
    spec.contact.penalty = 0.0
    o = Oracle(spec)
    o.run(3)
    # nodes barely moved in 3 steps: penetration ~ |v| * 3 dt per node
    react = o.plate_reaction()
    n_nodes = spec.coords.shape[0]
    assert react[0, 2] == pytest.approx(n_nodes * cc.KPEN * (-abs(v) * 3 * dt) * -1.0, rel=1e-3)


def test_generator_no_overlap_and_deterministic():
    from dynlattice_b200.lattices import generate_fibres
    n, L, r = 300, 10e-3, 0.1e-3
    box = 50e-3 * (n / 20000) ** (1 / 3)
    c1, conn, erod, tries = generate_fibres(n, L, 4, r, box, seed=7)
    c2, _, _, _ = generate_fibres(n, L, 4, r, box, seed=7)
    c3, _, _, _ = generate_fibres(n, L, 4, r, box, seed=8)
    assert np.array_equal(c1, c2) and not np.array_equal(c1, c3)
    assert tries >= n
    ends = c1.reshape(n, 5, 3)
    seg = np.linalg.norm(ends[:, -1] - ends[:, 0], axis=1)
    assert np.allclose(seg, L, rtol=1e-12)
    centres = 0.5 * (ends[:, 0] + ends[:, -1])
    assert centres.min() >= 0.0 and centres.max() <= box
    # brute-force minimum distance between rods (clamped segments)
    a, b = ends[:, 0], ends[:, -1]
    dmin = np.inf
    for i in range(n):
        p, q = a[i], b[i]
        for j in range(i + 1, n):
            dmin = min(dmin, _seg_dist(p, q, a[j], b[j]))
    assert dmin >= 2 * r
    assert conn.shape == (4 * n, 2) and np.array_equal(erod, np.repeat(np.arange(n), 4))


def _seg_dist(p1, q1, p2, q2):
    d1, d2, r = q1 - p1, q2 - p2, p1 - p2
    a, e, f = d1 @ d1, d2 @ d2, d2 @ r
    c, b = d1 @ r, d1 @ d2
    den = a * e - b * b
    s = np.clip((b * f - c * e) / den, 0, 1) if den > 1e-300 else 0.0
    t = (b * s + f) / e
    if t < 0:
        t, s = 0.0, np.clip(-c / a, 0, 1)
    elif t > 1:
        t, s = 1.0, np.clip((b - c) / a, 0, 1)
    return np.linalg.norm(p1 + d1 * s - p2 - d2 * t)
