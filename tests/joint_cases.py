"""Joint-contact cases (JointContactModel): rods whose end points are the
joints.  The reference's condition for a pair (within 2r now, farther than 2r
apart in the reference configuration) is exercised both ways."""
import numpy as np

from dynlattice_b200 import lattices
from dynlattice_b200.abi import JointContact, Material, ModelSpec

L = 2.0 ** -7     # rod length
RJ = 2.0 ** -10   # joint radius
KJ = 50.0         # joint penalty
GAP = 3 * RJ      # reference gap between the facing tips of rods A and B


def rods_with_joints(rods, elems=4, radius=RJ, penalty=KJ, dt=1e-8, margin=0.0):
    """rods: list of (start[3], end[3]); the joints are the rod ends, in node order."""
    coords, conn, erod, joints = [], [], [], []
    for r, (a, b) in enumerate(rods):
        a, b = np.asarray(a, float), np.asarray(b, float)
        n0 = len(coords)
        for i in range(elems + 1):
            coords.append(a + (b - a) * i / elems)
        for e in range(elems):
            conn.append((n0 + e, n0 + e + 1))
            erod.append(r)
        joints += [n0, n0 + elems]
    mat = Material.circle_section(0.1e-3, young=3e9, poisson_ratio=0.35, density=1200.0)
    spec = ModelSpec(coords=np.array(coords), conn=np.array(conn, np.int32), elem_rod=np.array(erod, np.int32),
                     materials=[mat], n_gauss=2, dt=dt,
                     joint_contact=JointContact(joints=joints, radius=radius, penalty=penalty, margin=margin),
                     name="joint_rods")
    spec.joints = np.array(joints, np.int32)
    spec.rod_nodes = [np.arange(r * (elems + 1), (r + 1) * (elems + 1)) for r in range(len(rods))]
    return spec


def tips():
    """Rod A along x; rod B on the same line, its start GAP (> 2r) after A's
    end; rod C starting RJ (< 2r) beside B's end in the reference
    configuration, so B--C is never a contact."""
    return rods_with_joints([((0, 0, 0), (L, 0, 0)),
                             ((L + GAP, 0, 0), (2 * L + GAP, 0, 0)),
                             ((2 * L + GAP, RJ, 0), (2 * L + GAP, RJ + L, 0))])


def tips_closed_state(spec, shift=(-2 * RJ, 0.3 * RJ, 0.2 * RJ)):
    """Displacements moving rods B and C together by `shift`: A's end and B's
    start come within 2r (a contact); B's end and C's start stay RJ apart
    (no contact: they were close in the reference configuration)."""
    u = np.zeros((spec.n_nodes, 3))
    for r in (1, 2):
        u[spec.rod_nodes[r]] = shift
    return u


def joint_force(spec, u, a, b):
    """-k (2r - d) n on joint a from joint b (internal-force sign), n = (x_b - x_a)/d."""
    x = spec.coords + u[:, :3]
    dvec = x[b] - x[a]
    d = np.linalg.norm(dvec)
    jc = spec.joint_contact
    return -jc.penalty * (2 * jc.radius - d) * dvec / d, d


def fibre_joints(n_rods=300, seed=3, radius=1e-3, penalty=KJ, plates=True):
    """Random fibre network (rod--rod contact, both plates) whose rod ends
    are joints with the given joint radius."""
    spec = lattices.fibre_network(n_rods=n_rods, seed=seed, plate_velocity=5.0)
    if not plates:
        spec.contact.plates = []
    per = spec.n_nodes // n_rods
    joints = np.stack([np.arange(n_rods) * per, np.arange(n_rods) * per + per - 1], axis=1).ravel()
    spec.joint_contact = JointContact(joints=joints.astype(np.int32), radius=radius, penalty=penalty)
    spec.joints = joints.astype(np.int32)
    return spec


def brute_pairs(spec, u):
    """All joint pairs the reference's findContacts_ selects at displacements u."""
    J = spec.joints
    X = spec.coords[J]
    x = X + u[J, :3]
    r2 = 2 * spec.joint_contact.radius
    out = []
    for i in range(len(J)):
        d = np.linalg.norm(x[i + 1:] - x[i], axis=1)
        d0 = np.linalg.norm(X[i + 1:] - X[i], axis=1)
        for k in np.nonzero((d <= r2) & (d0 > r2))[0]:
            a, b = int(J[i]), int(J[i + 1 + k])
            out.append((min(a, b), max(a, b)))
    return sorted(out)
