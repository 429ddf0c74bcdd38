"""Shared comparison helpers of the parity tests."""
import numpy as np


def quat_angle_between(th_a, th_b):
    """Geodesic angle between rotations given as rotation vectors (rows)."""
    from scipy.spatial.transform import Rotation as Rot
    ra = Rot.from_rotvec(np.asarray(th_a).reshape(-1, 3))
    rb = Rot.from_rotvec(np.asarray(th_b).reshape(-1, 3))
    return (ra.inv() * rb).magnitude()


def rel_err(a, b, scale=None):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    s = np.abs(b).max() if scale is None else scale
    return float(np.abs(a - b).max() / max(s, 1e-300))
