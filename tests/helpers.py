"""Shared helpers for the parity tests."""
import math

import numpy as np

from turboransac_b200 import scenes


def normalized(f):
    return np.ascontiguousarray(np.stack([(f.uv[:, 0] - f.K[2]) / f.K[0], (f.uv[:, 1] - f.K[3]) / f.K[1]], 1))


def sq_thr(f, px=4.0):
    t = px / (0.5 * (f.K[0] + f.K[1]))
    return t * t


def quat_angle(q1, q2):
    """Rotation angle (rad) between two unit quaternions: 4 asin(|q1 - s q2| / 2), s = sign(q1.q2)."""
    q1 = np.asarray(q1, np.float64) / np.linalg.norm(q1)
    q2 = np.asarray(q2, np.float64) / np.linalg.norm(q2)
    s = 1.0 if float(np.dot(q1, q2)) >= 0 else -1.0
    return 4.0 * math.asin(min(1.0, float(np.linalg.norm(q1 - s * q2)) / 2.0))


def residual_px(P, xn, X, focal):
    """Per-point FP64 reprojection error in pixels for a 3x4 pose (msac.cuh formula)."""
    Z = X @ P[:, :3].T + P[:, 3]
    inv = 1.0 / Z[:, 2]
    r0 = Z[:, 0] * inv - xn[:, 0]
    r1 = Z[:, 1] * inv - xn[:, 1]
    return np.sqrt(r0 * r0 + r1 * r1) * focal, Z[:, 2]


def near_threshold(P, xn, X, focal, px=4.0, band=1e-4):
    r, z = residual_px(P, xn, X, focal)
    return np.abs(r - px) < band


def pose_errors(q, t, f):
    return scenes.pose_error(scenes.quat_to_rotmat(q), np.asarray(t), f.R_gt, f.t_gt)
