"""Rigid motion of the object per view, composed into projection matrices.

theta = (tx, ty, tz, rx, ry, rz): a translation in mm and rotations in degrees
about the volume's x, y, z axes.  A voxel at X in the reconstruction frame
sits at M(theta) X = R X + t during the view, R = Rz Ry Rx, so the view's
projection matrix becomes P(theta) = P0 M(theta).  Composition and the
derivatives dP/dtheta_j are computed in FP64 on the host.
"""
from __future__ import annotations

import numpy as np

_DEG = np.pi / 180.0


def _rot(axis: int, a: float):
    c, s = np.cos(a), np.sin(a)
    r, dr = np.eye(3), np.zeros((3, 3))
    i, j = [(1, 2), (0, 2), (0, 1)][axis]
    sign = -1.0 if axis == 1 else 1.0   # y: [[c, 0, s], [0, 1, 0], [-s, 0, c]]
    r[i, i], r[j, j], r[i, j], r[j, i] = c, c, -sign * s, sign * s
    dr[i, i], dr[j, j], dr[i, j], dr[j, i] = -s, -s, -sign * c, sign * c
    return r, dr


def rigid(theta) -> tuple[np.ndarray, np.ndarray]:
    """M(theta) (4 x 4) and dM/dtheta_j (6 x 4 x 4), FP64."""
    t = np.asarray(theta, np.float64)
    rx, drx = _rot(0, t[3] * _DEG)
    ry, dry = _rot(1, t[4] * _DEG)
    rz, drz = _rot(2, t[5] * _DEG)
    M = np.eye(4)
    M[:3, :3] = rz @ ry @ rx
    M[:3, 3] = t[:3]
    dM = np.zeros((6, 4, 4))
    for j in range(3):
        dM[j, j, 3] = 1.0
    dM[3, :3, :3] = rz @ ry @ drx * _DEG
    dM[4, :3, :3] = rz @ dry @ rx * _DEG
    dM[5, :3, :3] = drz @ ry @ rx * _DEG
    return M, dM


def moved_ptms(P0, theta) -> np.ndarray:
    """P0 M(theta_v) per view: (n, 12) FP64."""
    P0 = np.asarray(P0, np.float64).reshape(-1, 3, 4)
    th = np.asarray(theta, np.float64).reshape(-1, 6)
    return np.stack([P0[v] @ rigid(th[v])[0] for v in range(len(P0))]).reshape(-1, 12)


def ptm_derivatives(P0, theta) -> np.ndarray:
    """dP/dtheta_j = P0 dM/dtheta_j per view: (n, 6, 12) FP64."""
    P0 = np.asarray(P0, np.float64).reshape(-1, 3, 4)
    th = np.asarray(theta, np.float64).reshape(-1, 6)
    return np.stack([np.einsum("ik,jkl->jil", P0[v], rigid(th[v])[1]).reshape(6, 12) for v in range(len(P0))])


def seeded_motion(n_views: int, seed: int, shift_mm: float = 0.5, rot_deg: float = 0.3) -> np.ndarray:
    """(n, 6) motion, uniform in +/- shift_mm and +/- rot_deg."""
    rng = np.random.default_rng(seed)
    th = np.empty((n_views, 6))
    th[:, :3] = rng.uniform(-shift_mm, shift_mm, (n_views, 3))
    th[:, 3:] = rng.uniform(-rot_deg, rot_deg, (n_views, 3))
    return th
