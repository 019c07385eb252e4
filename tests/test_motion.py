"""Host-side geometry of the differentiation form (jenhine_b200/motion.py), on
the CPU: M(theta) is a rigid motion, P(0) = P0, and dP/dtheta matches FP64
central differences of P0 M(theta)."""
import numpy as np

from jenhine_b200.motion import moved_ptms, ptm_derivatives, rigid, seeded_motion
from jenhine_b200.phantom import ScanGeometry


def test_rigid_motion_is_a_rotation_and_a_shift():
    for th in seeded_motion(20, 5, shift_mm=3.0, rot_deg=20.0):
        M, _ = rigid(th)
        R = M[:3, :3]
        np.testing.assert_allclose(R @ R.T, np.eye(3), atol=1e-14)
        assert abs(np.linalg.det(R) - 1.0) < 1e-14
        np.testing.assert_array_equal(M[:3, 3], th[:3])
        np.testing.assert_array_equal(M[3], [0.0, 0.0, 0.0, 1.0])


def test_zero_motion_keeps_the_matrices():
    P0 = ScanGeometry(6, 500.0, 800.0, 40, 30, 2.0, 2.0, seed=1).ptms_f64()
    np.testing.assert_allclose(moved_ptms(P0, np.zeros((6, 6))), P0, rtol=0, atol=1e-12)


def test_derivatives_match_central_differences():
    g = ScanGeometry(5, 500.0, 800.0, 40, 30, 2.0, 2.0, flex_shift_px=0.5, gantry_tilt_deg=5.0, seed=2)
    P0 = g.ptms_f64()
    th = seeded_motion(5, 9, shift_mm=2.0, rot_deg=5.0)
    d = ptm_derivatives(P0, th)
    assert d.shape == (5, 6, 12)
    h = 1e-5
    for j in range(6):
        e = np.zeros_like(th)
        e[:, j] = h
        fd = (moved_ptms(P0, th + e) - moved_ptms(P0, th - e)) / (2 * h)
        scale = np.abs(fd).max()
        np.testing.assert_allclose(d[:, j], fd, rtol=0, atol=1e-7 * max(scale, 1.0))
