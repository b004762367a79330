"""The oracle's ShRotator restatement against the reference's own SH-rotation
tests (render/rasterizer/sh_rotation.rs:474-576): orthogonal band matrices,
rotated coefficients evaluated along d equal the rest coefficients evaluated
along R^T d, identity is a no-op, degree 0 is untouched."""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.filterwarnings("ignore::RuntimeWarning")


def axis_angle(axis, angle):
    """Rotation matrix (rows = output axes) about `axis` by `angle` (Rodrigues)."""
    a = np.asarray(axis, np.float64)
    a = a / np.linalg.norm(a)
    K = np.array([[0, -a[2], a[1]], [a[2], 0, -a[0]], [-a[1], a[0], 0]])
    return (np.eye(3) + np.sin(angle) * K + (1 - np.cos(angle)) * K @ K).astype(np.float32)


def rot_x(t):
    return axis_angle([1, 0, 0], t)


def rot_y(t):
    return axis_angle([0, 1, 0], t)


def rot_z(t):
    return axis_angle([0, 0, 1], t)


def col_major(R):
    """Column-major 9 floats of a row-indexed 3x3 matrix."""
    return np.ascontiguousarray(np.asarray(R, np.float32).T).ravel()


def sh_bands(d):
    """Real SH bands 1..3 of unit direction d, in the order of evaluate_sh
    (render/rasterizer/sh.rs:29-137), float64."""
    x, y, z = (float(v) for v in d)
    xx, yy, zz = x * x, y * y, z * z
    b1 = [-0.4886025119029199 * y, 0.4886025119029199 * z, -0.4886025119029199 * x]
    b2 = [1.0925484305920792 * x * y, -1.0925484305920792 * y * z,
          0.31539156525252005 * (2 * zz - xx - yy), -1.0925484305920792 * x * z,
          0.5462742152960396 * (xx - yy)]
    b3 = [-0.5900435899266435 * y * (3 * xx - yy), 2.890611442640554 * x * y * z,
          -0.4570457994644658 * y * (4 * zz - xx - yy),
          0.3731763325901154 * z * (2 * zz - 3 * xx - 3 * yy),
          -0.4570457994644658 * x * (4 * zz - xx - yy), 1.445305721320277 * z * (xx - yy),
          -0.5900435899266435 * x * (xx - 3 * yy)]
    return [np.array(b1), np.array(b2), np.array(b3)]


def sh_value(c48, d, degree):
    """Per channel: sum over bands 1..degree of c . Y_l(d) (DC left out)."""
    bands = sh_bands(d)
    out = np.zeros(3)
    starts = [0, 3, 8]
    for ch in range(3):
        rest = np.asarray(c48[3 + 15 * ch: 18 + 15 * ch], np.float64)
        for l in range(1, degree + 1):
            out[ch] += rest[starts[l - 1]: starts[l - 1] + 2 * l + 1] @ bands[l - 1]
    return out


ROTATIONS = [np.eye(3, dtype=np.float32), rot_y(0.4), rot_x(-0.9) @ rot_z(0.25),
             axis_angle([-1.0, 0.4, 0.8], 2.1)]
DIRS = [np.array([0.0, 0.0, 1.0]), np.array([0.3, -0.5, 0.81]), np.array([-0.7, 0.2, -0.68])]


def test_rotation_matrices_are_orthogonal():
    R = axis_angle([0.3, 1.0, -0.2], 0.7)
    for band in (1, 2, 3):
        M = oracle.sh_rotation_matrix(col_major(R), band).astype(np.float64)
        assert M.shape == (2 * band + 1,) * 2
        assert np.abs(M @ M.T - np.eye(2 * band + 1)).max() < 1e-6


def test_rotated_coefficients_match_the_rotated_direction():
    sh = np.zeros(48, np.float32)
    for c in range(3):
        for k in range(15):
            sh[3 + 15 * c + k] = np.sin((c + 1.0) * (k + 1.0) * 0.13) * 0.8
        sh[c] = 0.2 * (c + 1)
    for R in ROTATIONS:
        for degree in (1, 2, 3):
            rotated = oracle.ref_sh_rotate(sh, col_major(R), degree)
            np.testing.assert_array_equal(rotated[:3], sh[:3])
            for d in DIRS:
                d = d / np.linalg.norm(d)
                expected = sh_value(sh, R.astype(np.float64).T @ d, degree)
                actual = sh_value(rotated, d, degree)
                # The reference bounds this by 2e-3 on clamped colours; the
                # f32 matrices and f32 sums keep it near 1e-6.
                assert np.abs(actual - expected).max() < 1e-5, (degree, R, d)


def test_identity_is_a_no_op_and_degree_zero_untouched():
    sh = np.sin(np.arange(48, dtype=np.float32) * np.float32(0.37)).astype(np.float32)
    out = oracle.ref_sh_rotate(sh, col_major(np.eye(3)), 3)
    assert np.abs(out - sh).max() < 1e-6
    sh0 = np.zeros(48, np.float32)
    sh0[0], sh0[45] = 1.5, 0.25
    np.testing.assert_array_equal(oracle.ref_sh_rotate(sh0, col_major(rot_z(1.0)), 0), sh0)


def test_band_one_matrix_is_the_permuted_rotation():
    """Band 1 is (-y, z, -x) up to a constant: its matrix is R^T rearranged."""
    R = axis_angle([0.2, -0.7, 0.4], 1.3).astype(np.float64)
    M = oracle.sh_rotation_matrix(col_major(R), 1).astype(np.float64)
    # Y1(d) = C P d with P = [[0,-1,0],[0,0,1],[-1,0,0]]; Y1(R^T d) = P R^T P^-1 Y1(d)
    # and c' = D^T c, so M = D^T = (P R^T P^T)^T = P R P^T.
    P = np.array([[0, -1, 0], [0, 0, 1], [-1, 0, 0]], np.float64)
    np.testing.assert_allclose(M, P @ R @ P.T, atol=2e-7)


def test_higher_coefficients_above_the_degree_are_left_alone():
    rng = np.random.default_rng(3)
    sh = rng.normal(size=(5, 48)).astype(np.float32)
    R = col_major(axis_angle([1.0, 2.0, 0.5], -0.8))
    out = oracle.ref_sh_rotate(sh, R, 1).reshape(5, 48)
    for ch in range(3):
        base = 3 + 15 * ch
        np.testing.assert_array_equal(out[:, base + 3: base + 15], sh[:, base + 3: base + 15])
        assert not np.array_equal(out[:, base: base + 3], sh[:, base: base + 3])
