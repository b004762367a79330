"""QuantizedGaussianSceneSoa (scene/soa.rs:429-608) on the host: the packing
order, degree trimming, the reference's round-trip test (soa.rs:615-645:
covariance and SH within 2e-3 after quantising, compression ratios) and the
ingest path's decode, which the GPU test compares frame by frame."""
import numpy as np

from cindergs_b200.scene import (GaussianSceneSoa, QuantizedGaussianSceneSoa, activate_opacity,
                                 activate_rotation, activate_scale, compute_covariance_3d,
                                 pack_f16_pairs, random_scene, sh_packed_words_for_degree,
                                 unpack_f16_pairs)

f32 = np.float32


def test_pair_order_and_rounding():
    w = pack_f16_pairs(np.array([1.0], f32), np.array([-2.0], f32))
    assert int(w[0]) == 0x3C00 | (0xC000 << 16)
    # 1 + 2^-11 is halfway between f16 neighbours 1 and 1 + 2^-10: ties to even
    w = pack_f16_pairs(np.array([1.0 + 2.0 ** -11], f32), np.array([1.0 + 3 * 2.0 ** -11], f32))
    lo, hi = unpack_f16_pairs(w)
    assert lo[0] == 1.0 and hi[0] == 1.0 + 2.0 ** -9
    assert [sh_packed_words_for_degree(d) for d in range(4)] == [2, 6, 14, 24]


def one_vertex_scene():
    """The reference test's vertex: position, opacity logit, log-scales,
    rotation (w, x, y, z), DC and three higher-order coefficients."""
    scale = activate_scale(np.array([[-1.2, -1.8, -0.9]], f32))
    q = activate_rotation(np.array([[0.8, 0.3, -0.2, 0.4]], f32))
    cov = compute_covariance_3d(scale, q)
    sh = np.zeros((1, 48), f32)
    sh[0, 0:3] = [0.4, -0.2, 0.6]
    sh[0, 3] = 0.15
    sh[0, 18] = -0.12
    sh[0, 33] = 0.08
    return GaussianSceneSoa(np.array([[0.5, -0.25, 1.5]], f32), cov.astype(f32),
                            activate_opacity(np.array([1.2], f32)), sh)


def test_reference_round_trip():
    s = one_vertex_scene()
    q3 = QuantizedGaussianSceneSoa.from_soa(s)
    r = q3.to_soa()
    assert np.abs(r.covariances_3d - s.covariances_3d).max() < 2e-3
    assert np.abs(r.sh_coeffs - s.sh_coeffs).max() < 2e-3
    # bytes per splat: f32 scene 12 + 24 + 4 + 192; quantised 12 + 12 + 4 + 4 per SH word
    # (plus the reference's 4-byte rotation word, counted here as in its ratio)
    full = 12 + 24 + 4 + 192
    ratio = lambda d: full / (12 + 12 + 4 + 4 + 4 * sh_packed_words_for_degree(d))
    assert ratio(3) > 1.8 and ratio(2) > 2.5


def test_degree_trimming():
    s = random_scene(500, seed=3)
    for d in range(4):
        q = QuantizedGaussianSceneSoa.from_soa(s, d)
        assert q.sh_coeffs_f16_packed.shape == (500, sh_packed_words_for_degree(d))
        sh = q.unpack_sh_48()
        rest = (d + 1) ** 2 - 1
        for base in (3, 18, 33):
            assert np.all(sh[:, base + rest:base + 15] == 0.0)
            np.testing.assert_array_equal(sh[:, base:base + rest],
                                          s.sh_coeffs[:, base:base + rest].astype(np.float16).astype(f32))
        np.testing.assert_array_equal(sh[:, :3], s.sh_coeffs[:, :3].astype(np.float16).astype(f32))
