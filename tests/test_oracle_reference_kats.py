"""The oracle against the reference's own golden vectors and known answers.

Everything here runs on the CPU. The reference crate's tests are the pins:
the golden image hash (tests/gpu_parity_tests.rs:294-312), projection
(math/projection.rs:556-740), tile geometry and binning
(render/tiles/mod.rs:248-401, render/tiles/cpu_reference.rs:408-556) and the
compositor (render/rasterizer/cpu_reference.rs:247-358).
"""
import numpy as np
import pytest

import oracle


def identity_cam(fx, fy, cx, cy, w, h, near=0.2):
    cam = np.zeros(24, np.float32)
    cam[[0, 5, 10, 15]] = 1.0
    cam[16:23] = [fx, fy, cx, cy, w, h, near]
    return cam


def test_golden_image_hash():
    scene = oracle.fibonacci_cluster(256, 0.5, [0.0, 0.0, 2.0])
    cam = identity_cam(180, 180, 80, 60, 160, 120)
    img, _, _ = oracle.ref_render_scene(scene, cam, 160, 120, [0.05, 0.05, 0.07, 1.0],
                                        [0, 0, 0], 2)
    assert oracle.pixel_hash(img) == 0xBDD6381531150F06
    again, _, _ = oracle.ref_render_scene(scene, cam, 160, 120, [0.05, 0.05, 0.07, 1.0],
                                          [0, 0, 0], 2)
    assert oracle.pixel_hash(again) == 0xBDD6381531150F06


def test_projection_manual_reference():
    cam = identity_cam(1000, 1000, 500, 400, 1000, 800)
    xy, d, r, c = oracle.ref_project([[0, 0, 2]], [[0.04, 0, 0, 0.04, 0, 0.04]], cam)
    assert d[0] == 2.0 and xy[0].tolist() == [500.0, 400.0]
    assert r[0] == 301
    assert abs(c[0, 0] - 1.0 / 10000.3) < 1e-6 and c[0, 1] == 0.0
    assert abs(c[0, 2] - 1.0 / 10000.3) < 1e-6


def test_near_plane_and_frustum_culling():
    cam = identity_cam(500, 500, 250, 250, 500, 500)
    cov = [[0.01, 0, 0, 0.01, 0, 0.01]] * 4
    _, _, r, _ = oracle.ref_project([[0, 0, 0.1], [0, 0, 0.2], [0, 0, -5.0], [100, 0, 2]], cov, cam)
    assert r.tolist() == [0, 0, 0, 0]


def test_conic_positive_definite():
    cam = identity_cam(800, 800, 400, 300, 800, 600)
    covs = [[0.1, 0.02, 0.01, 0.08, 0.03, 0.15], [1, 0, 0, 1, 0, 1],
            [0.001, 0, 0, 0.001, 0, 0.001]]
    _, _, r, c = oracle.ref_project([[0, 0, 3]] * 3, covs, cam)
    assert (r > 0).all()
    assert (c[:, 0] > 0).all() and (c[:, 2] > 0).all()
    assert (c[:, 0] * c[:, 2] - c[:, 1] ** 2 > 0).all()


def test_radius_clamp_1024():
    cam = identity_cam(1000, 1000, 500, 500, 2000, 2000)
    _, _, r, _ = oracle.ref_project([[0, 0, 1]], [[1000, 0, 0, 1000, 0, 1000]], cam)
    assert r[0] == 1024


def test_binning_single_and_straddling():
    t, d, i, rg = oracle.ref_bin_and_sort([8, 8], [2.5], [2], 800, 600)
    assert t.tolist() == [0] and i.tolist() == [0]
    assert d[0] == np.float32(2.5).view(np.uint32)
    assert rg[0].tolist() == [0, 1] and rg[1].tolist() == [0, 0]
    t, _, _, _ = oracle.ref_bin_and_sort([16, 16], [3.0], [2], 800, 600)
    assert t.tolist() == [0, 1, 50, 51]


def test_binning_culled_and_offscreen():
    for xy, r in (([100, 100], 0), ([100, 100], -5), ([-50, 100], 10), ([900, 100], 10)):
        t, _, _, _ = oracle.ref_bin_and_sort(xy, [1.0], [r], 800, 600)
        assert t.size == 0


def test_binning_lexicographic_order():
    t, d, i, rg = oracle.ref_bin_and_sort([4, 4, 8, 8, 24, 8], [5.0, 1.0, 2.0], [2, 2, 2],
                                          800, 600)
    assert t.tolist() == [0, 0, 1] and i.tolist() == [1, 0, 2]
    assert d.view(np.float32).tolist() == [1.0, 5.0, 2.0]
    assert rg[0].tolist() == [0, 2] and rg[1].tolist() == [2, 3]


def test_binning_ranges_are_total():
    pts = [8, 8, 40, 32, 100, 100, 8, 40, 300, 200]
    radii = [30, 20, 10, 0, 60]
    t, d, i, rg = oracle.ref_bin_and_sort(pts, [1, 2, 3, 4, 5], radii, 800, 600)
    assert t.size > 0
    assert (np.asarray(radii)[i] > 0).all()
    covered = 0
    for tile, (s, e) in enumerate(rg):
        covered += e - s
        assert (t[s:e] == tile).all()
    assert covered == t.size


def _xorshift(seed):
    state = [seed]

    def nxt():
        s = state[0]
        s ^= (s << 13) & 0xFFFFFFFFFFFFFFFF
        s ^= s >> 7
        s ^= (s << 17) & 0xFFFFFFFFFFFFFFFF
        state[0] = s
        return np.float32((s >> 40)) / np.float32(1 << 24)
    return nxt


def test_tight_ellipse_binning_has_no_false_negatives():
    """1000 random ellipses: every tile with a contributing pixel centre is
    reported, and tight binning emits fewer than half of the square-radius
    tiles (render/tiles/mod.rs:302-401, same xorshift sequence)."""
    W, H = 160, 128
    tx_n, ty_n = (W + 15) // 16, (H + 15) // 16
    nxt = _xorshift(0x123456789ABCDEF0)
    square_total = ellipse_total = 0
    px = np.arange(W, dtype=np.float32) + np.float32(0.5)
    py = np.arange(H, dtype=np.float32) + np.float32(0.5)
    for _ in range(1000):
        mu_x = np.float32(-20.0) + nxt() * np.float32(W + 40.0)
        mu_y = np.float32(-20.0) + nxt() * np.float32(H + 40.0)
        ang = nxt() * np.float32(np.pi)
        l1 = np.float32(0.5) + nxt() * np.float32(900.0)
        l2 = np.float32(0.5) + nxt() * np.float32(25.0)
        s, c = np.float32(np.sin(ang)), np.float32(np.cos(ang))
        sxx = c * c * l1 + s * s * l2
        sxy = s * c * (l1 - l2)
        syy = s * s * l1 + c * c * l2
        alpha = np.float32(0.01) + nxt() * np.float32(0.98)
        res = oracle.conic_extents(float(sxx), float(sxy), float(syy), float(alpha))
        if res is None:
            continue
        conic, ext = res
        r_iso = min(max(np.ceil(3.0 * np.sqrt(max(l1, l2) + 0.3)), 1.0), 1024.0)
        _, _, _, rg = oracle.ref_bin_and_sort([mu_x, mu_y], [1.0], [int(r_iso)], W, H)
        square_total += int((rg[:, 1] - rg[:, 0]).sum())
        dx = px[None, :] - mu_x
        dy = py[:, None] - mu_y
        q = np.float32(-0.5) * (conic[0] * dx * dx + np.float32(2.0) * conic[1] * dx * dy +
                                conic[2] * dy * dy)
        hit = (q >= -4.0) & (np.minimum(alpha * np.exp(q), 0.99) >= 1.0 / 255.0)
        x0 = int(np.clip(np.floor((mu_x - ext[0]) / 16), 0, tx_n - 1))
        x1 = int(np.clip(np.floor((mu_x + ext[0]) / 16), 0, tx_n - 1))
        y0 = int(np.clip(np.floor((mu_y - ext[1]) / 16), 0, ty_n - 1))
        y1 = int(np.clip(np.floor((mu_y + ext[1]) / 16), 0, ty_n - 1))
        visible = not (mu_x + ext[0] < 0 or mu_x - ext[0] >= W or mu_y + ext[1] < 0 or
                       mu_y - ext[1] >= H)
        for ty in range(ty_n):
            for tx in range(tx_n):
                pix = hit[ty * 16:(ty + 1) * 16, tx * 16:(tx + 1) * 16].any()
                in_box = visible and x0 <= tx <= x1 and y0 <= ty <= y1
                exact = in_box and oracle.ellipse_tile(float(mu_x), float(mu_y), conic,
                                                       float(alpha), tx, ty, W, H)
                ellipse_total += exact
                assert exact or not pix, (mu_x, mu_y, tx, ty)
    assert ellipse_total * 2 < square_total


def _single_tile(n):
    return np.array([[0, n]], np.uint32)


def test_compositor_half_pixel_centre():
    sh = np.zeros(48, np.float32)
    sh[0] = 1.0
    rgba8, f = oracle.ref_rasterize(16, 16, [0.5, 0.5], [1, 0, 1], [1.0], sh, [0, 0, 2], [0],
                                    _single_tile(1), [0, 0, 0, 1], [0, 0, 0], 0)
    assert f[0, 0, 0] > 0.7


def test_compositor_early_termination():
    sh = np.zeros((5, 48), np.float32)
    sh[0, :3] = [2.0, -2.0, -2.0]
    sh[1:, :3] = [-2.0, 2.0, -2.0]
    rgba8, f = oracle.ref_rasterize(16, 16, [0.5, 0.5] * 5, [1, 0, 1] * 5, [0.99] * 5, sh,
                                    np.zeros(15), np.arange(5), _single_tile(5), [0, 0, 0, 1],
                                    [0, 0, 0], 0)
    assert f[0, 0, 0] > 0.9 and f[0, 0, 1] < 0.1


def test_compositor_ragged_screen_background():
    rg = np.zeros((4, 2), np.uint32)
    rgba8, f = oracle.ref_rasterize(19, 19, [], [], [], np.zeros(0, np.float32), [], [], rg,
                                    [0.1, 0.2, 0.3, 1.0], [0, 0, 0], 0)
    assert f.shape == (19, 19, 4)
    assert abs(f[18, 18, 0] - 0.1) < 1e-5 and abs(f[18, 18, 1] - 0.2) < 1e-5
