"""Float64 evaluation of the frame's formulas on a sample: the error floor of
the f32 pipeline.

The reference computes every stage in f32. Its formulas evaluated in f64 on
the same inputs (rest scene, bindings, cage vertices, camera) give the values
f32 rounding is measured against: deformed means and covariances of sampled
Gaussians (tet-cage Stage 1: x' = sum w_k x_k, J S J^T with the 1e-4
diagonal floor, render/kernels/deformation.rs:874-1060), and composited RGB
of sampled pixels (Stage 1, the EWA projection with inverse-ray SH,
render/kernels/project.rs:1020-1289, and front-to-back blending,
render/kernels/compositor.rs:787-882, all in f64). The compositor's discrete
decisions (which splats a tile lists) come from the f32 frame being judged:
the floor measures rounding, not binning.

Used by bench.py (the `error_floor` entry) and the tests; it reads the
frame's buffers through the public API and needs no oracle.
"""
from __future__ import annotations

import numpy as np

from . import _abi

f64 = np.float64
SH_C0 = 0.28209479177387814
SH_C1 = 0.4886025119029199
SH_C2 = (1.0925484305920792, -1.0925484305920792, 0.31539156525252005, -1.0925484305920792,
         0.5462742152960396)
SH_C3 = (-0.5900435899266435, 2.890611442640554, -0.4570457994644658, 0.3731763325901154,
         -0.4570457994644658, 1.445305721320277, -0.5900435899266435)


def tet_jacobians(verts, elems, inv_dm):
    """J = D_s D_m^-1 per tet [T, 3, 3] (deformation.rs:684-730); D_m^-1 is
    the input the frame uses (column-major [T, 9])."""
    v = np.asarray(verts, f64).reshape(-1, 3)
    e = np.asarray(elems, np.int64).reshape(-1, 4)
    ds = np.stack([v[e[:, 1]] - v[e[:, 0]], v[e[:, 2]] - v[e[:, 0]], v[e[:, 3]] - v[e[:, 0]]],
                  axis=2)  # columns x1-x0, x2-x0, x3-x0
    a = np.asarray(inv_dm, f64).reshape(-1, 3, 3).transpose(0, 2, 1)  # column-major -> [r, c]
    return ds @ a


def polar_rotations(J):
    """The kernel's polar rotation in f64: J scaled to unit |det|, five
    Newton-Schulz steps R <- (R + R^-T) / 2, a reflection fixed by negating
    the last column (deformation.rs:810-865); identity for |det J| < 1e-8."""
    det = np.linalg.det(J)
    small = np.abs(det) < 1e-8
    R = J * np.where(small, 1.0, np.abs(det))[:, None, None] ** (-1.0 / 3.0)
    R[small] = np.eye(3)
    for _ in range(5):
        R = 0.5 * (R + np.linalg.inv(R).transpose(0, 2, 1))
    flip = np.linalg.det(R) < 0
    R[flip, :, 2] *= -1.0
    R[small] = np.eye(3)
    return R


def deform(rest_pos, rest_cov, rest_opa, bind_tet, bind_w, verts, elems, inv_dm):
    """Deformed positions [n, 3], covariances [n, 6] and opacities [n] of the
    given Gaussians in f64 (no strain split, no Mip: the benchmark frame's
    settings); unbound ones keep their rest values."""
    J = tet_jacobians(verts, elems, inv_dm)
    v = np.asarray(verts, f64).reshape(-1, 3)
    e = np.asarray(elems, np.int64).reshape(-1, 4)
    bt = np.asarray(bind_tet, np.int64)
    n = bt.shape[0]
    pos = np.asarray(rest_pos, f64).reshape(n, 3).copy()
    c6 = np.asarray(rest_cov, f64).reshape(n, 6)
    cov = c6.copy()
    opa = np.asarray(rest_opa, f64).copy()
    b = bt < e.shape[0]
    if b.any():
        w = np.asarray(bind_w, f64).reshape(n, 4)[b]
        corners = v[e[bt[b]]]  # [m, 4, 3]
        pos[b] = np.einsum("mk,mkd->md", w, corners)
        cb = c6[b]
        S = np.stack([cb[:, [0, 1, 2]], cb[:, [1, 3, 4]], cb[:, [2, 4, 5]]], axis=1)
        Jb = J[bt[b]]
        M = Jb @ S @ Jb.transpose(0, 2, 1)
        cov[b] = np.stack([np.maximum(M[:, 0, 0], 1e-4), M[:, 0, 1], M[:, 0, 2],
                           np.maximum(M[:, 1, 1], 1e-4), M[:, 1, 2],
                           np.maximum(M[:, 2, 2], 1e-4)], axis=1)
        s_det = np.clip(np.linalg.det(Jb), 0.6, 1.8)
        base = np.clip(1.0 - opa[b], 1e-4, 0.999)
        opa[b] = np.clip(1.0 - base ** (1.0 / s_det), 0.05, 0.99)
    return pos, cov, opa


def eval_sh(c, d, deg):
    """eval_sh_f32 (project.rs:798-895) in f64: c [m, 48], d [m, 3] unit."""
    x, y, z = d[:, 0], d[:, 1], d[:, 2]
    rgb = SH_C0 * c[:, 0:3]
    if deg >= 1:
        basis = [-SH_C1 * y, SH_C1 * z, -SH_C1 * x]
        if deg >= 2:
            xx, yy, zz, xy, yz, xz = x * x, y * y, z * z, x * y, y * z, x * z
            basis += [SH_C2[0] * xy, SH_C2[1] * yz, SH_C2[2] * (2 * zz - xx - yy),
                      SH_C2[3] * xz, SH_C2[4] * (xx - yy)]
            if deg >= 3:
                basis += [SH_C3[0] * y * (3 * xx - yy), SH_C3[1] * xy * z,
                          SH_C3[2] * y * (4 * zz - xx - yy),
                          SH_C3[3] * z * (2 * zz - 3 * xx - 3 * yy),
                          SH_C3[4] * x * (4 * zz - xx - yy), SH_C3[5] * z * (xx - yy),
                          SH_C3[6] * x * (xx - 3 * yy)]
        B = np.stack(basis, axis=1)  # [m, k]
        k = B.shape[1]
        for ch in range(3):
            rgb[:, ch] += np.einsum("mk,mk->m", B, c[:, 3 + 15 * ch:3 + 15 * ch + k])
    return np.clip(rgb + 0.5, 0.0, 1.0)


def project(pos, cov, opa, sh, R, cam24, cam_pos, deg):
    """project_gaussians_v2 (project.rs:1084-1289) in f64 for splats that the
    frame kept: centre, conic, compensated alpha, RGB along R^T d."""
    V = np.asarray(cam24, f64)
    W = V[:16].reshape(4, 4).T  # column-major view -> [r, c]
    fx, fy, cx, cy = V[16:20]
    p = np.asarray(pos, f64)
    t = p @ W[:3, :3].T + W[:3, 3]
    tx, ty, tz = t[:, 0], t[:, 1], t[:, 2]
    c6 = np.asarray(cov, f64)
    S = np.stack([c6[:, [0, 1, 2]], c6[:, [1, 3, 4]], c6[:, [2, 4, 5]]], axis=1)
    C = W[:3, :3] @ S @ W[:3, :3].T
    Jp = np.zeros((p.shape[0], 2, 3))
    Jp[:, 0, 0] = fx / tz
    Jp[:, 0, 2] = -fx * tx / (tz * tz)
    Jp[:, 1, 1] = fy / tz
    Jp[:, 1, 2] = -fy * ty / (tz * tz)
    S2 = Jp @ C @ Jp.transpose(0, 2, 1)
    sxx, sxy, syy = S2[:, 0, 0], S2[:, 0, 1], S2[:, 1, 1]
    raw_det = np.maximum(sxx * syy - sxy * sxy, 0.0)
    px_, py_ = sxx + 0.3, syy + 0.3
    det = px_ * py_ - sxy * sxy
    alpha = np.clip(np.asarray(opa, f64) * np.sqrt(np.clip(raw_det / det, 0.0, 1.0)), 0.0, 1.0)
    conic = np.stack([py_ / det, -sxy / det, px_ / det], axis=1)
    mu = np.stack([fx * tx / tz + cx, fy * ty / tz + cy], axis=1)
    d = p - np.asarray(cam_pos, f64)
    d /= np.maximum(np.linalg.norm(d, axis=1, keepdims=True), 1e-4)
    d = np.einsum("mji,mj->mi", R, d)  # R^T d
    rgb = eval_sh(np.asarray(sh, f64), d, deg)
    return mu, conic, alpha, rgb


def composite_pixels(px, py, ids, mu, conic, alpha, rgb, bg):
    """Front-to-back blending of one tile's list (compositor.rs:787-882) in
    f64 for pixels (px, py); ids index mu/conic/alpha/rgb in list order."""
    pcx, pcy = px + 0.5, py + 0.5
    acc = np.zeros((px.shape[0], 3))
    T = np.ones(px.shape[0])
    live = np.ones(px.shape[0], bool)
    cut = 1.0 / 255.0
    for g in ids:
        if not alpha[g] > cut:
            continue
        dx, dy = pcx - mu[g, 0], pcy - mu[g, 1]
        q = -0.5 * (conic[g, 0] * dx * dx + 2.0 * conic[g, 1] * dx * dy + conic[g, 2] * dy * dy)
        q = np.minimum(q, 0.0)
        a = np.minimum(0.99, alpha[g] * np.exp(q))
        use = live & (q >= -4.0) & (a >= cut)
        w = np.where(use, a * T, 0.0)
        acc += w[:, None] * rgb[g]
        T = np.where(use, T * (1.0 - a), T)
        stop = use & (T < 1e-3)
        T = np.where(stop, 0.0, T)
        live &= ~stop
        if not live.any():
            break
    return np.clip(acc + T[:, None] * np.asarray(bg[:3], f64), 0.0, 1.0)


def frame_floor(st, scene, cages, cam, comp, n_gauss=20_000, n_tiles=16, seed=0):
    """Error floor of the last frame rendered by `st` (f32 RGBA written, 16x16
    tiles, no split/Mip): float64 Stage 1 of `n_gauss` sampled Gaussians and
    float64 Stages 1, 2 and 4 of every pixel of `n_tiles` sampled non-empty
    tiles, against the f32 frame. Returns a dict of error statistics."""
    rng = np.random.default_rng(seed)
    n = scene.count
    g_pos = st.read_buffer(_abi.BUF_DEFORMED_POS, np.float32)
    if g_pos.size != 3 * n:
        raise ValueError("the error floor covers frames without strain splitting")
    g_pos = g_pos.reshape(-1, 3)
    g_cov = st.read_buffer(_abi.BUF_DEFORMED_COV, np.float32).reshape(-1, 6)
    elems, inv, _, bt, bw = cages.flatten()
    verts = cages.flat_vertices()
    idx = rng.choice(n, min(n, n_gauss), replace=False)
    pos64, cov64, _ = deform(scene.positions[idx], scene.covariances_3d[idx],
                             scene.opacities[idx], bt[idx], bw[idx], verts, elems, inv)
    scale = float(np.abs(pos64).max())
    pos_err = np.abs(g_pos[idx].astype(f64) - pos64).max(axis=1) / scale
    cov_rel = np.abs(g_cov[idx].astype(f64) - cov64) / np.maximum(np.abs(cov64), 1e-12)
    diag = cov_rel[:, [0, 3, 5]]

    # RGB: every pixel of sampled tiles, the tiles' lists from the f32 frame
    W, H = comp.screen_width, comp.screen_height
    tiles_x = (W + 15) // 16
    ranges = st.read_buffer(_abi.BUF_TILE_RANGES, np.uint32).reshape(-1, 2)
    ids = st.read_buffer(_abi.BUF_SORTED_IDS, np.uint32)
    img = st.readback_framebuffer_f32(W, H)
    nonempty = np.nonzero(ranges[:, 1] > ranges[:, 0])[0]
    tiles = rng.choice(nonempty, min(len(nonempty), n_tiles), replace=False)
    Rall = polar_rotations(tet_jacobians(verts, elems, inv))
    cam24 = cam.to_array()
    rgb_err = []
    for t in tiles:
        lst = ids[ranges[t, 0]:ranges[t, 1]].astype(np.int64)
        uniq, inv_idx = np.unique(lst, return_inverse=True)
        p64, c64, o64 = deform(scene.positions[uniq], scene.covariances_3d[uniq],
                               scene.opacities[uniq], bt[uniq], bw[uniq], verts, elems, inv)
        tet = bt[uniq].astype(np.int64)
        R = np.where((tet < elems.shape[0])[:, None, None], Rall[np.minimum(tet, len(Rall) - 1)],
                     np.eye(3))
        mu, conic, alpha, rgb = project(p64, c64, o64, scene.sh_coeffs[uniq], R, cam24,
                                        comp.camera_position, comp.sh_degree)
        ty, tx = divmod(int(t), tiles_x)
        yy, xx = np.mgrid[ty * 16:min(ty * 16 + 16, H), tx * 16:min(tx * 16 + 16, W)]
        out = composite_pixels(xx.ravel().astype(f64), yy.ravel().astype(f64), inv_idx, mu,
                               conic, alpha, rgb, comp.background_color)
        got = img[yy.ravel(), xx.ravel(), :3].astype(f64)
        rgb_err.append(np.abs(got - out).max(axis=1))
    rgb_err = np.concatenate(rgb_err) if rgb_err else np.zeros(1)
    return {
        "gaussians_sampled": int(len(idx)),
        "pixels_sampled": int(rgb_err.size),
        "position_max_rel": float(pos_err.max()), "position_mean_rel": float(pos_err.mean()),
        "position_scale": scale,
        "covariance_diag_max_rel": float(diag.max()),
        "covariance_diag_mean_rel": float(diag.mean()),
        "rgb_max_abs": float(rgb_err.max()), "rgb_mean_abs": float(rgb_err.mean()),
        "judge": "f64 evaluation of the same formulas on the same inputs",
    }
