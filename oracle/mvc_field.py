"""CPU oracle for the learned MVC weight field -- test infrastructure only.

A float64 numpy restatement of the network the GPU kernels evaluate and train
(Fourier features -> 4 x 128 SiLU -> V outputs, partition of unity by
w0 = z + (1 - sum z) / V, then the linear-precision projection
w = w0 - Vb^T M (Vb w0 - [1; x]) with Vb = [1; rest vertices] and
M = (Vb Vb^T)^-1), rounding to bf16 exactly where the kernels store
bf16: the features, each layer's SiLU output, the weights used by the matrix
products, and (in the backward pass) dL/dz and dL/dpre before they enter a
product. Only the tests use this module.

The field has no counterpart in the reference; what it must reproduce is the
exact mean value coordinates (deformation/mvc.rs:366-471, restated in
cgs_oracle.cpp and pinned by the reference's MVC tests, mvc.rs:802-907).

Parameter block layout (offsets from ``cgs_mvc_field_layout``): W1 [128 x 64],
b1, W2, b2, W3, b3 [128 x 128 / 128], W4, b4, W5 [V x 128], b5 [V], row-major
out x in.
"""
from __future__ import annotations

import numpy as np

BANDS = 8
N_IN = 64
HID = 128
NAMES = ["W1", "b1", "W2", "b2", "W3", "b3", "W4", "b4", "W5", "b5"]


def bf16(a) -> np.ndarray:
    """Round to the nearest bf16 (ties to even) via float32, as
    __float2bfloat16_rn does on a float32 value; returned as float64."""
    f = np.asarray(a, np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def unpack(params: np.ndarray, offsets: dict, V: int) -> dict:
    shapes = {"W1": (HID, N_IN), "b1": (HID,), "W2": (HID, HID), "b2": (HID,),
              "W3": (HID, HID), "b3": (HID,), "W4": (HID, HID), "b4": (HID,),
              "W5": (V, HID), "b5": (V,)}
    out = {}
    for k, shp in shapes.items():
        n = int(np.prod(shp))
        out[k] = np.asarray(params[offsets[k]:offsets[k] + n], np.float64).reshape(shp)
    return out


# The kernels form x^ = (x - c) * (1/s), the band argument w_b * x^ and the
# derivative (w_b * cos) * (1/s) in float32 before rounding to bf16; the high
# bands turn float32-vs-float64 differences into different bf16 roundings,
# so the oracle forms them in float32 too (switched off for derivative checks).
EMULATE_F32 = True


def features(x: np.ndarray, enc: np.ndarray):
    """Features [n, 64] and their x-derivatives [n, 64, 3]: x^ = (x - c) / s,
    then sin and cos of 2^b (pi/2) x^_d for b = 0..7, d = 0..2, zero-padded."""
    n = np.asarray(x).reshape(-1, 3).shape[0]
    f = np.zeros((n, N_IN))
    df = np.zeros((n, N_IN, 3))
    if EMULATE_F32:
        x32 = np.asarray(x, np.float32).reshape(-1, 3)
        e32 = np.asarray(enc, np.float32)
        xh = ((x32 - e32[:3]) * e32[3]).astype(np.float32)
        inv_s = e32[3]
        rnd = np.float32
    else:
        inv_s = float(enc[3])
        xh = (np.asarray(x, np.float64).reshape(-1, 3) - np.asarray(enc[:3], np.float64)) * inv_s
        rnd = np.float64
    f[:, :3] = xh
    for d in range(3):
        df[:, d, d] = inv_s
    for b in range(BANDS):
        w = rnd(2.0 ** b) * rnd(np.pi / 2.0)
        for d in range(3):
            j = 3 + 6 * b + 2 * d
            arg = (w * xh[:, d]).astype(rnd).astype(np.float64)
            sn, cs = rnd(np.sin(arg)), rnd(np.cos(arg))
            f[:, j], f[:, j + 1] = sn, cs
            df[:, j, d] = (w * cs).astype(rnd) * inv_s
            df[:, j + 1, d] = (-w * sn).astype(rnd) * inv_s
    return f, df


def _silu(x):
    return x / (1.0 + np.exp(-x))


def _silu_grad(x):
    s = 1.0 / (1.0 + np.exp(-x))
    return s * (1.0 + x * (1.0 - s))


def forward(P: dict, x: np.ndarray, enc: np.ndarray):
    """(z [n, V], cache) as the training kernels compute it."""
    f, _ = features(x, enc)
    a = [bf16(f)]
    pre = []
    for l in range(1, 5):
        p = a[-1] @ bf16(P[f"W{l}"]).T + P[f"b{l}"]
        pre.append(p)
        a.append(bf16(_silu(p)))
    z = a[-1] @ bf16(P["W5"]).T + P["b5"]
    return z, (a, pre)


def pou(z: np.ndarray) -> np.ndarray:
    V = z.shape[1]
    return z + (1.0 - z.sum(axis=1, keepdims=True)) / V


def lp_matrix(rest_verts: np.ndarray) -> np.ndarray:
    """M = (Vb Vb^T)^-1 for Vb = [1; v_j] (4 x V), rounded to float32 as the
    kernels receive it."""
    v = np.asarray(rest_verts, np.float32).astype(np.float64)
    Vb = np.concatenate([np.ones((1, len(v))), v.T], 0)
    return np.linalg.inv(Vb @ Vb.T).astype(np.float32).astype(np.float64)


def project(w0: np.ndarray, x: np.ndarray, rest_verts: np.ndarray, M: np.ndarray):
    """(w, r): the linear-precision projection of w0 and the residual
    r = sum_j w0_j v_j - x of w0."""
    v = np.asarray(rest_verts, np.float64)
    r = w0 @ v - np.asarray(x, np.float64)
    u = r @ M[:, 1:4].T                       # [n, 4]
    return w0 - (u[:, :1] + u[:, 1:] @ v.T), r


def loss_and_grads(P: dict, x: np.ndarray, wt: np.ndarray, rest_verts: np.ndarray,
                   enc: np.ndarray, lam: float):
    """Loss terms (weight, residual without lambda) and gradients of
    L = (1/B) sum_b sum_j (w - w*)^2 + lam (1/B) sum_b |r|^2 / (3 s^2)."""
    x = np.asarray(x, np.float64).reshape(-1, 3)
    B = x.shape[0]
    s2 = (1.0 / float(np.float32(enc[3]))) ** 2
    vr = np.asarray(rest_verts, np.float64)
    M = lp_matrix(rest_verts)
    z, (a, pre) = forward(P, x, enc)
    w, r = project(pou(z), x, vr, M)
    e = w - np.asarray(wt, np.float64)
    l_w = float((e * e).sum() / B)
    l_r = float((r * r).sum() / (3.0 * B * s2))
    g = 2.0 * e / B
    Vg = np.concatenate([g.sum(1, keepdims=True), g @ vr], 1)   # [B, 4] = (Vb g)^T
    q = Vg @ M.T
    g0 = g - (q[:, :1] + q[:, 1:] @ vr.T) + lam * 2.0 / (3.0 * B * s2) * (r @ vr.T)
    dz = g0 - g0.mean(axis=1, keepdims=True)
    grads = {"W5": bf16(dz).T @ a[4], "b5": dz.sum(axis=0)}
    dh = bf16(dz) @ bf16(P["W5"])
    for l in range(4, 0, -1):
        dp = dh * _silu_grad(pre[l - 1])
        grads[f"W{l}"] = bf16(dp).T @ a[l - 1]
        grads[f"b{l}"] = dp.sum(axis=0)
        if l > 1:
            dh = bf16(dp) @ bf16(P[f"W{l}"])
    return (l_w, l_r), grads


def _folded(W5: np.ndarray, b5: np.ndarray, verts: np.ndarray):
    """(P_u [128, 3], p0_u) with sum_j w0_j u_j = h @ P_u + p0_u."""
    u = np.asarray(verts, np.float64)
    ub = u.mean(axis=0)
    c = W5.sum(axis=0)
    return W5.T @ u - np.outer(c, ub), b5 @ u + (1.0 - b5.sum()) * ub


def position_and_jacobian(P: dict, x: np.ndarray, verts, enc: np.ndarray,
                          rest_verts: np.ndarray):
    """Fused inference: positions [n, 3] and gradients F [n, 3, 3]
    (F[:, :, k] = d x' / d x_k) of the projected weights on cage vertices
    `verts`, or (verts None) the network's own rest position sum_j w0_j v_j.
    h and dh/dx are rounded to bf16 before the folded output layer (bf16 W5,
    fp32 b5), as the kernel does."""
    x = np.asarray(x, np.float64).reshape(-1, 3)
    f, df = features(x, enc)
    h = bf16(f)                                     # [n, 64]
    t = bf16(np.transpose(df, (0, 2, 1)))           # [n, 3, 64]
    for l in range(1, 5):
        W = bf16(P[f"W{l}"])
        p = h @ W.T + P[f"b{l}"]
        dp = t @ W.T                                 # [n, 3, 128]
        slope = _silu_grad(p)
        h, t = bf16(_silu(p)), bf16(dp * slope[:, None, :])
    W5 = bf16(P["W5"])
    Pr, p0r = _folded(W5, P["b5"], rest_verts)
    yr = h @ Pr + p0r
    Fr = np.einsum("nkh,hc->nck", t, Pr)
    if verts is None:
        return yr, Fr
    Pc, p0c = _folded(W5, P["b5"], verts)
    vr = np.asarray(rest_verts, np.float64)
    vc = np.asarray(verts, np.float64)
    S = np.concatenate([vc.sum(0)[:, None], vc.T @ vr], 1)    # [3, 4] = v'^T Vb^T
    A3 = (S @ lp_matrix(rest_verts))[:, 1:]
    pos = h @ Pc + p0c - (yr - x) @ A3.T
    F = np.einsum("nkh,hc->nck", t, Pc) - np.einsum("ndk,cd->nck", Fr, A3) + A3[None]
    return pos, F


def weights(P: dict, x: np.ndarray, enc: np.ndarray, rest_verts: np.ndarray) -> np.ndarray:
    """Final (projected) weights [n, V]."""
    z, _ = forward(P, x, enc)
    w, _ = project(pou(z), x, rest_verts, lp_matrix(rest_verts))
    return w
