"""Scene data: the reference's GaussianSceneSoa layout, activations and the
seeded synthetic scenes the benchmark configurations are defined on.

Layout (scene/soa.rs:30-52): positions [N,3], covariances_3d [N,6] packed
(xx, xy, xz, yy, yz, zz), opacities [N] (activated), sh_coeffs [N,48]
channel-major (DC r,g,b; 15 R rest; 15 G rest; 15 B rest; rasterizer/sh.rs:56-61),
all float32. Activations follow math/covariance.rs:13-98 with glam's
operation order, evaluated in float32.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

f32 = np.float32
MIN_SCALE = f32(1e-4)


@dataclass
class GaussianSceneSoa:
    positions: np.ndarray      # [N,3] f32
    covariances_3d: np.ndarray  # [N,6] f32
    opacities: np.ndarray      # [N] f32
    sh_coeffs: np.ndarray      # [N,48] f32 (or f16 for the quantised SH layout)

    @property
    def count(self) -> int:
        return int(self.opacities.shape[0])

    def __len__(self) -> int:
        return self.count

    def validate(self) -> None:
        n = self.count
        assert self.positions.shape == (n, 3) and self.positions.dtype == np.float32
        assert self.covariances_3d.shape == (n, 6) and self.covariances_3d.dtype == np.float32
        assert self.opacities.shape == (n,) and self.opacities.dtype == np.float32
        assert self.sh_coeffs.shape == (n, 48) and self.sh_coeffs.dtype in (np.float32, np.float16)

    def as_dict(self) -> dict:
        return dict(pos=self.positions.ravel(), cov=self.covariances_3d.ravel(),
                    opa=self.opacities, sh=self.sh_coeffs.astype(np.float32).ravel())

    @staticmethod
    def from_arrays(pos, cov, opa, sh) -> "GaussianSceneSoa":
        s = GaussianSceneSoa(np.ascontiguousarray(pos, f32).reshape(-1, 3),
                             np.ascontiguousarray(cov, f32).reshape(-1, 6),
                             np.ascontiguousarray(opa, f32).reshape(-1),
                             np.ascontiguousarray(sh).reshape(-1, 48))
        s.validate()
        return s


def sh_bases_for_degree(sh_degree: int) -> int:
    """SH basis functions up to a degree (soa.rs:331-338)."""
    return {0: 1, 1: 4, 2: 9}.get(int(sh_degree), 16)


def sh_packed_words_for_degree(sh_degree: int) -> int:
    """u32 words of f16 pairs per splat (soa.rs:342-344)."""
    return (sh_bases_for_degree(sh_degree) * 3 + 1) // 2


def pack_f16_pairs(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    """low = f16(a), high = f16(b), round to nearest even (soa.rs:348-352)."""
    ha = np.asarray(a, np.float32).astype(np.float16).view(np.uint16).astype(np.uint32)
    hb = np.asarray(b, np.float32).astype(np.float16).view(np.uint16).astype(np.uint32)
    return ha | (hb << np.uint32(16))


def unpack_f16_pairs(w: np.ndarray):
    """(low, high) of f16 pair words as float32 (soa.rs:356-360)."""
    w = np.asarray(w, np.uint32)
    lo = (w & np.uint32(0xFFFF)).astype(np.uint16).view(np.float16).astype(np.float32)
    hi = (w >> np.uint32(16)).astype(np.uint16).view(np.float16).astype(np.float32)
    return lo, hi


@dataclass
class QuantizedGaussianSceneSoa:
    """QuantizedGaussianSceneSoa (scene/soa.rs:429-608): f32 positions and
    opacities, covariances as three words of f16 pairs per splat, SH up to
    `sh_degree` as f16 pairs in the order DC rgb, then each channel's higher
    orders. The reference's octahedral rotation word is used by no stage of
    the frame and is not kept."""
    positions: np.ndarray              # [N,3] f32
    covariances_f16_packed: np.ndarray  # [N,3] u32
    opacities: np.ndarray              # [N] f32
    sh_coeffs_f16_packed: np.ndarray   # [N,words] u32
    sh_degree: int = 3

    @property
    def count(self) -> int:
        return int(self.opacities.shape[0])

    def __len__(self) -> int:
        return self.count

    def fingerprint_arrays(self):
        return (self.positions, self.covariances_f16_packed, self.opacities,
                self.sh_coeffs_f16_packed)

    @staticmethod
    def from_soa(scene: GaussianSceneSoa, sh_degree: int = 3) -> "QuantizedGaussianSceneSoa":
        """from_soa_with_degree (soa.rs:453-498)."""
        deg = min(int(sh_degree), 3)
        bases = sh_bases_for_degree(deg)
        rest = bases - 1
        c = np.asarray(scene.covariances_3d, np.float32)
        cov = np.stack([pack_f16_pairs(c[:, 0], c[:, 1]), pack_f16_pairs(c[:, 2], c[:, 3]),
                        pack_f16_pairs(c[:, 4], c[:, 5])], axis=1)
        sh = np.asarray(scene.sh_coeffs, np.float32)
        words = sh_packed_words_for_degree(deg)
        lin = np.zeros((scene.count, words * 2), np.float32)
        lin[:, 0:3] = sh[:, 0:3]
        if rest:
            lin[:, 3:3 + rest] = sh[:, 3:3 + rest]
            lin[:, 3 + rest:3 + 2 * rest] = sh[:, 18:18 + rest]
            lin[:, 3 + 2 * rest:3 + 3 * rest] = sh[:, 33:33 + rest]
        packed = pack_f16_pairs(lin[:, 0::2], lin[:, 1::2])
        return QuantizedGaussianSceneSoa(np.ascontiguousarray(scene.positions, np.float32),
                                         np.ascontiguousarray(cov, np.uint32),
                                         np.ascontiguousarray(scene.opacities, np.float32),
                                         np.ascontiguousarray(packed, np.uint32), deg)

    def unpack_covariance_3d(self) -> np.ndarray:
        """[N,6] (soa.rs:508-515)."""
        out = np.empty((self.count, 6), np.float32)
        for k in range(3):
            out[:, 2 * k], out[:, 2 * k + 1] = unpack_f16_pairs(self.covariances_f16_packed[:, k])
        return out

    def unpack_sh_48(self) -> np.ndarray:
        """[N,48] channel-major, zeros above the degree (soa.rs:518-546)."""
        bases = sh_bases_for_degree(self.sh_degree)
        rest = bases - 1
        lo, hi = unpack_f16_pairs(self.sh_coeffs_f16_packed)
        lin = np.empty((self.count, lo.shape[1] * 2), np.float32)
        lin[:, 0::2], lin[:, 1::2] = lo, hi
        lin[:, bases * 3:] = 0.0
        out = np.zeros((self.count, 48), np.float32)
        out[:, 0:3] = lin[:, 0:3]
        if rest:
            out[:, 3:3 + rest] = lin[:, 3:3 + rest]
            out[:, 18:18 + rest] = lin[:, 3 + rest:3 + 2 * rest]
            out[:, 33:33 + rest] = lin[:, 3 + 2 * rest:3 + 3 * rest]
        return out

    def to_soa(self) -> GaussianSceneSoa:
        """Dequantized scene (soa.rs:549-560), SH kept as float32."""
        return GaussianSceneSoa(self.positions.copy(), self.unpack_covariance_3d(),
                                self.opacities.copy(), self.unpack_sh_48())


def activate_opacity(raw: np.ndarray) -> np.ndarray:
    """1 / (1 + exp(-raw)) (covariance.rs:13-15)."""
    raw = raw.astype(f32)
    return (f32(1.0) / (f32(1.0) + np.exp(-raw))).astype(f32)


def activate_scale(raw: np.ndarray) -> np.ndarray:
    """max(exp(raw), 1e-4) per axis (covariance.rs:21-27)."""
    return np.maximum(np.exp(raw.astype(f32)), MIN_SCALE).astype(f32)


def activate_rotation(raw_wxyz: np.ndarray) -> np.ndarray:
    """Normalised quaternion (x, y, z, w) from PLY order (w, x, y, z); identity
    below norm 1e-6 (covariance.rs:36-51). Returns [N,4] as x, y, z, w."""
    r = raw_wxyz.astype(f32)
    w, x, y, z = r[:, 0], r[:, 1], r[:, 2], r[:, 3]
    norm = np.sqrt(((x * x + y * y) + z * z) + w * w).astype(f32)
    small = norm < f32(1e-6)
    inv = (f32(1.0) / np.where(small, f32(1.0), norm)).astype(f32)
    q = np.stack([x * inv, y * inv, z * inv, w * inv], axis=1).astype(f32)
    q[small] = np.array([0, 0, 0, 1], f32)
    return q


def quat_to_mat3(q_xyzw: np.ndarray) -> np.ndarray:
    """glam Mat3::from_quat; returns [N,3,3] as [n, column, row]."""
    x, y, z, w = (q_xyzw[:, k] for k in range(4))
    x2, y2, z2 = x + x, y + y, z + z
    xx, xy, xz = x * x2, x * y2, x * z2
    yy, yz, zz = y * y2, y * z2, z * z2
    wx, wy, wz = w * x2, w * y2, w * z2
    one = f32(1.0)
    cols = np.empty((q_xyzw.shape[0], 3, 3), f32)
    cols[:, 0] = np.stack([one - (yy + zz), xy + wz, xz - wy], axis=1)
    cols[:, 1] = np.stack([xy - wz, one - (xx + zz), yz + wx], axis=1)
    cols[:, 2] = np.stack([xz + wy, yz - wx, one - (xx + yy)], axis=1)
    return cols


def compute_covariance_3d(scale: np.ndarray, q_xyzw: np.ndarray) -> np.ndarray:
    """Sigma = (R S)(R S)^T packed (xx, xy, xz, yy, yz, zz) (covariance.rs:61-98)."""
    R = quat_to_mat3(q_xyzw.astype(f32))
    M = (R * scale.astype(f32)[:, :, None]).astype(f32)  # column k scaled by s_k
    def entry(i, j):
        return ((M[:, 0, i] * M[:, 0, j] + M[:, 1, i] * M[:, 1, j]) + M[:, 2, i] * M[:, 2, j]).astype(f32)
    return np.stack([entry(0, 0), entry(1, 0), entry(2, 0), entry(1, 1), entry(2, 1), entry(2, 2)],
                    axis=1).astype(f32)


def random_unit_quaternions(rng: np.random.Generator, n: int) -> np.ndarray:
    """Uniformly random unit quaternions (Shoemake 1992) in PLY order (w, x, y, z)."""
    u = rng.random((n, 3))
    a = np.sqrt(1.0 - u[:, 0])
    b = np.sqrt(u[:, 0])
    t1 = 2.0 * np.pi * u[:, 1]
    t2 = 2.0 * np.pi * u[:, 2]
    x, y = a * np.sin(t1), a * np.cos(t1)
    z, w = b * np.sin(t2), b * np.cos(t2)
    return np.stack([w, x, y, z], axis=1).astype(f32)


def random_scene(n: int, seed: int = 0, box: float | None = None) -> GaussianSceneSoa:
    """The synthetic scene of the benchmark configurations.

    numpy Generator(PCG64(seed)), drawn in this order: means ~ N(0, I3);
    log-scales ~ U[-4.5, -2.0] per axis; Shoemake-uniform unit quaternions;
    opacity logits ~ N(0, 1); SH degree 3 (48 coefficients) with DC ~ N(0, 0.5)
    and higher orders ~ N(0, 0.05). Covariances and opacities are activated as
    a PLY vertex would be (soa.rs:113-125). With ``box`` set, the means are
    scaled by box / max|mean| so the cloud fills [-box, box]^3 (scales are
    left as drawn).
    """
    rng = np.random.Generator(np.random.PCG64(seed))
    means = rng.standard_normal((n, 3)).astype(f32)
    log_scales = rng.uniform(-4.5, -2.0, (n, 3)).astype(f32)
    quats = random_unit_quaternions(rng, n)
    logits = rng.standard_normal(n).astype(f32)
    sh = np.empty((n, 48), f32)
    sh[:, 0:3] = rng.normal(0.0, 0.5, (n, 3))
    sh[:, 3:] = rng.normal(0.0, 0.05, (n, 45))
    if box is not None and n > 0:
        m = float(np.abs(means).max())
        if m > 0:
            means = (means * f32(box / m)).astype(f32)
    cov = compute_covariance_3d(activate_scale(log_scales), activate_rotation(quats))
    return GaussianSceneSoa(means, cov, activate_opacity(logits), sh)


def fibonacci_cluster(count: int, radius: float, center) -> GaussianSceneSoa:
    """Fibonacci-sphere cluster with rainbow DC colour (scene/synthetic.rs:6-44),
    evaluated with numpy float32 transcendental functions."""
    i = np.arange(count, dtype=f32)
    golden = (f32(1.0) + np.sqrt(f32(5.0))) / f32(2.0)
    t = (i + f32(0.5)) / f32(count)
    r = f32(radius) * np.cbrt(t)
    theta = np.arccos(np.clip(f32(1.0) - f32(2.0) * t, -1, 1)).astype(f32)
    phi = (f32(2.0 * np.pi) * (i / golden)).astype(f32)
    c = np.asarray(center, f32)
    pos = np.stack([c[0] + r * np.sin(theta) * np.cos(phi), c[1] + r * np.sin(theta) * np.sin(phi),
                    c[2] + r * np.cos(theta)], axis=1).astype(f32)
    cov = np.tile(np.array([0.0004, 0, 0, 0.0004, 0, 0.0004], f32), (count, 1))
    opa = np.full(count, 0.88, f32)
    sh = np.zeros((count, 48), f32)
    sh_c0 = f32(0.28209479)
    for k, ph in enumerate((0.0, 2.094, 4.188)):
        col = f32(0.5) + f32(0.5) * np.sin(i * f32(0.02) + f32(ph))
        sh[:, k] = (col - f32(0.5)) / sh_c0
    return GaussianSceneSoa(pos, cov, opa, sh)
