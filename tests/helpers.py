"""Shared scene/camera fixtures and GPU-vs-oracle frame comparison."""
import numpy as np

import oracle
from cindergs_b200 import (CameraUniforms, CompositorUniforms, GaussianSceneSoa, random_scene)
from cindergs_b200 import _abi

f32 = np.float32


def varied_scene() -> GaussianSceneSoa:
    """The reference's 48-splat anisotropic fixture (tests/gpu_parity_tests.rs:64-99)."""
    n = 48
    i = np.arange(n, dtype=f32)
    golden = (f32(1.0) + np.sqrt(f32(5.0))) / f32(2.0)
    t = (i + f32(0.5)) / f32(n)
    theta = np.arccos(np.clip(f32(1) - f32(2) * t, -1, 1)).astype(f32)
    phi = (f32(2 * np.pi) * (i / golden)).astype(f32)
    r = f32(0.6)
    pos = np.stack([r * np.sin(theta) * np.cos(phi), r * np.sin(theta) * np.sin(phi),
                    r * np.cos(theta) + f32(2.0)], axis=1).astype(f32)
    sx = f32(0.02) + f32(0.01) * np.abs(np.sin(i * f32(0.3)))
    sy = f32(0.03) + f32(0.01) * np.abs(np.cos(i * f32(0.7)))
    sz = f32(0.015) + f32(0.005) * np.abs(np.sin(i * f32(0.11)))
    cov = np.stack([sx * sx, np.full(n, 0.0004, f32), np.full(n, 0.0002, f32), sy * sy,
                    np.full(n, 0.0003, f32), sz * sz], axis=1).astype(f32)
    opa = (f32(0.35) + f32(0.5) * (np.sin(i * f32(0.27)) * f32(0.5) + f32(0.5))).astype(f32)
    k = np.arange(48)
    sh = (np.sin(((i[:, None].astype(np.int64) * 17 + k[None, :] * 31)).astype(f32) * f32(0.013))
          * f32(0.4)).astype(f32)
    sh[:, 0] = 1.2
    sh[:, 1] = 0.4
    return GaussianSceneSoa(pos, cov, opa, sh)


def parity_camera(w, h) -> CameraUniforms:
    """test_camera (tests/gpu_parity_tests.rs:52-62)."""
    return CameraUniforms.from_look_at((0.0, 0.0, -1.0), (0.0, 0.0, 2.0), (0, 1, 0),
                                       np.deg2rad(50.0), w, h, 0.2)


def config0_camera(w=1280, h=720) -> CameraUniforms:
    return CameraUniforms.from_look_at((0.0, 0.0, 4.0), (0, 0, 0), (0, 1, 0), np.deg2rad(60.0),
                                       w, h, 0.2)


def compositor(w, h, cam: CameraUniforms, deg=3, bg=(0.02, 0.03, 0.05, 1.0)):
    return CompositorUniforms(w, h, bg, tuple(float(x) for x in cam.eye()), deg)


def oracle_frame(scene, cam, comp, cage=None, **kw):
    return oracle.v2_frame(scene.as_dict(), cam.to_array(),
                           dict(width=comp.screen_width, height=comp.screen_height,
                                bg=np.asarray(comp.background_color, f32),
                                cam_pos=np.asarray(comp.camera_position, f32),
                                sh_degree=comp.sh_degree), cage=cage, **kw)


def gpu_buffers(st, key64=False):
    out = dict(
        attrs=st.read_buffer(_abi.BUF_SPLAT_ATTRS, np.float32),
        ext=st.read_buffer(_abi.BUF_EXTENTS, np.uint32),
        offsets=st.read_buffer(_abi.BUF_TILE_OFFSETS, np.uint32),
        sorted_ids=st.read_buffer(_abi.BUF_SORTED_IDS, np.uint32),
        ranges=st.read_buffer(_abi.BUF_TILE_RANGES, np.uint32),
    )
    out["sorted_keys"] = st.read_buffer(_abi.BUF_SORTED_KEYS, np.uint64 if key64 else np.uint32)
    return out


def assert_stage23_exact(g, o, key64=False):
    """Stage 2 outputs and every Stage 3 integer bit-exact against the oracle."""
    np.testing.assert_array_equal(g["ext"], o["ext"], err_msg="extents")
    np.testing.assert_array_equal(g["attrs"].view(np.uint32), o["attrs"].view(np.uint32),
                                  err_msg="splat attributes (bits)")
    np.testing.assert_array_equal(g["offsets"], o["offsets"], err_msg="scan offsets")
    if key64:
        ok = (o["sorted_tiles"].astype(np.uint64) << np.uint64(32)) | o["sorted_depths"].astype(np.uint64)
        np.testing.assert_array_equal(g["sorted_keys"], ok, err_msg="sorted 64-bit keys")
    else:
        np.testing.assert_array_equal(g["sorted_keys"], o["sorted_keys"], err_msg="sorted keys")
    np.testing.assert_array_equal(g["sorted_ids"], o["sorted_ids"], err_msg="sorted ids")
    np.testing.assert_array_equal(g["ranges"], o["ranges"], err_msg="tile ranges")
