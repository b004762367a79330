"""GPU parity of the four-stage frame against the oracle (v2 semantics).

Stage 2 attributes and every Stage 3 integer (extents, scan offsets, sorted
keys and ids, tile ranges) must be bit-exact; Stage 4 RGB within 2e-3 absolute
in f32 and within one RGBA8 step (the reference's GPU tests allow a mean RGB
difference of 5e-3, tests/gpu_parity_tests.rs:231-290).
"""
import numpy as np
import pytest

import oracle
from cindergs_b200 import _abi
from cindergs_b200 import (CameraUniforms, CompositorUniforms, GaussianSceneSoa, random_scene)
from helpers import (assert_stage23_exact, compositor, config0_camera, gpu_buffers, oracle_frame,
                     parity_camera, varied_scene)

pytestmark = pytest.mark.gpu
RGB_TOL = 2e-3


def run_both(st, scene, cam, comp, **kw):
    t = st.execute_frame_gpu(scene, None, cam, comp, kw.get("split", 0.0), kw.get("mip", 0.0),
                             kw.get("min_opa", 1.0 / 255.0), kw.get("min_rad", 0.5),
                             profile_stages=True, force_stage3=True, write_f32=True,
                             radix_bits=kw.get("radix_bits", 0),
                             entry_sort=kw.get("entry_sort", 0))
    g = gpu_buffers(st, key64=t.used_64bit_keys)
    g["rgba8"] = st.readback_framebuffer_rgba8(comp.screen_width, comp.screen_height)
    g["f32"] = st.readback_framebuffer_f32(comp.screen_width, comp.screen_height)
    o = oracle_frame(scene, cam, comp, mip=kw.get("mip", 0.0), min_opa=kw.get("min_opa", 1 / 255.0),
                     min_rad=kw.get("min_rad", 0.5))
    return t, g, o


def check_image(g, o):
    d = np.abs(g["f32"] - o["rgba_f32"])
    assert d.max() <= RGB_TOL, f"max |rgba| diff {d.max()}"
    d8 = np.abs(g["rgba8"].astype(np.int32) - o["rgba8"].astype(np.int32))
    assert d8.max() <= 1, f"max rgba8 diff {d8.max()}"


SORTS = [_abi.SORT_RADIX, _abi.SORT_TRANSPOSE]


@pytest.mark.parametrize("entry_sort", SORTS)
def test_varied_scene_96px(gpu_state, entry_sort):
    scene = varied_scene()
    cam = parity_camera(96, 96)
    comp = compositor(96, 96, cam, deg=3)
    t, g, o = run_both(gpu_state, scene, cam, comp, entry_sort=entry_sort)
    assert t.total_tile_entries == o["entries"] > 0
    assert t.surviving_gaussians == o["surviving"]
    assert_stage23_exact(g, o)
    check_image(g, o)


@pytest.mark.parametrize("radix_bits,entry_sort", [(0, _abi.SORT_TRANSPOSE), (0, _abi.SORT_RADIX),
                                                   (8, _abi.SORT_RADIX), (5, _abi.SORT_RADIX),
                                                   (4, _abi.SORT_RADIX)])
def test_config0_scene_100k_720p(gpu_state, radix_bits, entry_sort):
    scene = random_scene(100_000, seed=0)
    cam = config0_camera(1280, 720)
    comp = compositor(1280, 720, cam, deg=3, bg=(0.0, 0.0, 0.0, 1.0))
    t, g, o = run_both(gpu_state, scene, cam, comp, radix_bits=radix_bits, entry_sort=entry_sort)
    assert t.total_tile_entries == o["entries"] > 100_000
    assert_stage23_exact(g, o)
    check_image(g, o)


def test_mip_and_culling_thresholds(gpu_state):
    scene = varied_scene()
    cam = parity_camera(96, 96)
    comp = compositor(96, 96, cam, deg=2)
    t, g, o = run_both(gpu_state, scene, cam, comp, mip=0.001, min_opa=0.01)
    assert t.surviving_gaussians == o["surviving"]
    assert_stage23_exact(g, o)
    check_image(g, o)


@pytest.mark.parametrize("entry_sort", SORTS)
@pytest.mark.parametrize("wh", [(19, 19), (1, 1), (17, 300)])
def test_ragged_viewports(gpu_state, wh, entry_sort):
    w, h = wh
    scene = random_scene(20_000, seed=3)
    cam = config0_camera(w, h)
    comp = compositor(w, h, cam, deg=1)
    t, g, o = run_both(gpu_state, scene, cam, comp, entry_sort=entry_sort)
    assert_stage23_exact(g, o)
    check_image(g, o)


def test_empty_scene(gpu_state):
    scene = GaussianSceneSoa(np.zeros((0, 3), np.float32), np.zeros((0, 6), np.float32),
                             np.zeros(0, np.float32), np.zeros((0, 48), np.float32))
    cam = config0_camera(64, 48)
    comp = compositor(64, 48, cam, bg=(0.1, 0.2, 0.3, 1.0))
    t = gpu_state.execute_frame_gpu(scene, None, cam, comp, force_stage3=True, write_f32=True)
    assert t.total_tile_entries == 0
    img = gpu_state.readback_framebuffer_f32(64, 48)
    np.testing.assert_allclose(img.reshape(-1, 4), np.tile([0.1, 0.2, 0.3, 1.0], (64 * 48, 1)),
                               atol=1e-7)


def test_all_culled_behind_camera(gpu_state):
    scene = random_scene(1000, seed=1)
    scene.positions[:, 2] = 10.0  # behind the camera at z=4 looking down -z
    cam = config0_camera(128, 64)
    comp = compositor(128, 64, cam)
    t, g, o = run_both(gpu_state, scene, cam, comp)
    assert t.total_tile_entries == 0 and t.surviving_gaussians == 0
    check_image(g, o)


def test_64bit_key_path_8k(gpu_state):
    """More than 65,535 tiles selects (tile, raw depth) keys (gpu_state.rs:1064)."""
    scene = random_scene(50_000, seed=5)
    cam = config0_camera(7680, 4320)
    comp = compositor(7680, 4320, cam, deg=3)
    t, g, o = run_both(gpu_state, scene, cam, comp)
    assert t.used_64bit_keys
    assert_stage23_exact(g, o, key64=True)
    check_image(g, o)


@pytest.mark.parametrize("wh,entry_sort", [((1920, 1080), _abi.SORT_RADIX),
                                           ((1920, 1080), _abi.SORT_TRANSPOSE),
                                           ((7680, 4320), _abi.SORT_TRANSPOSE)])
def test_huge_splats(gpu_state, wh, entry_sort):
    """Every 37th splat scaled 20x: tile boxes of up to 8,160 (1080p) and
    16,641 (8K, 64-bit keys) tiles, so binning warps exceed their stored
    ballot masks (4,096 candidates) and hit records (1,024) and re-walk their
    candidates for the rest."""
    w, h = wh
    scene = random_scene(3000, seed=21)
    scene.covariances_3d[::37] *= 400.0
    cam = config0_camera(w, h)
    comp = compositor(w, h, cam, deg=1)
    t, g, o = run_both(gpu_state, scene, cam, comp, entry_sort=entry_sort)
    counts = np.diff(np.append(o["offsets"], o["entries"]))
    assert counts.max() > 4096
    assert t.total_tile_entries == o["entries"]
    assert_stage23_exact(g, o, key64=t.used_64bit_keys)
    check_image(g, o)


def test_stage3_cache_and_repeatability(gpu_state):
    scene = random_scene(30_000, seed=7)
    cam = config0_camera(320, 240)
    comp = compositor(320, 240, cam)
    st = gpu_state
    t1 = st.execute_frame_gpu(scene, None, cam, comp, force_stage3=True)
    a = st.readback_framebuffer_rgba8(320, 240)
    t2 = st.execute_frame_gpu(scene, None, cam, comp)
    b = st.readback_framebuffer_rgba8(320, 240)
    assert not t1.stage3_cached and t2.stage3_cached
    np.testing.assert_array_equal(a, b)
    cam2 = CameraUniforms.from_look_at((0.4, 0.2, 4.0), (0, 0, 0), (0, 1, 0), np.deg2rad(60), 320,
                                       240, 0.2)
    t3 = st.execute_frame_gpu(scene, None, cam2, comp)
    assert not t3.stage3_cached


def test_key_buffer_overflow_is_rebinned(gpu_state):
    """A fresh context sizes its key buffers before it knows the entry count;
    a frame whose entries overflow them is binned again, so the readback and
    every Stage 3 buffer still match the oracle."""
    from cindergs_b200 import GpuPipelineState
    st = GpuPipelineState(0)
    try:
        scene = random_scene(4000, seed=13)
        scene.covariances_3d[:] = np.array([0.09, 0.0, 0.0, 0.09, 0.0, 0.09], np.float32)
        scene.positions *= np.float32(0.4)
        cam = config0_camera(1920, 1080)
        comp = compositor(1920, 1080, cam, deg=1)
        t, g, o = run_both(st, scene, cam, comp)
        assert t.total_tile_entries == o["entries"] > (1 << 20)  # initial buffers: 2^20
        assert_stage23_exact(g, o)
        check_image(g, o)
        # the next frame runs with grown buffers
        t2 = st.execute_frame_gpu(scene, None, cam, comp, force_stage3=True)
        assert t2.total_tile_entries == o["entries"]
    finally:
        st.close()
