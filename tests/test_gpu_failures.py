"""Failure paths, made to happen on purpose without faulting the GPU.

* Allocation failure: a device-memory budget (cgs_ctx_set_device_budget)
  below what a scene or frame needs makes the growth fail with CGS_E_OOM, as
  a failed cudaMalloc does; the context stays usable once the budget allows
  the allocation (the reference's error surface: render/gpu.rs:14-30).
* Bounded waits: cgs_ctx_wait_drill runs the chained-scan look-back, the
  radix sort's digit look-back and the compositor's mbarrier wait against a
  flag or barrier that nothing completes; each gives up after its polls,
  the call returns CGS_E_TIMEOUT, and the next frame renders correctly.
"""
import numpy as np
import pytest

from cindergs_b200 import GpuPipelineState, random_scene
from cindergs_b200 import _abi
from helpers import assert_stage23_exact, compositor, config0_camera, gpu_buffers, oracle_frame

pytestmark = pytest.mark.gpu


def small_frame_matches_oracle(st, scene, w=320, h=180):
    cam = config0_camera(w, h)
    comp = compositor(w, h, cam, deg=3, bg=(0.0, 0.0, 0.0, 1.0))
    t = st.execute_frame_gpu(scene, None, cam, comp, force_stage3=True, write_f32=True)
    g = gpu_buffers(st)
    o = oracle_frame(scene, cam, comp)
    assert t.total_tile_entries == o["entries"] > 0
    assert_stage23_exact(g, o)
    img = st.readback_framebuffer_f32(w, h)
    assert float(np.abs(img - o["rgba_f32"]).max()) <= 2e-3


def test_device_budget_gives_oom_and_recovers():
    st = GpuPipelineState(0)
    try:
        big = random_scene(1_000_000, seed=3)
        st.set_device_budget(32 << 20)  # the resident scene alone needs ~240 MB
        with pytest.raises(_abi.CgsError) as e:
            st.upload_scene(big)
        assert e.value.code == _abi.CGS_E_OOM
        assert "budget" in str(e.value)
        # a scene that fits, then a frame whose arena outgrows the budget
        small = random_scene(20_000, seed=5)
        st.set_device_budget(0)
        st.upload_scene(small)
        held = st.device_bytes()
        st.set_device_budget(held + (1 << 20))
        cam = config0_camera(1920, 1080)
        comp = compositor(1920, 1080, cam)
        with pytest.raises(_abi.CgsError) as e:
            st.execute_frame_gpu(small, None, cam, comp, force_stage3=True)
        assert e.value.code == _abi.CGS_E_OOM
        st.set_device_budget(0)
        small_frame_matches_oracle(st, small)
    finally:
        st.close()


def test_bounded_waits_give_up_and_context_survives():
    st = GpuPipelineState(0)
    try:
        scene = random_scene(30_000, seed=6)
        st.upload_scene(scene)
        small_frame_matches_oracle(st, scene)
        rc, mask = st.wait_drill(1 << 16)
        assert rc == _abi.CGS_E_TIMEOUT, rc
        assert mask == 0b111, mask
        # the context is usable afterwards and frames are still exact
        small_frame_matches_oracle(st, scene)
        rc, mask = st.wait_drill(1 << 10)
        assert rc == _abi.CGS_E_TIMEOUT and mask == 0b111
        small_frame_matches_oracle(st, scene, 640, 360)
    finally:
        st.close()
