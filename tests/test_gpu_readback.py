"""Asynchronous framebuffer readback (cgs_readback_rgba8_async /
cgs_readback_wait): a frame's pixels copied while later frames render equal
the synchronous readback of the same frame; at most two copies are in
flight (a third call waits for the oldest); waiting twice, or for an unknown
ticket, behaves as documented."""
import numpy as np
import pytest
import torch

from cindergs_b200 import _abi, random_scene
from helpers import compositor, config0_camera

pytestmark = pytest.mark.gpu


def orbit_camera(k, w, h):
    from cindergs_b200 import CameraUniforms
    a = 0.3 * k
    eye = (4.0 * np.sin(a), 0.5, 4.0 * np.cos(a))
    return CameraUniforms.from_look_at(eye, (0, 0, 0), (0, 1, 0), np.deg2rad(60), w, h, 0.2)


def test_async_readback_matches_sync(gpu_state):
    st = gpu_state
    st.invalidate()
    scene = random_scene(60_000, seed=2)
    st.upload_scene(scene)
    w, h = 640, 360
    cams = [orbit_camera(k, w, h) for k in range(6)]
    # reference images, one synchronous readback per frame
    want = []
    for cam in cams:
        st.execute_frame_gpu(scene, None, cam, compositor(w, h, cam, deg=3), force_stage3=True)
        want.append(st.readback_framebuffer_rgba8(w, h))
    # the same frames with asynchronous copies into page-locked images; the
    # next frame is enqueued before the previous copy is waited for
    outs = [torch.empty((h, w, 4), dtype=torch.uint8).pin_memory().numpy() for _ in range(3)]
    tickets = []
    for k, cam in enumerate(cams):
        st.execute_frame_gpu(scene, None, cam, compositor(w, h, cam, deg=3), force_stage3=True,
                             stage_timings=False)
        tickets.append(st.readback_framebuffer_rgba8_async(outs[k % 3]))
        if k >= 1:
            st.readback_wait(tickets[k - 1])
            np.testing.assert_array_equal(outs[(k - 1) % 3], want[k - 1])
    st.readback_wait(tickets[-1])
    np.testing.assert_array_equal(outs[(len(cams) - 1) % 3], want[-1])
    st.readback_wait(tickets[-1])  # already waited for: returns at once
    assert tickets == sorted(tickets) and len(set(tickets)) == len(tickets)


def test_third_copy_waits_for_the_oldest(gpu_state):
    st = gpu_state
    st.invalidate()
    scene = random_scene(20_000, seed=4)
    st.upload_scene(scene)
    w, h = 320, 180
    outs = [np.empty((h, w, 4), np.uint8) for _ in range(3)]  # pageable memory works too
    imgs, tickets = [], []
    for k in range(3):
        cam = orbit_camera(k, w, h)
        st.execute_frame_gpu(scene, None, cam, compositor(w, h, cam, deg=2), force_stage3=True)
        imgs.append(st.readback_framebuffer_rgba8(w, h))
        tickets.append(st.readback_framebuffer_rgba8_async(outs[k]))
    # the third call waited for the first: its image is complete already
    np.testing.assert_array_equal(outs[0], imgs[0])
    for t in tickets:
        st.readback_wait(t)
    for o, im in zip(outs, imgs):
        np.testing.assert_array_equal(o, im)
    with pytest.raises(_abi.CgsError) as e:
        st.readback_wait(tickets[-1] + 100)
    assert e.value.code == _abi.CGS_E_ARG
    with pytest.raises(_abi.CgsError) as e:
        st.readback_framebuffer_rgba8_async(np.empty((h + 1, w, 4), np.uint8))
    assert e.value.code == _abi.CGS_E_ARG


def test_overflowed_earlier_frame_is_rendered_again():
    """A frame whose tile entries outgrow the key buffers while a later frame
    is already in flight is rendered again, from its own camera and cage
    vertices, when its asynchronous readback is waited for: the pixels equal
    a synchronous render of that frame by another context."""
    from cindergs_b200 import GpuPipelineState, workloads
    w, h = 1280, 720
    wl = workloads.tet_cage_orbit(n=40_000, width=w, height=h)
    wl.scene.covariances_3d[:] *= np.float32(40.0)  # large splats: many entries close up
    sim = wl.cage.simulator
    rest = wl.cage.mesh.rest_vertices.copy()
    rng = np.random.default_rng(3)
    verts = [(rest + rng.normal(0, 0.04, rest.shape)).astype(np.float32) for _ in range(3)]
    from cindergs_b200 import CameraUniforms
    far = CameraUniforms.from_look_at((0.0, 0.5, 40.0), (0, 0, 0), (0, 1, 0), np.deg2rad(60), w, h,
                                      0.2)
    near = CameraUniforms.from_look_at((0.0, 0.3, 2.2), (0, 0, 0), (0, 1, 0), np.deg2rad(60), w, h,
                                       0.2)
    # the expected pixels of the big frame, from a context sized by it
    ref = GpuPipelineState(0)
    try:
        ref.upload_scene(wl.scene)
        cages_r = wl.bind(ref)
        sim.current_positions = verts[1]
        ref.execute_frame_gpu(wl.scene, cages_r, near, compositor(w, h, near, deg=3),
                              force_stage3=True)
        want = ref.readback_framebuffer_rgba8(w, h)
    finally:
        ref.close()
    st = GpuPipelineState(0)
    try:
        st.upload_scene(wl.scene)
        cages = wl.cages  # the bindings made above, uploaded to this context too
        sim.current_positions = verts[0]
        t0 = st.execute_frame_gpu(wl.scene, cages, far, compositor(w, h, far, deg=3),
                                  force_stage3=True)
        out = torch.empty((h, w, 4), dtype=torch.uint8).pin_memory().numpy()
        sim.current_positions = verts[1]
        st.execute_frame_gpu(wl.scene, cages, near, compositor(w, h, near, deg=3),
                             force_stage3=True, stage_timings=False)
        ticket = st.readback_framebuffer_rgba8_async(out)
        sim.current_positions = verts[2]
        st.execute_frame_gpu(wl.scene, cages, far, compositor(w, h, far, deg=3),
                             force_stage3=True, stage_timings=False)
        st.readback_wait(ticket)
        np.testing.assert_array_equal(out, want)
        assert want[..., :3].max() > 0
        # the frame after it renders as usual
        sim.current_positions = verts[1]
        st.execute_frame_gpu(wl.scene, cages, near, compositor(w, h, near, deg=3),
                             force_stage3=True)
        np.testing.assert_array_equal(st.readback_framebuffer_rgba8(w, h), want)
        assert t0.total_tile_entries < 1_000_000
    finally:
        st.close()
