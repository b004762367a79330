"""GPU parity of Stage 1 (tet-cage deformation) and the GPU binder.

The deformed positions, covariances and opacities, the per-tet Jacobians,
rotations and stretches, the split children (placed in parent order) and all
downstream Stage 2/3 buffers must match the oracle bit for bit; the image
within 2e-3.
"""
import numpy as np
import pytest

import oracle
from cindergs_b200 import Cage, CageScene, TetMesh, UNBOUND, random_scene
from cindergs_b200 import _abi
from cindergs_b200.workloads import tet_cage_orbit
from helpers import (assert_stage23_exact, compositor, config0_camera, gpu_buffers, oracle_frame)

pytestmark = pytest.mark.gpu


def cage_dict(cages):
    elems, inv, nverts, bt, bw = cages.flatten()
    return dict(verts=cages.flat_vertices(), elems=elems, inv_dm=inv, bind_tet=bt, bind_w=bw)


def deformed_frame(st, scene, cages, cam, comp, split, mip):
    t = st.execute_frame_gpu(scene, cages, cam, comp, split, mip, 1.0 / 255.0, 0.5,
                             profile_stages=True, force_stage3=True, write_f32=True)
    g = gpu_buffers(st)
    g["pos"] = st.read_buffer(_abi.BUF_DEFORMED_POS, np.float32)
    g["cov"] = st.read_buffer(_abi.BUF_DEFORMED_COV, np.float32)
    g["opa"] = st.read_buffer(_abi.BUF_DEFORMED_OPA, np.float32)
    g["J"] = st.read_buffer(_abi.BUF_TET_JACOBIANS, np.float32)
    g["R"] = st.read_buffer(_abi.BUF_TET_ROTATIONS, np.float32)
    g["S"] = st.read_buffer(_abi.BUF_TET_STRETCH, np.float32)
    g["meta"] = st.read_buffer(_abi.BUF_SPLIT_META, np.uint32)
    g["f32"] = st.readback_framebuffer_f32(comp.screen_width, comp.screen_height)
    o = oracle_frame(scene, cam, comp, cage=cage_dict(cages), mip=mip, split_thr=split)
    return t, g, o


def bits(a):
    return np.asarray(a, np.float32).view(np.uint32)


@pytest.mark.parametrize("split,mip", [(0.0, 0.0), (0.0, 0.001), (1.25, 0.001), (1.1, 0.0)])
def test_grid_cage_deform_parity(gpu_state, split, mip):
    st = gpu_state
    n = 60_000
    scene = random_scene(n, seed=21, box=1.0)
    st.upload_scene(scene)
    mesh = TetMesh.create_grid_cage((3, 3, 3), (-1.1,) * 3, (1.1,) * 3)
    cage = Cage("g", mesh)
    cages = CageScene.auto_bind([cage], st, n)
    rng = np.random.default_rng(5)
    cage.simulator.current_positions = (mesh.rest_vertices * np.float32(1.15) + rng.normal(
        0, 0.07, mesh.rest_vertices.shape)).astype(np.float32)
    cam = config0_camera(640, 360)
    comp = compositor(640, 360, cam, deg=3)
    t, g, o = deformed_frame(st, scene, cages, cam, comp, split, mip)
    np.testing.assert_array_equal(bits(g["J"]), bits(o["J"]), err_msg="tet J")
    np.testing.assert_array_equal(bits(g["R"]), bits(o["R"]), err_msg="tet R")
    np.testing.assert_array_equal(bits(g["S"]), bits(o["stretch"]), err_msg="tet stretch")
    assert t.active_gaussians == n + o["splits"]
    if split > 0:
        assert o["splits"] > 0
        np.testing.assert_array_equal(g["meta"], o["meta"], err_msg="split meta")
    np.testing.assert_array_equal(bits(g["pos"]), bits(o["def_pos"]), err_msg="positions")
    np.testing.assert_array_equal(bits(g["cov"]), bits(o["def_cov"]), err_msg="covariances")
    np.testing.assert_array_equal(bits(g["opa"]), bits(o["def_opa"]), err_msg="opacities")
    assert_stage23_exact(g, o)
    assert np.abs(g["f32"] - o["rgba_f32"]).max() <= 2e-3


def test_gpu_binding_matches_oracle(gpu_state):
    st = gpu_state
    n = 50_000
    scene = random_scene(n, seed=2, box=1.05)
    st.upload_scene(scene)
    mesh = TetMesh.create_grid_cage((5, 5, 5), (-1.1,) * 3, (1.1,) * 3)
    for bounds in (None, mesh.bounds()):
        t, w = st.bind_tets(mesh, bounds=bounds)
        ot, ow = oracle.bind_points(scene.positions, mesh.rest_vertices, mesh.elements,
                                    mesh.inv_dm, bounds)
        np.testing.assert_array_equal(t, ot)
        np.testing.assert_array_equal(bits(w), bits(ow))
    # a box cage that leaves part of the scene outside: unbound stays UNBOUND
    box = TetMesh.create_box_cage((-0.5, -0.5, -0.5), (0.5, 0.5, 0.5))
    t, w = st.bind_tets(box, bounds=box.bounds())
    ot, ow = oracle.bind_points(scene.positions, box.rest_vertices, box.elements, box.inv_dm,
                                box.bounds())
    np.testing.assert_array_equal(t, ot)
    assert (t == UNBOUND).any() and (t != UNBOUND).any()


def test_dirty_flags_and_stage_cache(gpu_state):
    """Frame 1 deforms; camera move -> Stage 1 skipped, Stage 3 rebuilt; static
    frame -> both cached, identical pixels; cage move -> Stage 1 again
    (tests/gpu_parity_tests.rs:1053-1205)."""
    st = gpu_state
    wl = tet_cage_orbit(n=40_000, width=320, height=240)
    st.upload_scene(wl.scene)
    cages = wl.bind(st)
    cam1, cam2 = wl.camera(0), wl.camera(7)
    t1 = st.execute_frame_gpu(wl.scene, cages, cam1, wl.compositor(cam1))
    assert not t1.stage1_skipped and not t1.stage3_cached
    t2 = st.execute_frame_gpu(wl.scene, cages, cam2, wl.compositor(cam2))
    assert t2.stage1_skipped and not t2.stage3_cached
    a = st.readback_framebuffer_rgba8(320, 240)
    t3 = st.execute_frame_gpu(wl.scene, cages, cam2, wl.compositor(cam2))
    assert t3.stage1_skipped and t3.stage3_cached
    b = st.readback_framebuffer_rgba8(320, 240)
    np.testing.assert_array_equal(a, b)
    wl.step()
    t4 = st.execute_frame_gpu(wl.scene, cages, cam2, wl.compositor(cam2))
    assert not t4.stage1_skipped and not t4.stage3_cached


def test_multi_cage_first_cage_wins(gpu_state):
    st = gpu_state
    n = 30_000
    scene = random_scene(n, seed=9, box=1.0)
    st.upload_scene(scene)
    c1 = Cage("a", TetMesh.create_grid_cage((2, 2, 2), (-1.05, -1.05, -1.05), (0.2, 1.05, 1.05)))
    c2 = Cage("b", TetMesh.create_grid_cage((2, 2, 2), (-0.2, -1.05, -1.05), (1.05, 1.05, 1.05)))
    cages = CageScene.auto_bind([c1, c2], st, n)
    assert (cages.bind_cage == 0).any() and (cages.bind_cage == 1).any()
    overlap = (scene.positions[:, 0] > -0.19) & (scene.positions[:, 0] < 0.19)
    assert (cages.bind_cage[overlap] == 0).all()
    rng = np.random.default_rng(0)
    for c in (c1, c2):
        c.simulator.current_positions = (c.mesh.rest_vertices + rng.normal(
            0, 0.05, c.mesh.rest_vertices.shape)).astype(np.float32)
    cam = config0_camera(320, 180)
    comp = compositor(320, 180, cam, deg=2)
    t, g, o = deformed_frame(st, scene, cages, cam, comp, 1.2, 0.001)
    np.testing.assert_array_equal(bits(g["pos"]), bits(o["def_pos"]))
    assert_stage23_exact(g, o)
