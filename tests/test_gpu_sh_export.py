"""SH coefficient rotation and the deformed-scene export on the GPU.

cgs_sh_rotate must equal the oracle's ShRotator restatement
(render/rasterizer/sh_rotation.rs) bit for bit: the f64 band matrices are
built in the reference's operation order on both sides and applied with an
f32 running sum. cgs_export_deformed must return Stage 1's own deformed
records (bit-equal to the frame buffers) with each splat's coefficients
rotated by its tet's or polygon-cage slot's rotation (a split child by its
parent's), and its PLY bytes must reload to the same scene.
"""
import numpy as np
import pytest

import oracle
from cindergs_b200 import (Cage, CageScene, CameraUniforms, CompositorUniforms, GpuPipelineState,
                           PolyCageMesh, QuantizedGaussianSceneSoa, TetMesh, ply, random_scene)
from cindergs_b200 import _abi
from helpers import compositor, config0_camera

pytestmark = pytest.mark.gpu
f32 = np.float32
MVC_BOUND = 0xFFFFFFFE


def bits(a):
    return np.asarray(a, f32).view(np.uint32)


def random_rotations(k, seed):
    rng = np.random.default_rng(seed)
    q = rng.normal(size=(k, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    x, y, z, w = q.T
    R = np.stack([np.stack([1 - 2 * (y * y + z * z), 2 * (x * y - w * z), 2 * (x * z + w * y)], -1),
                  np.stack([2 * (x * y + w * z), 1 - 2 * (x * x + z * z), 2 * (y * z - w * x)], -1),
                  np.stack([2 * (x * z - w * y), 2 * (y * z + w * x), 1 - 2 * (x * x + y * y)], -1)],
                 axis=1)
    return R.astype(f32)  # [k, row, col]


def col_major(R):
    return np.ascontiguousarray(np.asarray(R, f32).T).ravel()


def expected_rotation(sh, R9_of, source, degree):
    """sh [n,48] rotated per splat by R9_of[source[i]] (column-major 9), or
    left as is where source[i] < 0, grouped by rotation for the oracle."""
    out = np.asarray(sh, f32).copy()
    for r in np.unique(source[source >= 0]):
        sel = np.nonzero(source == r)[0]
        out[sel] = oracle.ref_sh_rotate(out[sel], R9_of[r], degree).reshape(-1, 48)
    return out


@pytest.fixture(scope="module")
def st():
    s = GpuPipelineState(0)
    yield s
    s.close()


@pytest.mark.parametrize("degree", [1, 2, 3])
def test_sh_rotate_matches_the_oracle(st, degree):
    n, k = 20_000, 61
    rng = np.random.default_rng(degree)
    sh = rng.normal(0, 0.3, size=(n, 48)).astype(f32)
    rots = random_rotations(k, seed=degree + 10)
    index = rng.integers(0, k, n).astype(np.uint32)
    got = st.sh_rotate(sh, rots, index, degree)
    want = expected_rotation(sh, [col_major(R) for R in rots], index.astype(np.int64), degree)
    np.testing.assert_array_equal(bits(got), bits(want))
    # without an index: rotation i % k
    got2 = st.sh_rotate(sh[:500], rots, None, degree)
    want2 = expected_rotation(sh[:500], [col_major(R) for R in rots], np.arange(500) % k, degree)
    np.testing.assert_array_equal(bits(got2), bits(want2))


def test_sh_rotate_rejects_an_out_of_range_index(st):
    sh = np.ones((8, 48), f32)
    rots = random_rotations(2, seed=1)
    import torch
    t = torch.as_tensor(sh).cuda()
    with pytest.raises(_abi.CgsError) as e:
        st.sh_rotate(t, rots, np.array([0, 1, 2, 0, 1, 7, 0, 1], np.uint32), 3)
    assert e.value.code == _abi.CGS_E_ARG
    out = t.cpu().numpy()
    np.testing.assert_array_equal(out[[2, 5]], sh[[2, 5]])  # left unchanged
    assert not np.array_equal(out[0], sh[0])


def tet_setup(st, n, quantized=False):
    st.invalidate()
    scene = random_scene(n, seed=21, box=1.0)
    if quantized:
        q = QuantizedGaussianSceneSoa.from_soa(scene, 3)
        st.upload_scene(q)
        scene = q.to_soa()
    else:
        st.upload_scene(scene)
    mesh = TetMesh.create_grid_cage((3, 3, 3), (-1.1,) * 3, (1.1,) * 3)
    cage = Cage("g", mesh)
    cages = CageScene.auto_bind([cage], st, n)
    rng = np.random.default_rng(5)
    cage.simulator.current_positions = (mesh.rest_vertices * f32(1.15) + rng.normal(
        0, 0.07, mesh.rest_vertices.shape)).astype(f32)
    return scene, cages


@pytest.mark.parametrize("split,quantized", [(0.0, False), (1.1, False), (1.1, True)])
def test_export_of_a_tet_cage_frame(st, split, quantized):
    n = 40_000
    scene, cages = tet_setup(st, n, quantized)
    cam = config0_camera(320, 180)
    comp = compositor(320, 180, cam, deg=3)
    t = st.execute_frame_gpu(scene, cages, cam, comp, split, 0.0, force_stage3=True)
    out = st.export_deformed(sh_degree=3)
    total = t.active_gaussians
    assert out.count == total
    if split > 0:
        assert total > n
    pos = st.read_buffer(_abi.BUF_DEFORMED_POS, f32).reshape(-1, 3)
    cov = st.read_buffer(_abi.BUF_DEFORMED_COV, f32).reshape(-1, 6)
    opa = st.read_buffer(_abi.BUF_DEFORMED_OPA, f32)
    np.testing.assert_array_equal(bits(out.positions), bits(pos))
    np.testing.assert_array_equal(bits(out.covariances_3d), bits(cov))
    np.testing.assert_array_equal(bits(out.opacities), bits(opa))
    R = st.read_buffer(_abi.BUF_TET_ROTATIONS, f32).reshape(-1, 9)
    _, _, _, bind_tet, _ = cages.flatten()
    meta = st.read_buffer(_abi.BUF_SPLIT_META, np.uint32).reshape(-1, 2)
    parent = np.concatenate([np.arange(n), meta[:, 0].astype(np.int64)])
    tet = np.concatenate([bind_tet.astype(np.int64), meta[:, 1].astype(np.int64)])
    source = np.where(tet < R.shape[0], tet, -1)
    want = expected_rotation(scene.sh_coeffs[parent], R, source, 3)
    np.testing.assert_array_equal(bits(out.sh_coeffs), bits(want))
    # a lower degree rotates only its bands
    out1 = st.export_deformed(sh_degree=1)
    np.testing.assert_array_equal(bits(out1.sh_coeffs),
                                  bits(expected_rotation(scene.sh_coeffs[parent], R, source, 1)))


def test_export_of_a_polygon_cage_frame(st):
    cage = PolyCageMesh.icosphere([0, 0, 0], 1.15, 3).displace_sinusoids(0.1, 8, seed=0)
    n = 2000
    scene = random_scene(n, seed=5)
    rng = np.random.default_rng(6)
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    scene.positions[:] = (d * (1.3 * rng.uniform(0, 1, n) ** (1 / 3))[:, None]).astype(f32)
    st.invalidate()
    st.upload_scene(scene)
    st.upload_cages(None)
    st.mvc_cage_upload(cage)
    st.mvc_bind()
    v, t = cage.rest_vertices.astype(np.float64), 0.7
    moved = (v + np.stack([0.25 * np.sin(2.0 * v[:, 1] + t), 0.15 * np.cos(1.5 * v[:, 0] - t),
                           0.2 * np.sin(v[:, 2] * 3.0 + 0.5 * t)], axis=1)).astype(f32)
    st.mvc_vertices_update(moved)
    cam = CameraUniforms.from_look_at((0, 0, 4), (0, 0, 0), (0, 1, 0), np.deg2rad(60), 320, 240, 0.2)
    comp = CompositorUniforms(320, 240, (0, 0, 0, 1), tuple(float(x) for x in cam.eye()), 3)
    t = st.execute_frame_gpu(scene, None, cam, comp, 1.15, 0.0, force_stage3=True)
    out = st.export_deformed(3)
    assert out.count == t.active_gaussians > n
    gidx, _ = st.mvc_read_bindings()
    R = st.read_buffer(_abi.BUF_MVC_ROTATIONS, f32).reshape(-1, 9)
    slot_of = np.full(n, -1, np.int64)
    slot_of[gidx] = np.arange(gidx.shape[0])
    meta = st.read_buffer(_abi.BUF_SPLIT_META, np.uint32).reshape(-1, 2)
    assert (meta[:, 1] == MVC_BOUND).all()
    parent = np.concatenate([np.arange(n), meta[:, 0].astype(np.int64)])
    source = slot_of[parent]
    want = expected_rotation(scene.sh_coeffs[parent], R, source, 3)
    np.testing.assert_array_equal(bits(out.sh_coeffs), bits(want))
    np.testing.assert_array_equal(bits(out.positions),
                                  bits(st.read_buffer(_abi.BUF_DEFORMED_POS, f32).reshape(-1, 3)))


def test_export_without_cages_is_the_rest_scene_and_ply_round_trips(st, tmp_path):
    st.invalidate()
    scene = random_scene(5000, seed=9)
    st.upload_scene(scene)
    st.upload_cages(None)
    out = st.export_deformed(3)
    np.testing.assert_array_equal(out.positions, scene.positions)
    np.testing.assert_array_equal(out.covariances_3d, scene.covariances_3d)
    np.testing.assert_array_equal(out.opacities, scene.opacities)
    np.testing.assert_array_equal(out.sh_coeffs, scene.sh_coeffs)
    # deformed PLY bytes of a tet frame reload to the exported scene
    scene2, cages = tet_setup(st, 20_000)
    cam = config0_camera(320, 180)
    st.execute_frame_gpu(scene2, cages, cam, compositor(320, 180, cam, deg=3), 1.1, 0.0)
    snap = st.export_deformed(3)
    path = tmp_path / "deformed.ply"
    st.export_deformed_ply(path, 3)
    loaded = ply.load_file(path)
    assert loaded.count == snap.count
    np.testing.assert_array_equal(loaded.positions, snap.positions)
    np.testing.assert_array_equal(loaded.sh_coeffs, snap.sh_coeffs)
    # A record keeps (scale >= 1e-4, rotation): the file holds the covariance
    # with its eigenvalues clamped to 1e-8 (to_raw_vertices, soa.rs:304-328),
    # which changes the split's indefinite children (f32 Cardano split,
    # deformation.rs:1120-1189) and nothing else.
    c = snap.covariances_3d.astype(np.float64)
    C = np.stack([np.stack([c[:, 0], c[:, 1], c[:, 2]], 1), np.stack([c[:, 1], c[:, 3], c[:, 4]], 1),
                  np.stack([c[:, 2], c[:, 4], c[:, 5]], 1)], 1)
    ev, V = np.linalg.eigh(C)
    P = np.einsum("nij,nj,nkj->nik", V, np.maximum(ev, 1e-8), V)
    proj = np.stack([P[:, 0, 0], P[:, 0, 1], P[:, 0, 2], P[:, 1, 1], P[:, 1, 2], P[:, 2, 2]], 1)
    rel = np.abs(loaded.covariances_3d - proj).max(axis=1) / np.abs(proj).max(axis=1)
    assert rel.max() < 1e-5
    # moving the cage without a frame leaves no deformed scene to export
    cages.cages[0].simulator.current_positions = (
        cages.cages[0].simulator.current_positions * f32(1.01)).astype(f32)
    st.sync_scene_and_cages(scene2, cages)
    with pytest.raises(_abi.CgsError) as e:
        st.export_deformed(3)
    assert e.value.code == _abi.CGS_E_STATE
