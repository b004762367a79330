"""Polygon-cage MVC on the GPU against the oracle's restatement of
deformation/mvc.rs: exact weights (special cases included), the bindings
(inside test, weights, central-difference gradients) and the Stage 1
deformation of bound Gaussians, including strain splits and the 3D Mip filter.

Tolerances: weights and bindings differ from the host only through the
transcendentals (asin, sin, atan2 on the device vs glibc). Each f32 evaluation
is up to ~3e-5 from an f64 one on these cages, so the two agree to 1e-4, the
device is checked to be no farther from f64 than the host, and gradients,
which divide weight differences by 2h, agree to 5e-5 / h.
Deformed means and covariances are compared on identical bindings at the
north-star bar of 1e-5 relative.
"""
import numpy as np
import pytest

import oracle
from cindergs_b200 import (CameraUniforms, CompositorUniforms, GaussianSceneSoa, GpuPipelineState,
                           PolyCageMesh, random_scene)
from cindergs_b200 import _abi

pytestmark = pytest.mark.gpu
f32 = np.float32


def workload_cage():
    return PolyCageMesh.icosphere([0, 0, 0], 1.15, 3).displace_sinusoids(0.1, 8, seed=0)


def ball_points(n, seed, radius=1.0):
    rng = np.random.default_rng(seed)
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    r = radius * rng.uniform(0, 1, n) ** (1.0 / 3.0)
    return (d * r[:, None]).astype(f32)


@pytest.fixture(scope="module")
def st():
    s = GpuPipelineState(0)
    yield s
    s.close()


@pytest.mark.parametrize("which", ["box", "octahedron", "workload"])
def test_exact_weights_match_oracle(st, which):
    cage = {"box": PolyCageMesh.create_box_surface_cage([-1.0, -2.0, -0.5], [2.0, 1.5, 2.5]),
            "octahedron": PolyCageMesh.create_octahedron_cage([0.3, -0.2, 0.4], 2.0),
            "workload": workload_cage()}[which]
    st.mvc_cage_upload(cage)
    pts = ball_points(300, seed=3, radius=0.9)
    # special points: a cage vertex, a face centroid, a point outside
    v = cage.rest_vertices
    t = cage.triangles[0]
    pts = np.concatenate([pts, v[5:6], ((v[t[0]] + v[t[1]] + v[t[2]]) / 3)[None],
                          np.array([[4.0, 0.5, 0.0]], f32)]).astype(f32)
    g = st.mvc_weights(pts)
    o = oracle.mvc_weights(pts, v, cage.triangles)
    # Only points inside the cage are ever bound; outside, the formula cancels
    # badly (even the host's f32 result is ~1e-3 from f64 there).
    inside = np.abs(cage.winding_numbers(pts)) >= 0.5
    assert inside[300] and not inside[302]  # the cage vertex is in, (4, 0.5, 0) is out
    np.testing.assert_allclose(g[inside], o[inside], atol=1e-4, rtol=0)
    # error floor: both f32 evaluations against f64 (the device's asin/sin and
    # glibc's differ in the last bits; neither is closer to f64 by much)
    e64 = mvc_weights_f64(pts[inside], v, cage.triangles)
    err_gpu, err_orc = np.abs(g[inside] - e64).max(), np.abs(o[inside] - e64).max()
    assert err_gpu <= 2.0 * err_orc + 1e-6, (err_gpu, err_orc)
    assert np.abs(g[inside].sum(1) - 1.0).max() < 1e-4
    rec = g[inside] @ v
    assert np.linalg.norm(rec - pts[inside], axis=1).max() < 2e-4
    assert abs(g[300, 5] - 1.0) < 1e-6  # the vertex itself


def mvc_weights_f64(points, verts, tris):
    """compute_mvc_weights (mvc.rs:366-471) in float64: the error floor."""
    v = verts.astype(np.float64)
    out = np.zeros((len(points), len(v)))
    for k, x in enumerate(np.asarray(points, np.float64)):
        diff = v - x
        d = np.linalg.norm(diff, axis=1)
        if (d < 1e-6).any():
            out[k, np.argmax(d < 1e-6)] = 1.0
            continue
        u = diff / d[:, None]
        i0, i1, i2 = tris[:, 0], tris[:, 1], tris[:, 2]
        l0 = np.linalg.norm(u[i1] - u[i2], axis=1)
        l1 = np.linalg.norm(u[i2] - u[i0], axis=1)
        l2 = np.linalg.norm(u[i0] - u[i1], axis=1)
        t0, t1, t2 = (2 * np.arcsin(np.clip(l * 0.5, 0, 1)) for l in (l0, l1, l2))
        h = 0.5 * (t0 + t1 + t2)
        bnd = np.abs(np.pi - h) < 1e-5
        if bnd.any():
            f = np.argmax(bnd)
            w = np.array([np.sin(t0[f]) * d[i1[f]] * d[i2[f]], np.sin(t1[f]) * d[i2[f]] * d[i0[f]],
                          np.sin(t2[f]) * d[i0[f]] * d[i1[f]]])
            out[k, [i0[f], i1[f], i2[f]]] = w / w.sum()
            continue
        s0, s1, s2 = np.sin(t0), np.sin(t1), np.sin(t2)
        sh = np.sin(h)
        c0 = np.clip(2 * sh * np.sin(h - t0) / (s1 * s2) - 1, -1, 1)
        c1 = np.clip(2 * sh * np.sin(h - t1) / (s2 * s0) - 1, -1, 1)
        c2 = np.clip(2 * sh * np.sin(h - t2) / (s0 * s1) - 1, -1, 1)
        sg = np.where(np.einsum("ij,ij->i", u[i2], np.cross(u[i0], u[i1])) >= 0, 1.0, -1.0)
        q0, q1, q2 = (sg * np.sqrt(np.maximum(1 - c * c, 0)) for c in (c0, c1, c2))
        ok = ~((np.abs(s0) < 1e-6) | (np.abs(s1) < 1e-6) | (np.abs(s2) < 1e-6) |
               (np.abs(q0) <= 1e-6) | (np.abs(q1) <= 1e-6) | (np.abs(q2) <= 1e-6))
        m0 = (t0 - c1 * t2 - c2 * t1) / (2 * d[i0] * s1 * q2)
        m1 = (t1 - c2 * t0 - c0 * t2) / (2 * d[i1] * s2 * q0)
        m2 = (t2 - c0 * t1 - c1 * t0) / (2 * d[i2] * s0 * q1)
        w = np.zeros(len(v))
        np.add.at(w, i0[ok], m0[ok])
        np.add.at(w, i1[ok], m1[ok])
        np.add.at(w, i2[ok], m2[ok])
        out[k] = w / w.sum()
    return out


def mvc_scene(n, seed):
    rng = np.random.default_rng(seed)
    scene = random_scene(n, seed=seed)
    pts = ball_points(n, seed + 1, radius=1.3)  # some outside the cage
    scene.positions[:] = pts
    return scene


def cage_motion(cage, t):
    v = cage.rest_vertices.astype(np.float64)
    d = np.stack([0.25 * np.sin(2.0 * v[:, 1] + t), 0.15 * np.cos(1.5 * v[:, 0] - t),
                  0.2 * np.sin(v[:, 2] * 3.0 + 0.5 * t)], axis=1)
    return (v + d).astype(f32)


def test_bindings_match_oracle(st):
    cage = workload_cage()
    scene = mvc_scene(600, seed=11)
    st.upload_scene(scene)
    st.upload_cages(None)
    st.mvc_cage_upload(cage)
    nb = st.mvc_bind()
    inside_o, wg_o = oracle.mvc_bind(scene.positions, cage.rest_vertices, cage.triangles)
    assert nb == int(inside_o.sum()) > 0
    gidx, wg = st.mvc_read_bindings()
    np.testing.assert_array_equal(gidx, np.nonzero(inside_o)[0])
    np.testing.assert_allclose(wg[..., 0], wg_o[inside_o][..., 0], atol=5e-5, rtol=0)
    # central differences divide weight differences by 2h (h = 1e-3 x the
    # cage diagonal): the weights' 5e-5 becomes 5e-5 / h on the gradients
    h = oracle.mvc_step(cage.rest_vertices)
    np.testing.assert_allclose(wg[..., 1:], wg_o[inside_o][..., 1:], atol=5e-5 / h, rtol=0)


def deformed_arrays(st):
    pos = st.read_buffer(_abi.BUF_DEFORMED_POS, np.float32).reshape(-1, 3)
    cov = st.read_buffer(_abi.BUF_DEFORMED_COV, np.float32).reshape(-1, 6)
    opa = st.read_buffer(_abi.BUF_DEFORMED_OPA, np.float32)
    return pos, cov, opa


@pytest.mark.parametrize("split,mip", [(0.0, 0.0), (1.15, 0.0), (1.15, 0.001)])
def test_deformation_matches_oracle(st, split, mip):
    cage = workload_cage()
    scene = mvc_scene(2000, seed=5)
    st.upload_scene(scene)
    st.upload_cages(None)
    st.mvc_cage_upload(cage)
    st.mvc_bind()
    deformed = cage_motion(cage, 0.7)
    st.mvc_vertices_update(deformed)
    cam = CameraUniforms.from_look_at((0, 0, 4), (0, 0, 0), (0, 1, 0), np.deg2rad(60), 320, 240,
                                      0.2)
    comp = CompositorUniforms(320, 240, (0, 0, 0, 1), tuple(float(x) for x in cam.eye()), 3)
    st.execute_frame_gpu(scene, None, cam, comp, split, mip, force_stage3=True)
    gidx, wg = st.mvc_read_bindings()
    inside = np.zeros(scene.count, np.uint8)
    inside[gidx] = 1
    wg_full = np.zeros((scene.count, cage.num_vertices, 4), f32)
    wg_full[gidx] = wg
    o = oracle.mvc_deform(scene.positions, scene.covariances_3d, scene.opacities, inside, wg_full,
                          deformed, split_thr=split, mip=mip)
    pos, cov, opa = deformed_arrays(st)
    assert pos.shape[0] == o["pos"].shape[0]
    if split > 0:
        assert pos.shape[0] > scene.count  # the motion stretches some regions beyond 1.15
    # bound Gaussians: identical sums in the reference order -> identical means
    b = inside.astype(bool)
    np.testing.assert_array_equal(pos[:scene.count][b], o["pos"][:scene.count][b])
    scale = np.abs(o["cov"]).max(axis=1, keepdims=True)
    np.testing.assert_allclose(cov / scale, o["cov"] / scale, atol=1e-5, rtol=0)
    np.testing.assert_allclose(pos, o["pos"], rtol=1e-5, atol=1e-6)
    np.testing.assert_allclose(opa, o["opa"], rtol=1e-5, atol=1e-6)
    R = st.read_buffer(_abi.BUF_MVC_ROTATIONS, np.float32).reshape(-1, 9)
    np.testing.assert_allclose(R, o["R"][gidx], atol=1e-5)


def test_tet_bindings_win_over_the_polygon_cage(st):
    """Gaussians bound to a tet cage are not bound to the polygon cage."""
    from cindergs_b200 import Cage, CageScene, TetMesh
    cage = workload_cage()
    scene = mvc_scene(500, seed=9)
    st.upload_scene(scene)
    tet = Cage("inner", TetMesh.create_box_cage([-0.3, -0.3, -0.3], [0.3, 0.3, 0.3]))
    cs = CageScene.auto_bind([tet], st, scene.count)
    st.sync_scene_and_cages(scene, cs)
    st.mvc_cage_upload(cage)
    nb = st.mvc_bind()
    tet_bound = cs.bind_cage != 0xFFFFFFFF
    inside_o, _ = oracle.mvc_bind(scene.positions, cage.rest_vertices, cage.triangles)
    assert tet_bound.sum() > 0
    assert nb == int((inside_o & ~tet_bound).sum())
