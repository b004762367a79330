"""Learned MVC weight field on the GPU against the oracle's restatement
(oracle/mvc_field.py) and against exact MVC.

Gradients of one batch agree with the oracle's float64 backward pass (which
rounds to bf16 where the kernels do) to 2% per parameter block: the two sides
round fp32 sums that differ in the last bits, so an occasional bf16 rounding
goes the other way. Weights and the fused inference agree with the oracle
within the bounds below, measured relative to the cage half-extent s (the
position) or the largest entry of the oracle's gradient (F).

Training is checked by what it gains: on held-out interior points the trained
network's deformed positions are compared with exact MVC on deformed cages,
against the same weights without the network (an untrained network's outputs
are ~uniform, and their linear-precision projection is the best affine
approximation of the cage motion). Frames with learned bindings keep the
residual fallbacks bit-identical to the exact bindings.
"""
import numpy as np
import pytest

import oracle
from oracle import mvc_field as of
from cindergs_b200 import CameraUniforms, CompositorUniforms, GpuPipelineState
from cindergs_b200 import _abi
from test_gpu_mvc import ball_points, cage_motion, mvc_scene, workload_cage

pytestmark = pytest.mark.gpu
f32 = np.float32


@pytest.fixture(scope="module")
def fst():
    s = GpuPipelineState(0)
    cage = workload_cage()
    s.mvc_cage_upload(cage)
    s.mvc_field_create(seed=7)
    yield s, cage
    s.close()


def inside_points(cage, n, seed, radius=1.0):
    p = ball_points(4 * n, seed, radius)
    p = p[np.abs(cage.winding_numbers(p)) >= 0.5]
    assert len(p) >= n
    return np.ascontiguousarray(p[:n])


def perturbed_params(st, seed):
    """A network with non-trivial outputs (the initial output layer is ~0)."""
    st.mvc_field_create(seed=seed)
    off, tot, enc = st.mvc_field_layout()
    p = st.mvc_field_params().astype(np.float64)
    V = st._mvc_V
    rng = np.random.default_rng(seed)
    p[off["W5"]:off["W5"] + V * 128] = rng.normal(0, 0.02, V * 128)
    for k in ("b1", "b2", "b3", "b4"):
        p[off[k]:off[k] + 128] = rng.normal(0, 0.1, 128)
    p[off["b5"]:off["b5"] + V] += rng.normal(0, 1e-3, V)
    p = p.astype(f32)
    st.mvc_field_params(p)
    return of.unpack(p, off, V), off, enc


def test_gradients_match_oracle(fst):
    st, cage = fst
    P, off, enc = perturbed_params(st, seed=3)
    pts = inside_points(cage, 256, seed=21)
    w = st.mvc_weights(pts)
    g, loss = st.mvc_field_grads(pts, w, lam=1.0)
    (lw, lr), go = of.loss_and_grads(P, pts, w, cage.rest_vertices, enc, 1.0)
    assert abs(loss[0] - lw) <= 1e-3 * lw and abs(loss[1] - lr) <= 1e-3 * lr + 1e-9, (loss, lw, lr)
    V = cage.num_vertices
    for k in of.NAMES:
        n = go[k].size
        gk = g[off[k]:off[k] + n].astype(np.float64)
        ref = go[k].reshape(-1)
        rel = np.linalg.norm(gk - ref) / np.linalg.norm(ref)
        assert rel < 2e-2, (k, rel)
    assert V == P["W5"].shape[0]


def test_eval_and_inference_match_oracle(fst):
    st, cage = fst
    P, off, enc = perturbed_params(st, seed=5)
    s = 1.0 / float(enc[3])
    pts = inside_points(cage, 2000, seed=22)
    w = st.mvc_field_eval(pts)
    wo = of.weights(P, pts, enc, cage.rest_vertices)
    # a layer input whose fp32 and f64 values round to different bf16 values
    # moves every later activation of that point: rare, so bound the mean,
    # the 99th percentile of per-point maxima, and loosely the maximum
    dw = np.abs(w - wo)
    q99 = np.quantile(dw.max(axis=1), 0.99)
    assert dw.mean() < 1e-5 and q99 < 2e-4 and dw.max() < 5e-3, (dw.mean(), q99, dw.max())
    np.testing.assert_allclose(w.sum(1), 1.0, atol=1e-5)
    lp = np.linalg.norm(w.astype(np.float64) @ cage.rest_vertices - pts, axis=1) / s
    assert lp.max() < 2e-5, lp.max()  # linear precision by construction
    deformed = cage_motion(cage, 0.7)
    st.mvc_vertices_update(deformed)
    pos, F = st.mvc_field_infer(pts)
    po, Fo = of.position_and_jacobian(P, pts, deformed, enc, cage.rest_vertices)
    dp = np.linalg.norm(pos - po, axis=1) / s
    print(f"\nfield inference vs oracle: position mean {dp.mean():.2e} "
          f"p99 {np.quantile(dp, 0.99):.2e} max {dp.max():.2e} (of s)")
    assert dp.mean() < 2e-4 and np.quantile(dp, 0.99) < 1e-3 and dp.max() < 1e-2, dp.max()
    Fscale = np.abs(Fo).max()
    dF = np.abs(F - Fo).max(axis=(1, 2)) / Fscale
    print(f"gradient F: mean {dF.mean():.2e} p99 {np.quantile(dF, 0.99):.2e} max {dF.max():.2e} "
          f"(of max |F|)")
    assert dF.mean() < 1e-3 and np.quantile(dF, 0.99) < 1e-2 and dF.max() < 5e-2, dF.max()
    # the folded output layer reproduces sum_j w_j v'_j of the evaluated weights
    rec = w.astype(np.float64) @ deformed.astype(np.float64)
    assert (np.linalg.norm(pos - rec, axis=1) / s).mean() < 2e-5
    # the network's own rest position (residual diagnostic)
    pr, Fr = st.mvc_field_infer(pts, rest=True)
    pro, Fro = of.position_and_jacobian(P, pts, None, enc, cage.rest_vertices)
    dr = np.linalg.norm(pr - pro, axis=1) / s
    assert dr.mean() < 2e-4 and np.quantile(dr, 0.99) < 1e-3, (dr.mean(), dr.max())
    st.mvc_vertices_update(cage.rest_vertices)


def relative_position_error(st, cage, pts, deformed, s):
    """Mean |x'_learned - x'_exact| / s on a deformed cage."""
    st.mvc_vertices_update(deformed)
    pos, _ = st.mvc_field_infer(pts)
    exact = st.mvc_weights(pts).astype(np.float64) @ deformed.astype(np.float64)
    st.mvc_vertices_update(cage.rest_vertices)
    return float((np.linalg.norm(pos - exact, axis=1) / s).mean())


@pytest.fixture(scope="module")
def trained(fst):
    st, cage = fst
    st.mvc_field_create(seed=11)
    _, _, enc = st.mvc_field_layout()
    s = 1.0 / float(enc[3])
    test_pts = inside_points(cage, 4000, seed=23)
    motions = {"sinusoids 0.1": cage.displace_sinusoids(0.1, 8, seed=1).rest_vertices,
               "large motion": cage_motion(cage, 0.7)}
    err0 = {k: relative_position_error(st, cage, test_pts, d, s) for k, d in motions.items()}
    train_pts = inside_points(cage, 65536, seed=24)
    w = st.mvc_weights(train_pts)
    loss = st.mvc_field_train(train_pts, w, steps=3000, batch=4096, lr=2e-3, lam=0.05, seed=5)
    err1 = {k: relative_position_error(st, cage, test_pts, d, s) for k, d in motions.items()}
    return dict(err0=err0, err1=err1, loss=loss, s=s, deformed=motions["large motion"])


def test_training_gain(fst, trained):
    """The trained network is far closer to exact MVC than the same weights
    without it (the affine approximation)."""
    for k in trained["err0"]:
        print(f"\nlearned field, {k}: mean relative position error {trained['err0'][k]:.3e} "
              f"without the network -> {trained['err1'][k]:.3e} trained; "
              f"loss terms {trained['loss']}")
        assert trained["err1"][k] < 0.1 * trained["err0"][k], trained
    assert trained["err1"]["sinusoids 0.1"] < 2e-3, trained
    assert trained["err1"]["large motion"] < 5e-3, trained


def frame_positions(st, scene):
    cam = CameraUniforms.from_look_at((0, 0, 4), (0, 0, 0), (0, 1, 0), np.deg2rad(60), 320, 240,
                                      0.2)
    comp = CompositorUniforms(320, 240, (0, 0, 0, 1), tuple(float(x) for x in cam.eye()), 3)
    st.execute_frame_gpu(scene, None, cam, comp, 0.0, 0.0, force_stage3=True)
    pos = st.read_buffer(_abi.BUF_DEFORMED_POS, np.float32).reshape(-1, 3)
    cov = st.read_buffer(_abi.BUF_DEFORMED_COV, np.float32).reshape(-1, 6)
    return pos, cov


def test_learned_bindings_in_the_frame(fst, trained):
    st, cage = fst
    s = trained["s"]
    # 90% of the Gaussians in the unit ball (the training domain), the rest
    # outside the cage
    scene = mvc_scene(3000, seed=31)
    pts = ball_points(3000, seed=32, radius=1.0)
    rng = np.random.default_rng(33)
    far = rng.random(3000) < 0.1
    pts[far] *= (1.45 / np.maximum(np.linalg.norm(pts[far], axis=1), 1e-3))[:, None]
    scene.positions[:] = pts
    st.upload_scene(scene)
    st.upload_cages(None)
    deformed = trained["deformed"]
    nb_exact = st.mvc_bind()
    gall, _ = st.mvc_read_bindings()
    inside = np.zeros(scene.count, bool)
    inside[gall] = True
    st.mvc_vertices_update(deformed)
    pos_e, cov_e = frame_positions(st, scene)
    # everything a fallback: the exact frame, bit for bit
    nb, nfb = st.mvc_bind_learned(threshold=0.0)
    assert nb == nb_exact and nfb == nb
    pos0, cov0 = frame_positions(st, scene)
    np.testing.assert_array_equal(pos0, pos_e)
    np.testing.assert_array_equal(cov0, cov_e)
    # nothing a fallback
    nb, nfb = st.mvc_bind_learned(threshold=1e9)
    assert nb == nb_exact and nfb == 0
    pos1, _ = frame_positions(st, scene)
    # residual-triggered fallbacks keep exact positions: a threshold at the
    # 90th percentile of the residuals sends about a tenth back to exact MVC
    raw, _ = st.mvc_field_infer(scene.positions[gall], rest=True)
    res = np.linalg.norm(raw - scene.positions[gall], axis=1) / s
    thr = float(np.quantile(res, 0.9))
    nb, nfb = st.mvc_bind_learned(threshold=thr, per_frame=True)
    assert nb == nb_exact and abs(nfb - int((res > thr).sum())) <= 2, (nfb, (res > thr).sum())
    pos3, cov3 = frame_positions(st, scene)
    # default: codes kept per Gaussian, output layer per frame -- the same
    # deformation up to summation order
    nb, nfb2 = st.mvc_bind_learned(threshold=thr)
    assert nfb2 == nfb
    pos2, cov2 = frame_positions(st, scene)
    d = np.linalg.norm(pos2 - pos3, axis=1) / s
    assert d.max() < 1e-6, d.max()
    cs = np.abs(cov3).max(axis=1, keepdims=True) + 1e-30
    assert (np.abs(cov2 - cov3) / cs).max() < 1e-5
    gidx, _ = st.mvc_read_bindings()
    assert len(gidx) == nfb
    np.testing.assert_array_equal(pos2[gidx], pos_e[gidx])
    np.testing.assert_array_equal(cov2[gidx], cov_e[gidx])
    out = ~inside
    np.testing.assert_array_equal(pos2[out], pos_e[out])
    e1 = np.linalg.norm(pos1[inside] - pos_e[inside], axis=1) / s
    e2 = np.linalg.norm(pos2[inside] - pos_e[inside], axis=1) / s
    print(f"\nlearned bindings: {nb} bound, {nfb} fallbacks at residual {thr:.3e}; mean "
          f"relative position error {e1.mean():.3e} (no fallback), {e2.mean():.3e} (with)")
    assert e2.mean() <= e1.mean() + 1e-9
    assert e1.mean() < 5e-3 and e2.mean() < 5e-3
    scale = np.abs(cov_e[inside]).max(axis=1, keepdims=True)
    dc = np.abs(cov2[inside] - cov_e[inside]) / scale
    assert dc.mean() < 5e-2, dc.mean()
    st.mvc_vertices_update(cage.rest_vertices)
