"""Parity at the benchmark sizes: the frames behind the reported numbers,
checked against the oracle (v2 mode) at full size.

* the tet-cage frame exactly as bench.py renders it: 1,100,000 Gaussians,
  1920x1080, the 750-tet spring cage after a few solver steps (GPU binding,
  Stage 1 positions/covariances/opacities, Stage 2 records and extents, Stage
  3 offsets/keys/ids/ranges bit-exact over ~26M tile entries, RGB <= 2e-3);
* frames alternating 640x360 and 1920x1080 on a 1M-Gaussian scene (the splat
  depth sort changes digit width between them: 8 bits at 360p, 7 at 1080p);
* the quantized (f16) scene ingest against the oracle fed the dequantized
  f32 arrays;
* one mixed-resolution step of cgs_execute_views (640x360, 1280x720,
  1920x1080), each view against the oracle;
* a 7680x4320 frame (129,600 tiles, 64-bit keys) of the large multi-cage
  scene on a Gaussian subsample, with its four spring-driven tet cages;
* the 3M-Gaussian polygon-cage (MVC) frame: exact stored bindings against the
  oracle on a sample, the learned field against the exact frame.
"""
import numpy as np
import pytest

import oracle
from cindergs_b200 import (CageScene, GpuPipelineState, QuantizedGaussianSceneSoa, random_scene,
                           workloads)
from cindergs_b200 import _abi
from helpers import assert_stage23_exact, compositor, config0_camera, gpu_buffers, oracle_frame

pytestmark = pytest.mark.gpu
RGB_TOL = 2e-3


def bits(a):
    return np.asarray(a, np.float32).view(np.uint32)


def cage_dict(cages):
    elems, inv, nverts, bt, bw = cages.flatten()
    return dict(verts=cages.flat_vertices(), elems=elems, inv_dm=inv, bind_tet=bt, bind_w=bw)


def stage1_buffers(st):
    return dict(pos=st.read_buffer(_abi.BUF_DEFORMED_POS, np.float32),
                cov=st.read_buffer(_abi.BUF_DEFORMED_COV, np.float32),
                opa=st.read_buffer(_abi.BUF_DEFORMED_OPA, np.float32))


@pytest.fixture(scope="module")
def st():
    s = GpuPipelineState(0)
    yield s
    s.close()


def test_bench_frame_full_size(st):
    wl = workloads.tet_cage_orbit()
    st.upload_scene(wl.scene)
    cages = wl.bind(st)
    mesh = wl.cage.mesh
    ot, ow = oracle.bind_points(wl.scene.positions, mesh.rest_vertices, mesh.elements,
                                mesh.inv_dm, mesh.bounds())
    np.testing.assert_array_equal(cages.bind_tet, ot, err_msg="bound tets")
    np.testing.assert_array_equal(bits(cages.bind_w), bits(ow), err_msg="barycentric weights")
    for _ in range(3):
        wl.step()
    cam = wl.camera(3)
    comp = wl.compositor(cam)
    t = st.execute_frame_gpu(wl.scene, cages, cam, comp, wl.strain_split_threshold,
                             wl.mip_filter_3d_var, 1.0 / 255.0, 0.5, force_stage3=True,
                             write_f32=True)
    g = gpu_buffers(st)
    g.update(stage1_buffers(st))
    img = st.readback_framebuffer_f32(wl.width, wl.height)
    o = oracle_frame(wl.scene, cam, comp, cage=cage_dict(cages), mip=wl.mip_filter_3d_var,
                     split_thr=wl.strain_split_threshold)
    n = wl.scene.count
    assert t.active_gaussians == n + o["splits"]
    assert t.total_tile_entries == o["entries"] > 20_000_000
    np.testing.assert_array_equal(bits(g["pos"][:3 * n]), bits(o["def_pos"][:3 * n]),
                                  err_msg="deformed positions")
    np.testing.assert_array_equal(bits(g["cov"][:6 * n]), bits(o["def_cov"][:6 * n]),
                                  err_msg="deformed covariances")
    np.testing.assert_array_equal(bits(g["opa"][:n]), bits(o["def_opa"][:n]),
                                  err_msg="deformed opacities")
    assert_stage23_exact(g, o)
    err = float(np.abs(img - o["rgba_f32"]).max())
    assert err <= RGB_TOL, err


def test_alternating_resolutions_1m(st):
    """360p (8-bit splat-sort digits) and 1080p (7-bit digits) frames in turn:
    each sort reads look-back words that the previous, differently wide
    sort left behind, so every frame checks that they were cleared."""
    scene = random_scene(1_000_000, seed=4)
    st.upload_scene(scene)
    st.upload_cages(None)
    for i, (w, h) in enumerate([(640, 360), (1920, 1080), (640, 360), (1920, 1080)]):
        cam = config0_camera(w, h)
        comp = compositor(w, h, cam, deg=3, bg=(0.0, 0.0, 0.0, 1.0))
        t = st.execute_frame_gpu(scene, None, cam, comp, force_stage3=True, write_f32=True)
        g = gpu_buffers(st)
        img = st.readback_framebuffer_f32(w, h)
        o = oracle_frame(scene, cam, comp)
        assert t.total_tile_entries == o["entries"] > 1_000_000, (i, w, h)
        assert_stage23_exact(g, o)
        assert float(np.abs(img - o["rgba_f32"]).max()) <= RGB_TOL, (i, w, h)


def test_quantized_frame_vs_oracle(st):
    """The f16 ingest (cgs_scene_upload_quantized: covariance pairs and
    degree-3 SH decoded on the GPU) renders what the oracle renders from the
    dequantized arrays (binary16 -> binary32 is exact)."""
    q = QuantizedGaussianSceneSoa.from_soa(random_scene(300_000, seed=8, box=1.0), 3)
    # the reference's f16 decode cases (tests/gpu_parity_tests.rs:1268-1293)
    # in the first splats: subnormal, negative subnormal, signed zero and
    # max-finite halves
    h = lambda x: int(np.float16(x).view(np.uint16))  # noqa: E731
    cases = np.array([[h(0.05), 0x0001, 0x8001, h(0.04), 0x03FF, h(0.06)],
                      [h(12.5), h(-0.75), 0x8000, h(8.0), 0x0000, h(10.0)],
                      [0x7BFF, 0, 0, h(1.0), 0, h(1.0)]], np.uint32)
    q.covariances_f16_packed[:3] = cases[:, 0::2] | (cases[:, 1::2] << 16)
    deq = q.to_soa()
    st.upload_scene(q)
    st.upload_cages(None)
    cam = config0_camera(1920, 1080)
    comp = compositor(1920, 1080, cam, deg=3, bg=(0.0, 0.0, 0.0, 1.0))
    t = st.execute_frame_gpu(q, None, cam, comp, force_stage3=True, write_f32=True)
    g = gpu_buffers(st)
    img = st.readback_framebuffer_f32(1920, 1080)
    o = oracle_frame(deq, cam, comp)
    assert t.total_tile_entries == o["entries"] > 1_000_000
    assert_stage23_exact(g, o)
    assert float(np.abs(img - o["rgba_f32"]).max()) <= RGB_TOL


def test_mixed_resolution_views_vs_oracle(st):
    wl, cams, comps = workloads.multiview_cage(n=400_000, views=3)
    st.upload_scene(wl.scene)
    cages = wl.bind(st)
    for _ in range(2):
        wl.step()
    imgs = st.view_images(comps)
    for use_graph in (False, True, True):  # eager, capture, replay
        stats = st.execute_views(wl.scene, cages, cams, comps, imgs, use_graph=use_graph)
        assert stats["total_tile_entries"] > 0
        for v, (cam, comp) in enumerate(zip(cams, comps)):
            got = imgs[v].cpu().numpy().view(np.uint8).reshape(comp.screen_height,
                                                               comp.screen_width, 4)
            o = oracle_frame(wl.scene, cam, comp, cage=cage_dict(cages))
            d = np.abs(got.astype(np.int32) - o["rgba8"].astype(np.int32))
            assert d.max() <= 1, (use_graph, v, d.max())
        wl.step()


def test_8k_64bit_multicage_subsample(st):
    """The large workload's geometry (four 384-tet spring cages over the upper
    half, 7680x4320, 129,600 tiles, 64-bit keys) on 400,000 of its Gaussians;
    the quantized layout and the learned polygon cage are checked by their own
    tests."""
    wl = workloads.large_multicage(n=400_000, radius=8.0)  # ~29M entries: the oracle's size
    scene = wl.scene.to_soa()
    st.upload_scene(scene)
    cs = CageScene.auto_bind(wl.cages, st, scene.count)
    cs.step(1.0 / 60.0)
    cs.step(1.0 / 60.0)
    cam = wl.camera(2)
    comp = wl.compositor(cam)
    t = st.execute_frame_gpu(scene, cs, cam, comp, force_stage3=True, write_f32=True)
    assert t.used_64bit_keys
    g = gpu_buffers(st, key64=True)
    img = st.readback_framebuffer_f32(wl.width, wl.height)
    o = oracle_frame(scene, cam, comp, cage=cage_dict(cs))
    assert t.total_tile_entries == o["entries"] > 1_000_000
    assert_stage23_exact(g, o, key64=True)
    assert float(np.abs(img - o["rgba_f32"]).max()) <= RGB_TOL


def test_mvc_polygon_cage_full_size(st):
    """The polygon-cage workload at its benchmark size: 3,000,000 Gaussians in
    the unit ball, the 642-vertex displaced icosphere cage, 1920x1080.
    Exact stored bindings: the deformed means and covariances of a
    10,000-Gaussian sample against the oracle's deform_scene_cpu restatement
    with the oracle's own bindings (its weights agree with the GPU's to 5e-5,
    so the comparison is statistical). Learned field, trained as the
    benchmark trains it: the error of its frame against the exact frame, and
    the per-frame network against the cached codes on the same frame."""
    import torch
    n = 3_000_000
    wl = workloads.mvc_cage_sphere(n=n)
    st.upload_scene(wl.scene)
    st.upload_cages(None)
    st.mvc_cage_upload(wl.cage)
    assert st.mvc_bind() > 0
    verts = wl.vertices(1)
    cam = wl.camera(1)
    comp = wl.compositor(cam)

    def frame():
        st.mvc_vertices_update(verts)
        st.execute_frame_gpu(wl.scene, None, cam, comp, 0.0, 0.0, force_stage3=True)
        pos = st.read_buffer(_abi.BUF_DEFORMED_POS, np.float32).reshape(-1, 3)[:n].copy()
        cov = st.read_buffer(_abi.BUF_DEFORMED_COV, np.float32).reshape(-1, 6)[:n].copy()
        return pos, cov

    pos_e, cov_e = frame()
    sidx = np.sort(np.random.default_rng(3).choice(n, 10_000, replace=False))
    inside, wg = oracle.mvc_bind(wl.scene.positions[sidx], wl.cage.rest_vertices,
                                 wl.cage.triangles)
    o = oracle.mvc_deform(wl.scene.positions[sidx], wl.scene.covariances_3d[sidx],
                          wl.scene.opacities[sidx], inside, wg, verts)
    m = len(sidx)
    dp = np.linalg.norm(pos_e[sidx].astype(np.float64) - o["pos"][:m], axis=1)
    print(f"\nexact MVC at 3M vs oracle (10k sample): position mean {dp.mean():.2e} "
          f"p99.9 {np.quantile(dp, 0.999):.2e} max {dp.max():.2e}")
    assert dp.mean() < 1e-5 and np.quantile(dp, 0.999) < 1e-4 and dp.max() < 1e-3
    out = ~inside.astype(bool)
    np.testing.assert_array_equal(pos_e[sidx][out], wl.scene.positions[sidx][out])
    scale = np.abs(o["cov"][:m]).max(axis=1) + 1e-30
    dc = np.abs(cov_e[sidx].astype(np.float64) - o["cov"][:m]).max(axis=1) / scale
    # covariances go through F = sum_j v_j grad(w_j)^T, whose central
    # differences divide the weights' 5e-5 agreement by 2h (h = 1e-3 x the
    # cage diagonal)
    assert dc.mean() < 1e-3 and dc.max() < 1e-2, (dc.mean(), dc.max())

    pts = torch.from_numpy(wl.training_points(2_000_000)).to("cuda:0")
    w = st.mvc_weights(pts)
    st.mvc_field_create(seed=1)
    st.mvc_field_train(pts, w, steps=6000, batch=4096, lr=2e-3, lam=0.05, seed=5)
    del w, pts
    torch.cuda.empty_cache()
    _, _, enc = st.mvc_field_layout()
    s = 1.0 / float(enc[3])
    sample = wl.scene.positions[np.random.default_rng(7).choice(n, 200_000, replace=False)]
    raw, _ = st.mvc_field_infer(sample, rest=True)
    thr = float(np.quantile(np.linalg.norm(raw - sample, axis=1) / s, 0.99))
    st.mvc_bind_learned(thr, per_frame=True)
    pos_pf, _ = frame()
    st.mvc_bind_learned(thr)
    pos_l, _ = frame()
    mode = np.linalg.norm(pos_l.astype(np.float64) - pos_pf, axis=1) / s
    err = np.linalg.norm(pos_l.astype(np.float64) - pos_e, axis=1) / s
    print(f"learned at 3M: error vs exact mean {err.mean():.2e} p99 {np.quantile(err, 0.99):.2e} "
          f"max {err.max():.2e} (of s); per-frame network vs codes max {mode.max():.2e}")
    assert mode.max() < 1e-6
    assert err.mean() < 1e-3 and np.quantile(err, 0.99) < 4e-3
