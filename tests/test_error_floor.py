"""The float64 error-floor evaluation (cindergs_b200.error_floor) restates
the same formulas as the f32 frame: on the tet-cage workload its Stage 1
Jacobians, polar rotations, deformed means, covariances and opacities and its
Stage 2 centres, conics, alphas and colours agree with the oracle's f32 v2
frame to within f32 rounding, and its compositor reproduces the oracle's
image to within the 2e-3 RGB tolerance. (The floor then measures how far the
f32 results lie from these f64 values.)"""
import numpy as np

import oracle
from cindergs_b200 import error_floor as ef
from cindergs_b200 import workloads


def test_f64_formulas_match_the_f32_frame():
    wl = workloads.tet_cage_orbit(n=20_000, width=320, height=180)
    m = wl.cage.mesh
    bt, bw = oracle.bind_points(wl.scene.positions, m.rest_vertices, m.elements, m.inv_dm,
                                m.bounds())
    for _ in range(3):
        wl.step()
    v = wl.cage.vertices()
    J, R, S = oracle.v2_tet_transforms(v, m.elements, m.inv_dm)
    J64 = ef.tet_jacobians(v, m.elements, m.inv_dm)
    R64 = ef.polar_rotations(J64)
    assert np.abs(J.reshape(-1, 3, 3).transpose(0, 2, 1) - J64).max() < 1e-5
    assert np.abs(R.reshape(-1, 3, 3).transpose(0, 2, 1) - R64).max() < 1e-5
    sc = wl.scene
    pos, cov, opa, _, _ = oracle.v2_deform_split(v, m.elements, J, S, bt, bw, sc.positions,
                                                 sc.covariances_3d, sc.opacities, 0.0, 0.0)
    p64, c64, o64 = ef.deform(sc.positions, sc.covariances_3d, sc.opacities, bt, bw, v,
                              m.elements, m.inv_dm)
    assert np.abs(pos.reshape(-1, 3) - p64).max() < 1e-5
    diag = [0, 3, 5]
    assert (np.abs(cov.reshape(-1, 6)[:, diag] - c64[:, diag]) / c64[:, diag]).max() < 1e-4
    assert np.abs(opa - o64).max() < 1e-5
    cam = wl.camera(3)
    comp = wl.compositor(cam)
    attrs, ext, _ = oracle.v2_project(pos, cov, opa, sc.sh_coeffs, cam.to_array(),
                                      comp.camera_position, 0.0, 1 / 255.0, 0.5, 3,
                                      n_rest=sc.count, bind_tet=bt, tet_R=R,
                                      num_tets=m.num_tets, split_meta=None)
    a = attrs.reshape(-1, 10)
    vis = ext != 0
    Rg = np.where((bt < m.num_tets)[:, None, None], R64[np.minimum(bt, m.num_tets - 1)],
                  np.eye(3))
    mu, conic, alpha, rgb = ef.project(p64, c64, o64, sc.sh_coeffs, Rg, cam.to_array(),
                                       comp.camera_position, 3)
    assert vis.sum() > 10_000
    assert np.abs(a[vis, 0:2] - mu[vis]).max() < 1e-3
    assert np.abs(a[vis, 5] - alpha[vis]).max() < 1e-4
    assert np.abs(a[vis, 6:9] - rgb[vis]).max() < 1e-5
    # the f64 compositor on the oracle's own lists reproduces its image
    o = oracle.v2_frame(sc.as_dict(), cam.to_array(),
                        dict(width=320, height=180, bg=np.asarray(comp.background_color, np.float32),
                             cam_pos=np.asarray(comp.camera_position, np.float32), sh_degree=3),
                        cage=dict(verts=v, elems=m.elements, inv_dm=m.inv_dm, bind_tet=bt,
                                  bind_w=bw))
    rg = o["ranges"].reshape(-1, 2)
    t = int(np.argmax(rg[:, 1] - rg[:, 0]))
    lst = o["sorted_ids"][rg[t, 0]:rg[t, 1]].astype(np.int64)
    ty, tx = divmod(t, (320 + 15) // 16)
    yy, xx = np.mgrid[ty * 16:ty * 16 + 16, tx * 16:tx * 16 + 16]
    out = ef.composite_pixels(xx.ravel().astype(float), yy.ravel().astype(float), lst, mu, conic,
                              alpha, rgb, comp.background_color)
    ref = o["rgba_f32"][yy.ravel(), xx.ravel(), :3]
    assert np.abs(out - ref).max() < 2e-3
