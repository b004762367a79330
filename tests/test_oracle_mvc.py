"""The oracle's restatement of the reference's polygon-cage MVC code
(deformation/mvc.rs) against the reference's own tests (mvc.rs:796-907) and
the host-side PolyCageMesh."""
import numpy as np
import pytest

import oracle
from cindergs_b200 import PolyCageMesh

f32 = np.float32


def test_presets_are_closed_manifolds():
    """test_mvc_presets_are_closed_manifolds (mvc.rs:799-811)."""
    box = PolyCageMesh.create_box_surface_cage([-1.0] * 3, [1.0] * 3)
    assert box.is_closed_manifold()
    assert abs(box.signed_volume() - 8.0) < 1e-4
    oct_ = PolyCageMesh.create_octahedron_cage([0.0] * 3, 1.5)
    assert oct_.is_closed_manifold() and oct_.signed_volume() > 0.0
    ico = PolyCageMesh.create_icosahedron_cage([0.0] * 3, 2.0)
    assert ico.is_closed_manifold() and ico.signed_volume() > 0.0


@pytest.mark.parametrize("which", ["box", "octahedron", "icosahedron"])
def test_linear_reproduction_inside_polyhedra(which):
    """test_mvc_linear_reproduction_inside_polyhedra (mvc.rs:813-832)."""
    cage = {"box": PolyCageMesh.create_box_surface_cage([-1.0, -2.0, -0.5], [2.0, 1.5, 2.5]),
            "octahedron": PolyCageMesh.create_octahedron_cage([0.3, -0.2, 0.4], 2.0),
            "icosahedron": PolyCageMesh.create_icosahedron_cage([-0.5, 0.5, 0.2], 2.5)}[which]
    p = np.array([0.45, -0.1, 0.35], f32)
    assert abs(oracle.mvc_winding(cage.rest_vertices, cage.triangles, p)) >= 0.5
    w = oracle.mvc_weights(p[None], cage.rest_vertices, cage.triangles)[0]
    assert abs(w.sum() - 1.0) < 1e-4
    rec = (w[:, None] * cage.rest_vertices).sum(0)
    assert np.linalg.norm(rec - p) < 1e-4


def test_vertex_and_face_boundary_reproduction():
    """test_mvc_vertex_and_face_boundary_reproduction (mvc.rs:834-845)."""
    oct_ = PolyCageMesh.create_octahedron_cage([0.0] * 3, 1.0)
    w_v = oracle.mvc_weights(np.array([[1.0, 0.0, 0.0]], f32), oct_.rest_vertices,
                             oct_.triangles)[0]
    assert abs(w_v[0] - 1.0) < 1e-6
    on_face = np.array([[1.0 / 3.0] * 3], f32)
    w_f = oracle.mvc_weights(on_face, oct_.rest_vertices, oct_.triangles)[0]
    rec = (w_f[:, None] * oct_.rest_vertices).sum(0)
    assert np.linalg.norm(rec - on_face[0]) < 1e-4


def test_obj_parsing_and_triangulation():
    """test_obj_parsing_and_triangulation (mvc.rs:847-863)."""
    obj = ("# Simple tetrahedron in OBJ\nv 0 0 0\nv 1 0 0\nv 0 1 0\nv 0 0 1\n"
           "f 1/1/1 3/2/1 2/3/1\nf 1 2 4\nf 2 3 4\nf 3 1 4\n")
    cage = PolyCageMesh.from_obj_str(obj)
    assert cage.num_vertices == 4 and cage.num_triangles == 4
    assert cage.is_closed_manifold()


def test_deform_scene_split_and_outside():
    """test_mvc_deform_scene_and_to_tet_mesh (mvc.rs:865-895): one Gaussian
    inside a stretched octahedron splits (threshold 1.3, Mip 0.001), the one
    outside keeps its rest position."""
    oct_ = PolyCageMesh.create_octahedron_cage([0.0] * 3, 2.0)
    pts = np.array([[0.1, 0.2, 0.0], [5.0, 0.0, 0.0]], f32)
    inside, wg = oracle.mvc_bind(pts, oct_.rest_vertices, oct_.triangles)
    assert inside.tolist() == [True, False]
    deformed = oct_.rest_vertices.copy()
    deformed[0, 0] += 3.0
    deformed[1, 0] -= 3.0
    cov = np.array([[0.02, 0, 0, 0.02, 0, 0.02]] * 2, f32)
    out = oracle.mvc_deform(pts, cov, np.array([0.8, 0.8], f32), inside, wg, deformed,
                            split_thr=1.3, mip=0.001)
    assert out["pos"].shape[0] == 3
    assert abs(out["pos"][1, 0] - 5.0) < 1e-6


def test_precomputed_gradients_match_local_jacobian():
    """test_mvc_precomputed_gradients_match_local_jacobian (mvc.rs:897-907):
    F from the stored gradients equals the central-difference Jacobian of the
    deformed position at 1e-5."""
    oct_ = PolyCageMesh.create_octahedron_cage([0.1, -0.2, 0.3], 2.5)
    pts = np.array([[0.2, -0.1, 0.4], [-0.4, 0.3, -0.1], [0.0, 0.0, 0.0]], f32)
    inside, wg = oracle.mvc_bind(pts, oct_.rest_vertices, oct_.triangles)
    assert inside.all()
    d = oct_.rest_vertices.copy()
    d[0, 0] += 0.45
    d[2, 1] -= 0.3
    d[4, 2] += 0.2
    h = oracle.mvc_step(oct_.rest_vertices)
    for i, p in enumerate(pts):
        F = np.stack([(wg[i, :, 1 + k][:, None] * d).sum(0) for k in range(3)], axis=1)
        cols = []
        for k in range(3):
            pp, pm = p.copy(), p.copy()
            pp[k] += f32(h)
            pm[k] -= f32(h)
            wp = oracle.mvc_weights(pp[None], oct_.rest_vertices, oct_.triangles)[0]
            wm = oracle.mvc_weights(pm[None], oct_.rest_vertices, oct_.triangles)[0]
            cols.append(((wp[:, None] * d).sum(0) - (wm[:, None] * d).sum(0)) * (0.5 / h))
        np.testing.assert_allclose(F, np.stack(cols, axis=1), atol=1e-5)


def test_icosphere_cage_of_the_mvc_workload():
    """The MVC workload's cage: a level-3 icosphere of radius 1.15 (642
    vertices, 1,280 triangles), closed, displaced by at most 0.1."""
    ico = PolyCageMesh.icosphere([0, 0, 0], 1.15, 3)
    assert (ico.num_vertices, ico.num_triangles) == (642, 1280)
    assert ico.is_closed_manifold()
    cage = ico.displace_sinusoids(0.1, 8, seed=0)
    assert cage.is_closed_manifold() and cage.signed_volume() > 0.0
    d = np.linalg.norm(cage.rest_vertices - ico.rest_vertices, axis=1)
    assert abs(d.max() - 0.1) < 1e-5
    wn = cage.winding_numbers([[0.0, 0.0, 0.0], [0.3, -0.2, 0.1], [3.0, 0.0, 0.0]])
    np.testing.assert_allclose(wn, [1.0, 1.0, 0.0], atol=1e-6)
