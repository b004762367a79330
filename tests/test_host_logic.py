"""Host-side set-up code: activations, cameras, cages, springs, bindings."""
import numpy as np
import pytest

import oracle
from cindergs_b200 import (Cage, CageScene, CageSpringSimulator, CameraUniforms, TetMesh,
                           UNBOUND, random_scene, scene_fingerprint)
from cindergs_b200.scene import activate_opacity, activate_rotation, compute_covariance_3d
from cindergs_b200.workloads import tet_cage_orbit


def test_look_at_lh_matches_glam():
    cam = CameraUniforms.from_look_at((0, 0, 4), (0, 0, 0), (0, 1, 0), np.deg2rad(60), 1280, 720)
    v = cam.view_matrix.reshape(4, 4)  # columns
    np.testing.assert_array_equal(v[0], [-1, 0, 0, 0])
    np.testing.assert_array_equal(v[1], [0, 1, 0, 0])
    np.testing.assert_array_equal(v[2], [0, 0, -1, 0])
    np.testing.assert_array_equal(v[3], [0, 0, 4, 1])
    assert abs(cam.focal_y - 360.0 / np.tan(np.deg2rad(30))) < 1e-3
    np.testing.assert_allclose(cam.eye(), [0, 0, 4], atol=1e-6)


def test_activations():
    assert activate_opacity(np.array([0.0], np.float32))[0] == 0.5
    q = activate_rotation(np.array([[0, 0, 0, 0], [2, 0, 0, 0]], np.float32))
    np.testing.assert_array_equal(q, [[0, 0, 0, 1], [0, 0, 0, 1]])
    cov = compute_covariance_3d(np.array([[0.2, 0.2, 0.2]], np.float32), q[:1])
    np.testing.assert_allclose(cov, [[0.04, 0, 0, 0.04, 0, 0.04]], atol=1e-9)


def test_random_scene_is_seeded_and_positive_definite():
    a, b = random_scene(5000, seed=3), random_scene(5000, seed=3)
    assert scene_fingerprint(a) != b"" and np.array_equal(a.covariances_3d, b.covariances_3d)
    c = a.covariances_3d.astype(np.float64)
    m1 = c[:, 0]
    m2 = c[:, 0] * c[:, 3] - c[:, 1] ** 2
    assert (m1 > 0).all() and (m2 > 0).all()
    boxed = random_scene(5000, seed=3, box=1.0)
    assert abs(np.abs(boxed.positions).max() - 1.0) < 1e-6


def test_grid_cage_topology():
    m = TetMesh.create_grid_cage((5, 5, 5), (-1.1,) * 3, (1.1,) * 3)
    assert m.num_tets == 750 and m.num_vertices == 216
    pts = np.random.default_rng(0).uniform(-1.09, 1.09, (4000, 3)).astype(np.float32)
    t, w = oracle.bind_points(pts, m.rest_vertices, m.elements, m.inv_dm, m.bounds())
    assert (t != UNBOUND).all()
    assert np.abs(w.sum(axis=1) - 1).max() < 1e-5
    assert w.min() > -1.1e-4  # contained (violation <= 1e-4)
    # the 6-tet split tiles each cube: the volumes add up to the box
    v = m.rest_vertices
    e = m.elements.astype(np.int64)
    vol = np.abs(np.linalg.det(np.stack([v[e[:, 1]] - v[e[:, 0]], v[e[:, 2]] - v[e[:, 0]],
                                         v[e[:, 3]] - v[e[:, 0]]], axis=1))) / 6
    assert abs(vol.sum() - 2.2 ** 3) < 1e-4


def test_box_cage_inverse_rest_shape():
    m = TetMesh.create_box_cage((0, 0, 0), (1, 1, 1))
    assert m.num_tets == 5
    v, e = m.rest_vertices, m.elements.astype(np.int64)
    for t in range(5):
        D = np.stack([v[e[t, k]] - v[e[t, 0]] for k in (1, 2, 3)], axis=1)
        inv = m.inv_dm[t].reshape(3, 3).T  # column-major
        np.testing.assert_allclose(inv @ D, np.eye(3), atol=1e-6)


def test_spring_convergence_and_frame_rate_independence():
    rest = np.array([[0, 0, 0], [1, 0, 0]], np.float32)
    s = CageSpringSimulator(rest)
    s.current_positions[1] = [2.0, 0.0, 0.0]
    for _ in range(600):
        s.step(1 / 60)
    assert np.abs(s.current_positions - rest).max() < 1e-3
    # velocity retention per 1/60 s is the same when stepping at 30 or 120 Hz
    g60 = CageSpringSimulator.frame_damping(0.92, 1 / 60)
    g30 = CageSpringSimulator.frame_damping(0.92, 1 / 30)
    g120 = CageSpringSimulator.frame_damping(0.92, 1 / 120)
    assert abs(g60 - 0.92) < 1e-6
    assert abs(g30 - g60 ** 2) < 1e-6 and abs(g120 ** 2 - g60) < 1e-6


def test_pinned_vertices_do_not_move():
    wl = tet_cage_orbit(n=10, width=64, height=64)
    sim = wl.cage.simulator
    pinned_before = sim.current_positions[sim.pinned].copy()
    assert sim.pinned.sum() == 36  # bottom layer of the 6x6x6 vertex grid
    for _ in range(10):
        wl.step()
    np.testing.assert_array_equal(sim.current_positions[sim.pinned], pinned_before)
    assert np.abs(sim.current_positions[~sim.pinned] - sim.rest_positions[~sim.pinned]).max() > 0


def test_flatten_offsets_multi_cage():
    a = Cage("a", TetMesh.create_box_cage((0, 0, 0), (1, 1, 1)))
    b = Cage("b", TetMesh.create_box_cage((2, 0, 0), (3, 1, 1)))
    bind_cage = np.array([0, 1, UNBOUND], np.uint32)
    bind_tet = np.array([3, 2, 0], np.uint32)
    bind_w = np.ones((3, 4), np.float32) * 0.25
    cs = CageScene([a, b], bind_cage, bind_tet, bind_w)
    elems, inv, nverts, gt, w = cs.flatten()
    assert elems.shape == (10, 4) and nverts == 16
    assert gt.tolist() == [3, 7, UNBOUND]
    assert (elems[5:] >= 8).all()
    assert (w[2] == 0).all()
