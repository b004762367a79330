"""The oracle's CageSpringSimulator restatement against the reference's own
dynamics tests (deformation/dynamics.rs:323-450) and against the host
simulator that drives the benchmark cages."""
import numpy as np

import oracle
from cindergs_b200.cage import CageSpringSimulator, TetMesh

f32 = np.float32
DEFAULT = dict(stiffness=180.0, damping=0.92, mass=1.0)


def run(rest, cur, vel, pinned, steps, dt, planes=None, **kw):
    p = dict(DEFAULT, **kw)
    for _ in range(steps):
        cur, vel = oracle.spring_step(rest, cur, vel, pinned, p["stiffness"], p["damping"],
                                      p["mass"], planes, dt)
    return cur, vel


def test_converges_to_rest():
    rest = np.array([[0, 0, 0], [1, 0, 0]], f32)
    cur = rest.copy()
    cur[0, 0] = 2.0
    cur, _ = run(rest, cur, np.zeros_like(rest), None, 120, 0.016)
    assert np.linalg.norm(cur[0] - rest[0]) < 0.05


def test_timestep_is_clamped():
    rest = np.zeros((1, 3), f32)
    cur = np.array([[1.0, 0, 0]], f32)
    cur, _ = run(rest, cur, np.zeros_like(rest), None, 1, 2.0)
    assert np.isfinite(cur).all() and abs(cur[0, 0]) < 10.0
    # dt <= 0 leaves the state alone
    same, v = run(rest, cur, np.ones_like(cur), None, 1, 0.0)
    np.testing.assert_array_equal(same, cur)
    np.testing.assert_array_equal(v, np.ones_like(cur))


def test_pinned_vertex_stays():
    rest = np.zeros((1, 3), f32)
    cur = np.full((1, 3), 5.0, f32)
    c, v = run(rest, cur, np.full((1, 3), 3.0, f32), np.array([1], np.uint8), 1, 0.016)
    np.testing.assert_array_equal(c, cur)
    np.testing.assert_array_equal(v, np.zeros((1, 3), f32))


def test_damping_is_frame_rate_independent():
    rest = np.zeros((1, 3), f32)
    start = np.array([[1.0, 0, 0]], f32)
    x = {hz: run(rest, start, np.zeros_like(rest), None, hz, 1.0 / hz)[0][0, 0] for hz in (30, 60, 120)}
    assert abs(x[120] - x[60]) < 2e-2 and abs(x[30] - x[60]) < 2e-2


def test_damping_coefficient_matches_the_60hz_retention():
    assert abs(oracle.spring_frame_damping(0.92, 1.0) - 0.92 ** 60) < 1e-5


def test_pins_and_a_ground_plane():
    rest = np.array([[0, 1, 0], [1, 1, 0], [2, 1, 0]], f32)
    cur = rest.copy()
    cur[0] = [0.0, 2.5, 0.0]
    cur[1] = [1.0, -1.0, 0.0]
    vel = np.zeros_like(rest)
    vel[1] = [0.0, -4.0, 0.0]
    ground = np.array([[0, 1, 0, 0.25, 0.25, 0.2, 0, 0]], f32)  # CollisionPlane::ground_y(0.25)
    c, v = run(rest, cur, vel, np.array([1, 0, 1], np.uint8), 1, 0.016, planes=ground)
    assert abs(c[0, 1] - 2.5) < 1e-6
    assert c[1, 1] >= 0.25 - 1e-5
    assert v[1, 1] >= 0.0  # reflected with restitution, no longer moving into the plane


def test_jiggle_impulse_is_radial():
    rest = np.array([[1, 0, 0], [-1, 0, 0], [0, 0, 0], [0, 2, 0]], f32)
    v = oracle.spring_impulse(rest, np.zeros_like(rest), np.array([0, 0, 0, 1], np.uint8), 0.5)
    c = rest.mean(axis=0)
    for i in range(3):
        d = rest[i] - c
        np.testing.assert_allclose(v[i], 0.5 * d / np.linalg.norm(d), rtol=1e-6)
    np.testing.assert_array_equal(v[3], [0, 0, 0])  # pinned


def test_host_simulator_follows_the_oracle():
    mesh = TetMesh.create_grid_cage((5, 5, 5), (-1.1,) * 3, (1.1,) * 3)
    sim = CageSpringSimulator(mesh.rest_vertices)
    sim.stiffness, sim.damping = f32(40.0), f32(np.exp(-4.0 / 60.0))
    rng = np.random.default_rng(0)
    sim.current_positions = (sim.rest_positions + rng.normal(0, 0.05, sim.rest_positions.shape)).astype(f32)
    sim.pinned[:] = sim.rest_positions[:, 1] <= sim.rest_positions[:, 1].min() + 1e-6
    cur, vel = sim.current_positions.copy(), sim.velocities.copy()
    for _ in range(30):
        sim.step(1.0 / 60.0)
        cur, vel = oracle.spring_step(sim.rest_positions, cur, vel, sim.pinned, sim.stiffness,
                                      sim.damping, sim.mass, None, 1.0 / 60.0)
    np.testing.assert_allclose(sim.current_positions, cur, rtol=1e-6, atol=1e-7)
    np.testing.assert_allclose(sim.velocities, vel, rtol=1e-5, atol=1e-7)
