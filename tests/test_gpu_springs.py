"""Cage spring dynamics on the device (cgs_springs_*) against the oracle's
CageSpringSimulator restatement (deformation/dynamics.rs:249-305), bit for
bit: per-cage stiffness, damping and mass, pins, a collision plane, clamped
and non-positive time steps, several steps per launch and the jiggle impulse.
A frame deformed by the device state equals one deformed by the same
vertices uploaded from the host."""
import numpy as np
import pytest

import oracle
from cindergs_b200 import Cage, CageScene, GpuPipelineState, TetMesh, random_scene
from cindergs_b200 import _abi
from cindergs_b200.cage import CollisionPlane
from helpers import compositor, config0_camera

pytestmark = pytest.mark.gpu
f32 = np.float32


def bits(a):
    return np.asarray(a, f32).view(np.uint32)


@pytest.fixture(scope="module")
def st():
    s = GpuPipelineState(0)
    yield s
    s.close()


def two_cages(st, n):
    st.invalidate()
    scene = random_scene(n, seed=3, box=1.0)
    st.upload_scene(scene)
    a = Cage("a", TetMesh.create_grid_cage((3, 3, 3), (-1.1, -1.1, -1.1), (0.0, 1.1, 1.1)))
    b = Cage("b", TetMesh.create_grid_cage((4, 4, 4), (0.0, -1.1, -1.1), (1.1, 1.1, 1.1)))
    cages = CageScene.auto_bind([a, b], st, n)
    rng = np.random.default_rng(4)
    for c, (k, damp, mass) in zip((a, b), ((40.0, 0.93551, 1.0), (180.0, 0.92, 2.5))):
        sim = c.simulator
        sim.stiffness, sim.damping, sim.mass = f32(k), f32(damp), f32(mass)
        sim.current_positions = (sim.rest_positions + rng.normal(0, 0.08, sim.rest_positions.shape)).astype(f32)
        sim.velocities = rng.normal(0, 0.3, sim.rest_positions.shape).astype(f32)
        sim.pinned[:] = sim.rest_positions[:, 1] <= sim.rest_positions[:, 1].min() + 1e-6
    # above the free layer at rest y = -0.367, so that layer is held by the plane
    a.simulator.collision_planes.append(CollisionPlane.ground_y(-0.3))
    st.upload_cages(cages)
    return scene, cages


def oracle_state(cages):
    return [(c.simulator.current_positions.copy(), c.simulator.velocities.copy()) for c in cages.cages]


def oracle_steps(cages, state, dt, steps):
    out = []
    for c, (cur, vel) in zip(cages.cages, state):
        sim = c.simulator
        planes = np.array([[*p.normal, p.offset, p.restitution, p.friction, 0, 0]
                           for p in sim.collision_planes], f32).reshape(-1, 8)
        for _ in range(steps):
            cur, vel = oracle.spring_step(sim.rest_positions, cur, vel, sim.pinned, sim.stiffness,
                                          sim.damping, sim.mass, planes, dt)
        out.append((cur, vel))
    return out


def test_device_springs_match_the_oracle(st):
    scene, cages = two_cages(st, 20_000)
    st.springs_upload(cages)
    state = oracle_state(cages)
    for dt, steps in ((1.0 / 60.0, 10), (1.0 / 120.0, 7), (2.0, 1), (0.0, 3), (-1.0, 1),
                      (1.0 / 60.0, 25)):
        st.springs_step(dt, steps)
        state = oracle_steps(cages, state, dt, steps)
    cur, vel = st.springs_read()
    np.testing.assert_array_equal(bits(cur), bits(np.concatenate([s[0] for s in state])))
    np.testing.assert_array_equal(bits(vel), bits(np.concatenate([s[1] for s in state])))
    # the ground plane holds cage a's free vertices at or above y = -0.3
    # (pinned vertices are not stepped: the bottom layer stays at y = -1.1)
    na = cages.cages[0].mesh.num_vertices
    free = ~cages.cages[0].simulator.pinned
    assert (cur[:na][free, 1] >= f32(-0.3) - 1e-6).all()
    assert (np.abs(cur[:na][free, 1] + 0.3) < 1e-6).sum() >= 8  # resting on the plane
    # jiggle impulse, then more steps
    st.springs_impulse(0.4)
    state = [(c, oracle.spring_impulse(sim.simulator.rest_positions, v, sim.simulator.pinned, 0.4))
             for (c, v), sim in zip(state, cages.cages)]
    st.springs_step(1.0 / 60.0, 5)
    state = oracle_steps(cages, state, 1.0 / 60.0, 5)
    cur, vel = st.springs_read()
    np.testing.assert_array_equal(bits(cur), bits(np.concatenate([s[0] for s in state])))
    np.testing.assert_array_equal(bits(vel), bits(np.concatenate([s[1] for s in state])))


def test_frames_deform_with_the_device_state(st):
    scene, cages = two_cages(st, 60_000)
    st.springs_upload(cages)
    cam = config0_camera(480, 270)
    comp = compositor(480, 270, cam, deg=3)
    st.springs_step(1.0 / 60.0, 12)
    st.execute_frame_gpu(scene, cages, cam, comp, 1.2, 0.0, force_stage3=True)
    img_dev = st.readback_framebuffer_rgba8(480, 270)
    pos_dev = st.read_buffer(_abi.BUF_DEFORMED_POS, f32)
    cur, vel = st.springs_read()
    # the same vertices uploaded from the host
    st.invalidate()
    st.upload_scene(scene)
    first = 0
    for c in cages.cages:
        nv = c.mesh.num_vertices
        c.simulator.current_positions = cur[first:first + nv].copy()
        first += nv
    st.execute_frame_gpu(scene, cages, cam, comp, 1.2, 0.0, force_stage3=True)
    np.testing.assert_array_equal(bits(st.read_buffer(_abi.BUF_DEFORMED_POS, f32)), bits(pos_dev))
    np.testing.assert_array_equal(st.readback_framebuffer_rgba8(480, 270), img_dev)
    # stepping without a frame between: no host vertex upload takes over
    st.springs_upload(cages)
    st.springs_step(1.0 / 60.0, 1)
    st.execute_frame_gpu(scene, cages, cam, comp, 1.2, 0.0)
    c2, _ = st.springs_read()
    assert not np.array_equal(c2, cur)


def test_springs_need_cages(st):
    st.invalidate()
    st.upload_scene(random_scene(1000, seed=1))
    st.upload_cages(None)
    with pytest.raises(_abi.CgsError) as e:
        st.springs_step(1.0 / 60.0)
    assert e.value.code == _abi.CGS_E_STATE
