"""The benchmark workloads, built from seeded synthetic inputs.

``tet_cage_orbit`` is the tetrahedral-cage deform + render workload: Gaussians
drawn as in ``random_scene`` with means scaled to fill [-1, 1]^3, a cage of
5 x 5 x 5 cubes over [-1.1, 1.1]^3 split into 6 tets each (750 tets, 216
vertices) whose bottom vertex layer is pinned and whose other vertices start
displaced by N(0, 0.05) and are driven by the spring solver (stiffness 40,
damping coefficient 4 s^-1, i.e. velocity retention exp(-4/60) per 1/60 s,
dt = 1/60), rendered at 1920 x 1080 by a camera orbiting the origin at radius
4 (one revolution per `frames` frames, 60 degree vertical field of view).
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from .cage import Cage, CageScene, TetMesh
from .camera import CameraUniforms, CompositorUniforms, orbit_camera
from .scene import GaussianSceneSoa, random_scene

f32 = np.float32


@dataclass
class CageOrbitWorkload:
    scene: GaussianSceneSoa
    cage: Cage
    width: int
    height: int
    frames: int
    radius: float
    sh_degree: int = 3
    background: tuple = (0.0, 0.0, 0.0, 1.0)
    strain_split_threshold: float = 0.0
    mip_filter_3d_var: float = 0.0
    dt: float = 1.0 / 60.0
    cages: CageScene | None = None

    def camera(self, frame: int) -> CameraUniforms:
        return orbit_camera(frame % self.frames, self.frames, self.radius, self.width,
                            self.height, 60.0)

    def compositor(self, cam: CameraUniforms) -> CompositorUniforms:
        return CompositorUniforms(self.width, self.height, self.background,
                                  tuple(float(x) for x in cam.eye()), self.sh_degree)

    def bind(self, pipeline) -> CageScene:
        """Binds the scene to the cage on the GPU (first call only)."""
        if self.cages is None:
            self.cages = CageScene.auto_bind([self.cage], pipeline, self.scene.count)
        return self.cages

    def step(self) -> None:
        self.cage.simulator.step(self.dt)


def tet_cage_orbit(n: int = 1_100_000, seed: int = 0, width: int = 1920, height: int = 1080,
                   frames: int = 120, cells: int = 5) -> CageOrbitWorkload:
    scene = random_scene(n, seed=seed, box=1.0)
    mesh = TetMesh.create_grid_cage((cells, cells, cells), (-1.1,) * 3, (1.1,) * 3)
    cage = Cage("grid", mesh)
    sim = cage.simulator
    sim.stiffness = f32(40.0)
    sim.damping = f32(np.exp(-4.0 / 60.0))
    ymin = mesh.rest_vertices[:, 1].min()
    sim.pinned = mesh.rest_vertices[:, 1] <= ymin
    rng = np.random.Generator(np.random.PCG64(seed + 1))
    disp = rng.normal(0.0, 0.05, mesh.rest_vertices.shape).astype(f32)
    disp[sim.pinned] = 0.0
    sim.current_positions = (mesh.rest_vertices + disp).astype(f32)
    return CageOrbitWorkload(scene, cage, width, height, frames, 4.0)
