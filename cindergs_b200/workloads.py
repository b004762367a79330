"""The benchmark workloads, built from seeded synthetic inputs.

``mvc_cage_sphere`` is the polygon-cage workload: Gaussians drawn as in
``random_scene`` with means uniform in the unit ball, a level-3 icosphere cage
of radius 1.15 (642 vertices, 1280 triangles) displaced by a smooth random
field of amplitude 0.1, deformed every frame by a moving smooth random field
of amplitude 0.1, rendered at 1920 x 1080 by the orbiting camera.

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
from .mvc import PolyCageMesh
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
                   frames: int = 120, cells: int = 5, box: float | None = 1.0) -> CageOrbitWorkload:
    scene = random_scene(n, seed=seed, box=box)
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


RESOLUTIONS = ((640, 360), (1280, 720), (1920, 1080))


def spiral_views(count: int = 64, fov_deg: float = 60.0):
    """(cameras, compositors) of `count` views on a spiral around the origin:
    view i at radius 3 + 2 t and elevation -30 + 90 t degrees (t = i / (count
    - 1)), azimuth advancing by the golden angle, looking at the origin, at
    resolutions cycling through 640x360, 1280x720 and 1920x1080."""
    cams, comps = [], []
    golden = np.pi * (3.0 - np.sqrt(5.0))
    for i in range(count):
        t = i / max(count - 1, 1)
        r = 3.0 + 2.0 * t
        el = np.deg2rad(-30.0 + 90.0 * t)
        az = golden * i
        eye = (r * np.cos(el) * np.sin(az), r * np.sin(el), r * np.cos(el) * np.cos(az))
        w, h = RESOLUTIONS[i % len(RESOLUTIONS)]
        cam = CameraUniforms.from_look_at(eye, (0, 0, 0), (0, 1, 0), np.deg2rad(fov_deg), w, h,
                                          0.2)
        cams.append(cam)
        comps.append(CompositorUniforms(w, h, (0.0, 0.0, 0.0, 1.0),
                                        tuple(float(x) for x in cam.eye()), 3))
    return cams, comps


def multiview_cage(n: int = 2_000_000, views: int = 64, seed: int = 0):
    """The batched multi-view workload: Gaussians as in ``random_scene``
    (means N(0, I3), not rescaled), the spring-driven tet cage of
    ``tet_cage_orbit`` deforming them once per step, and ``spiral_views``.
    Returns (CageOrbitWorkload, cameras, compositors)."""
    wl = tet_cage_orbit(n=n, seed=seed, box=None)
    cams, comps = spiral_views(views)
    return wl, cams, comps


@dataclass
class LargeMultiCageWorkload:
    """Quantized scene, several spring-driven tet cages and a polygon cage."""
    scene: object            # QuantizedGaussianSceneSoa
    cages: list              # tet cages (Cage)
    poly: "PolyCageWorkload"  # polygon cage and its motion (scene unused)
    width: int
    height: int
    frames: int
    radius: float
    dt: float = 1.0 / 60.0

    def camera(self, frame: int) -> CameraUniforms:
        return orbit_camera(frame % self.frames, self.frames, self.radius, self.width,
                            self.height, 60.0)

    def compositor(self, cam: CameraUniforms) -> CompositorUniforms:
        return CompositorUniforms(self.width, self.height, (0.0, 0.0, 0.0, 1.0),
                                  tuple(float(x) for x in cam.eye()), 3)


def spring_cage(lo, hi, cells: int, rng: np.random.Generator) -> Cage:
    """Grid cage of cells^3 cubes (6 tets each) over [lo, hi] with the spring
    parameters of the tet-cage workload: bottom layer pinned, the rest
    displaced by N(0, 0.05)."""
    mesh = TetMesh.create_grid_cage((cells, cells, cells), lo, hi)
    cage = Cage("grid", mesh)
    sim = cage.simulator
    sim.stiffness = f32(40.0)
    sim.damping = f32(np.exp(-4.0 / 60.0))
    sim.pinned = mesh.rest_vertices[:, 1] <= mesh.rest_vertices[:, 1].min()
    disp = rng.normal(0.0, 0.05, mesh.rest_vertices.shape).astype(f32)
    disp[sim.pinned] = 0.0
    sim.current_positions = (mesh.rest_vertices + disp).astype(f32)
    return cage


def large_multicage(n: int = 6_000_000, seed: int = 0, width: int = 7680, height: int = 4320,
                    frames: int = 30, radius: float = 4.0) -> LargeMultiCageWorkload:
    """The large-scene workload: Gaussians drawn as in ``random_scene`` and
    scaled into [-1, 1]^3, stored as a QuantizedGaussianSceneSoa (f16
    covariances and SH degree 3); four 4x4x4-cube (384-tet) spring cages over
    the upper half (x and z halves of [-1.1, 1.1], y in [0, 1.1]); the
    level-3 icosphere polygon cage of ``mvc_cage_sphere`` (its moving field)
    for the rest; 7680 x 4320 (129,600 tiles, 64-bit keys), a camera orbiting
    at `radius`."""
    from .scene import QuantizedGaussianSceneSoa
    scene = QuantizedGaussianSceneSoa.from_soa(random_scene(n, seed=seed, box=1.0), 3)
    rng = np.random.Generator(np.random.PCG64(seed + 1))
    cages = [spring_cage((x0, 0.0, z0), (x0 + 1.1, 1.1, z0 + 1.1), 4, rng)
             for x0 in (-1.1, 0.0) for z0 in (-1.1, 0.0)]
    poly = mvc_cage_sphere(n=1, seed=seed, width=width, height=height, frames=frames)
    return LargeMultiCageWorkload(scene, cages, poly, width, height, frames, radius)


def ball_points(n: int, rng: np.random.Generator, radius: float = 1.0) -> np.ndarray:
    """n points uniform in the ball of `radius` (direction from a normal
    sample, radius from the cube root of a uniform)."""
    d = rng.standard_normal((n, 3))
    d /= np.maximum(np.linalg.norm(d, axis=1, keepdims=True), 1e-12)
    r = radius * rng.uniform(0.0, 1.0, n) ** (1.0 / 3.0)
    return (d * r[:, None]).astype(f32)


@dataclass
class PolyCageWorkload:
    scene: GaussianSceneSoa
    cage: PolyCageMesh
    width: int
    height: int
    frames: int
    radius: float
    amplitude: float
    waves: np.ndarray       # [k, 3] wave vectors
    phases: np.ndarray      # [k]
    speeds: np.ndarray      # [k] phase change per frame
    dirs: np.ndarray        # [k, 3] unit displacement directions
    sh_degree: int = 3
    background: tuple = (0.0, 0.0, 0.0, 1.0)

    def camera(self, frame: int) -> CameraUniforms:
        return orbit_camera(frame % self.frames, self.frames, self.radius, self.width,
                            self.height, 60.0)

    def compositor(self, cam: CameraUniforms) -> CompositorUniforms:
        return CompositorUniforms(self.width, self.height, self.background,
                                  tuple(float(x) for x in cam.eye()), self.sh_degree)

    def vertices(self, frame: int) -> np.ndarray:
        """Cage vertices of a frame: rest + sum_k dir_k sin(k_k . v + phase_k +
        speed_k frame), scaled so the largest displacement is `amplitude`."""
        v = self.cage.rest_vertices.astype(np.float64)
        s = np.sin(v @ self.waves.T + self.phases[None, :] + self.speeds[None, :] * frame)
        d = s @ self.dirs
        d *= self.amplitude / max(np.linalg.norm(d, axis=1).max(), 1e-12)
        return (v + d).astype(f32)

    def training_points(self, n: int, seed: int = 1) -> np.ndarray:
        """Interior training points: uniform in the unit ball (where the
        Gaussians are)."""
        return ball_points(n, np.random.Generator(np.random.PCG64(seed)))


def mvc_cage_sphere(n: int = 3_000_000, seed: int = 0, width: int = 1920, height: int = 1080,
                    frames: int = 120) -> PolyCageWorkload:
    scene = random_scene(n, seed=seed)
    rng = np.random.Generator(np.random.PCG64(seed + 1000))
    scene.positions[:] = ball_points(n, rng)
    cage = PolyCageMesh.icosphere([0.0, 0.0, 0.0], 1.15, 3).displace_sinusoids(0.1, 8, seed=seed)
    k = 8
    dirs = rng.standard_normal((k, 3))
    dirs /= np.linalg.norm(dirs, axis=1, keepdims=True)
    waves = dirs * rng.uniform(2.0, 4.0, (k, 1))
    disp = rng.standard_normal((k, 3))
    disp /= np.linalg.norm(disp, axis=1, keepdims=True)
    return PolyCageWorkload(scene=scene, cage=cage, width=width, height=height, frames=frames,
                            radius=4.0, amplitude=0.1, waves=waves,
                            phases=rng.uniform(0.0, 2.0 * np.pi, k),
                            speeds=rng.uniform(0.02, 0.06, k), dirs=disp)
