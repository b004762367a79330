"""Tetrahedral cages: topology, rest-shape inverses, spring dynamics and
multi-cage bindings (deformation/mod.rs, deformation/dynamics.rs).

Host-side set-up code. Binding Gaussians to tets runs on the GPU through the
library (cgs_bind_tets). The spring step runs here over a few hundred
vertices, as in the reference, or on the device
(GpuPipelineState.springs_upload / springs_step, cgs_springs_*) where the
cage state then stays resident between frames.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

f32 = np.float32
UNBOUND = 0xFFFFFFFF


def _mat3_inverse_cols(c0, c1, c2):
    """glam Mat3::inverse of the matrix with columns c0, c1, c2 ([T,3] each);
    returns the inverse column-major [T,9]."""
    def cross(a, b):
        return np.stack([a[:, 1] * b[:, 2] - b[:, 1] * a[:, 2],
                         a[:, 2] * b[:, 0] - b[:, 2] * a[:, 0],
                         a[:, 0] * b[:, 1] - b[:, 0] * a[:, 1]], axis=1).astype(f32)
    tmp0 = cross(c1, c2)
    tmp1 = cross(c2, c0)
    tmp2 = cross(c0, c1)
    det = ((c2[:, 0] * tmp2[:, 0] + c2[:, 1] * tmp2[:, 1]) + c2[:, 2] * tmp2[:, 2]).astype(f32)
    inv_det = (f32(1.0) / det).astype(f32)
    a = tmp0 * inv_det[:, None]
    b = tmp1 * inv_det[:, None]
    c = tmp2 * inv_det[:, None]
    # from_cols(a, b, c).transpose(): column j of the result = row j of [a b c]
    out = np.stack([a[:, 0], b[:, 0], c[:, 0], a[:, 1], b[:, 1], c[:, 1], a[:, 2], b[:, 2],
                    c[:, 2]], axis=1).astype(f32)
    return out, det


@dataclass
class TetMesh:
    """Rest vertices [V,3], elements [T,4] and D_m^-1 [T,9] column-major
    (TetMesh::new, deformation/mod.rs:202-227: identity when |det D_m| <= 1e-8)."""
    rest_vertices: np.ndarray
    elements: np.ndarray
    inv_dm: np.ndarray = field(default=None)

    def __post_init__(self):
        self.rest_vertices = np.ascontiguousarray(self.rest_vertices, f32).reshape(-1, 3)
        self.elements = np.ascontiguousarray(self.elements, np.uint32).reshape(-1, 4)
        if self.inv_dm is None:
            v = self.rest_vertices
            e = self.elements.astype(np.int64)
            x0 = v[e[:, 0]]
            c0, c1, c2 = (v[e[:, 1]] - x0).astype(f32), (v[e[:, 2]] - x0).astype(f32), \
                (v[e[:, 3]] - x0).astype(f32)
            inv, det = _mat3_inverse_cols(c0, c1, c2)
            degenerate = ~(np.abs(det) > f32(1e-8))
            inv[degenerate] = np.array([1, 0, 0, 0, 1, 0, 0, 0, 1], f32)
            self.inv_dm = inv

    @property
    def num_vertices(self) -> int:
        return int(self.rest_vertices.shape[0])

    @property
    def num_tets(self) -> int:
        return int(self.elements.shape[0])

    def bounds(self):
        """Rest AABB padded by 1e-3 of its extent (mod.rs:236-252)."""
        if self.num_vertices == 0:
            return np.full(3, -0.5, f32), np.full(3, 0.5, f32)
        mn = self.rest_vertices.min(axis=0)
        mx = self.rest_vertices.max(axis=0)
        pad = (np.maximum(mx - mn, f32(1e-3)) * f32(1e-3)).astype(f32)
        return (mn - pad).astype(f32), (mx + pad).astype(f32)

    @staticmethod
    def create_box_cage(mn, mx) -> "TetMesh":
        """Box split into 5 tets (create_box_cage, mod.rs:353-380)."""
        a, b = np.asarray(mn, f32), np.asarray(mx, f32)
        verts = np.array([[a[0], a[1], a[2]], [b[0], a[1], a[2]], [b[0], b[1], a[2]],
                          [a[0], b[1], a[2]], [a[0], a[1], b[2]], [b[0], a[1], b[2]],
                          [b[0], b[1], b[2]], [a[0], b[1], b[2]]], f32)
        elems = np.array([[0, 1, 3, 4], [1, 2, 3, 6], [1, 4, 5, 6], [3, 4, 6, 7], [1, 3, 4, 6]],
                         np.uint32)
        return TetMesh(verts, elems)

    @staticmethod
    def create_grid_cage(cells, mn, mx) -> "TetMesh":
        """Grid of cells[0] x cells[1] x cells[2] cubes over [mn, mx], each cube
        split into 6 tets around its main diagonal (Freudenthal/Kuhn split, which
        matches across shared faces). 5^3 cubes give 750 tets and 216 vertices."""
        nx, ny, nz = (int(c) for c in cells)
        a, b = np.asarray(mn, np.float64), np.asarray(mx, np.float64)
        xs = np.linspace(a[0], b[0], nx + 1)
        ys = np.linspace(a[1], b[1], ny + 1)
        zs = np.linspace(a[2], b[2], nz + 1)
        gx, gy, gz = np.meshgrid(xs, ys, zs, indexing="ij")
        verts = np.stack([gx.ravel(), gy.ravel(), gz.ravel()], axis=1).astype(f32)

        def vid(i, j, k):
            return (i * (ny + 1) + j) * (nz + 1) + k

        perms = [(0, 1, 2), (0, 2, 1), (1, 0, 2), (1, 2, 0), (2, 0, 1), (2, 1, 0)]
        elems = []
        for i in range(nx):
            for j in range(ny):
                for k in range(nz):
                    for p in perms:
                        cur = [i, j, k]
                        tet = [vid(*cur)]
                        for ax in p:
                            cur = list(cur)
                            cur[ax] += 1
                            tet.append(vid(*cur))
                        elems.append(tet)
        return TetMesh(verts, np.array(elems, np.uint32))


@dataclass
class CollisionPlane:
    """Half-space normal . x >= offset with restitution and friction
    (CollisionPlane, dynamics.rs:4-33); the normal is normalised on creation."""
    normal: np.ndarray
    offset: float
    restitution: float = 0.25
    friction: float = 0.2

    def __post_init__(self):
        n = np.asarray(self.normal, f32).reshape(3)
        l2 = f32((n[0] * n[0] + n[1] * n[1]) + n[2] * n[2])
        self.normal = (n * (f32(1.0) / np.sqrt(l2))).astype(f32) if l2 > f32(1e-8) else \
            np.array([0, 1, 0], f32)
        self.offset = f32(self.offset)
        self.restitution = f32(min(max(float(self.restitution), 0.0), 1.0))
        self.friction = f32(min(max(float(self.friction), 0.0), 1.0))

    @staticmethod
    def ground_y(y: float) -> "CollisionPlane":
        """CollisionPlane::ground_y (dynamics.rs:35-39)."""
        return CollisionPlane(np.array([0, 1, 0], f32), y, 0.25, 0.2)

    def resolve(self, pos: np.ndarray, vel: np.ndarray, mask: np.ndarray) -> None:
        """resolve_contact (dynamics.rs:57-71) on the rows of `mask`, in place."""
        n = self.normal
        d = ((n[0] * pos[:, 0] + n[1] * pos[:, 1]) + n[2] * pos[:, 2] - self.offset).astype(f32)
        hit = mask & (d < 0)
        if not hit.any():
            return
        pos[hit] = (pos[hit] - n[None, :] * d[hit, None]).astype(f32)
        v = vel[hit]
        vn = ((v[:, 0] * n[0] + v[:, 1] * n[1]) + v[:, 2] * n[2]).astype(f32)
        vnorm = (n[None, :] * vn[:, None]).astype(f32)
        vtan = (v - vnorm).astype(f32)
        new = (vtan * (f32(1.0) - self.friction) - vnorm * self.restitution).astype(f32)
        vel[hit] = np.where((vn < 0)[:, None], new, v)


class CageSpringSimulator:
    """Semi-implicit Euler springs toward the rest pose with frame-rate
    independent exponential damping and pinned vertices
    (CageSpringSimulator::step, dynamics.rs:249-277)."""
    MAX_DT = f32(0.033)
    DAMPING_REFERENCE_HZ = f32(60.0)

    def __init__(self, rest_positions: np.ndarray):
        self.rest_positions = np.ascontiguousarray(rest_positions, f32).reshape(-1, 3).copy()
        self.current_positions = self.rest_positions.copy()
        self.velocities = np.zeros_like(self.rest_positions)
        self.stiffness = f32(180.0)
        self.damping = f32(0.92)  # velocity retention per 1/60 s
        self.mass = f32(1.0)
        self.pinned = np.zeros(self.rest_positions.shape[0], bool)
        self.collision_planes: list[CollisionPlane] = []

    @staticmethod
    def damping_coefficient(damping) -> np.float32:
        retention = f32(min(max(float(damping), 1.0e-4), 0.9999))
        return f32(-np.log(retention) * CageSpringSimulator.DAMPING_REFERENCE_HZ)

    @staticmethod
    def frame_damping(damping, dt) -> np.float32:
        return f32(np.exp(-CageSpringSimulator.damping_coefficient(damping) * f32(dt)))

    def step(self, dt: float) -> None:
        dt_sim = min(f32(dt), self.MAX_DT)
        if dt_sim <= 0:
            return
        inv_mass = f32(1.0) / max(self.mass, f32(0.001))
        gamma = self.frame_damping(self.damping, dt_sim)
        free = ~self.pinned
        disp = self.rest_positions - self.current_positions
        accel = disp * (self.stiffness * inv_mass)
        v = ((self.velocities + accel * dt_sim) * gamma).astype(f32)
        self.velocities = np.where(free[:, None], v, f32(0.0)).astype(f32)
        self.current_positions = np.where(free[:, None],
                                          self.current_positions + self.velocities * dt_sim,
                                          self.current_positions).astype(f32)
        for plane in self.collision_planes:
            plane.resolve(self.current_positions, self.velocities, free)

    def trigger_jiggle_impulse(self, magnitude: float) -> None:
        """Outward radial velocity pulse from the rest centroid on unpinned
        vertices (trigger_jiggle_impulse, dynamics.rs:280-305)."""
        n = self.rest_positions.shape[0]
        if n == 0:
            return
        c = np.zeros(3, f32)
        for p in self.rest_positions:  # sequential float32 sum, vertex order
            c = (c + p).astype(f32)
        c = (c / f32(n)).astype(f32)
        d = (self.rest_positions - c).astype(f32)
        with np.errstate(divide="ignore", invalid="ignore"):
            rcp = (f32(1.0) / np.sqrt((d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1]) + d[:, 2] * d[:, 2])).astype(f32)
        ok = np.isfinite(rcp) & (rcp > 0)
        r = np.where(ok[:, None], d * rcp[:, None], f32(0.0)).astype(f32)
        big = ((r[:, 0] * r[:, 0] + r[:, 1] * r[:, 1]) + r[:, 2] * r[:, 2]) > f32(1e-4)
        m = f32(magnitude)
        imp = np.where(big[:, None], r * m, np.array([0, 1, 0], f32) * m).astype(f32)
        free = ~self.pinned
        self.velocities[free] = (self.velocities[free] + imp[free]).astype(f32)

    def positions_array(self) -> np.ndarray:
        return self.current_positions


@dataclass
class Cage:
    name: str
    mesh: TetMesh

    def __post_init__(self):
        self.simulator = CageSpringSimulator(self.mesh.rest_vertices)

    def vertices(self) -> np.ndarray:
        return self.simulator.positions_array()


class CageScene:
    """Independent cages plus per-Gaussian ownership (CageScene, mod.rs:415-508):
    bind_cage [N] (UNBOUND when static), bind_tet [N] (tet inside its cage),
    bind_w [N,4] barycentric weights."""

    def __init__(self, cages, bind_cage, bind_tet, bind_w):
        self.cages = list(cages)
        self.bind_cage = np.ascontiguousarray(bind_cage, np.uint32)
        self.bind_tet = np.ascontiguousarray(bind_tet, np.uint32)
        self.bind_w = np.ascontiguousarray(bind_w, f32).reshape(-1, 4)

    @staticmethod
    def auto_bind(cages, pipeline, num_points: int) -> "CageScene":
        """Binds every cage to the resident scene's Gaussians inside its padded
        rest bounds; the first cage in the list owns overlapping Gaussians
        (CageScene::auto_bind, mod.rs:444-464). Runs on the GPU."""
        bind_cage = np.full(num_points, UNBOUND, np.uint32)
        bind_tet = np.zeros(num_points, np.uint32)
        bind_w = np.zeros((num_points, 4), f32)
        for ci, cage in enumerate(cages):
            mn, mx = cage.mesh.bounds()
            t, w = pipeline.bind_tets(cage.mesh, bounds=(mn, mx))
            take = (bind_cage == UNBOUND) & (t != UNBOUND)
            bind_cage[take] = ci
            bind_tet[take] = t[take]
            bind_w[take] = w[take]
        return CageScene(cages, bind_cage, bind_tet, bind_w)

    def step(self, dt: float) -> None:
        for c in self.cages:
            c.simulator.step(dt)

    def flatten(self):
        """Global tet topology across cages and global bindings
        (gpu_state.rs:248-293): vertex indices offset per cage, bindings mapped
        to the flattened tet index, 0xFFFFFFFF when unbound."""
        elems, inv, toff, voff = [], [], [], 0
        tcount = 0
        for c in self.cages:
            toff.append(tcount)
            elems.append(c.mesh.elements.astype(np.uint64) + voff)
            inv.append(c.mesh.inv_dm)
            voff += c.mesh.num_vertices
            tcount += c.mesh.num_tets
        elems = np.concatenate(elems).astype(np.uint32) if elems else np.zeros((0, 4), np.uint32)
        inv = np.concatenate(inv).astype(f32) if inv else np.zeros((0, 9), f32)
        toff = np.asarray(toff, np.uint64)
        gt = np.full(self.bind_cage.shape[0], UNBOUND, np.uint32)
        bound = self.bind_cage != UNBOUND
        gt[bound] = (toff[self.bind_cage[bound]] + self.bind_tet[bound]).astype(np.uint32)
        w = np.where(bound[:, None], self.bind_w, f32(0.0)).astype(f32)
        return elems, inv, voff, gt, w

    def flat_vertices(self) -> np.ndarray:
        return np.concatenate([c.vertices() for c in self.cages]).astype(f32)
