"""Polygon cages for mean value coordinates (deformation/mvc.rs).

PolyCageMesh mirrors the reference type: a closed, outward-oriented triangle
surface with the reference's presets (box, octahedron, icosahedron), an OBJ
parser, the closed-manifold and signed-volume checks, and the generalised
winding number used as the inside test. `icosphere` and `displace_sinusoids`
build the polygon cage of the MVC workload (a level-3 icosphere of radius
1.15, 642 vertices and 1,280 triangles, displaced by a smooth field). The
weights, bindings and the deformation itself run on the GPU through the C ABI
(`GpuPipelineState.mvc_*`).
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

f32 = np.float32


@dataclass
class PolyCageMesh:
    rest_vertices: np.ndarray  # [V, 3] f32
    triangles: np.ndarray      # [F, 3] u32, outward counter-clockwise

    def __post_init__(self):
        self.rest_vertices = np.ascontiguousarray(self.rest_vertices, f32).reshape(-1, 3)
        self.triangles = np.ascontiguousarray(self.triangles, np.uint32).reshape(-1, 3)

    @staticmethod
    def new(rest_vertices, triangles) -> "PolyCageMesh":
        """PolyCageMesh::new (mvc.rs:82-109): validates sizes and indices."""
        v = np.asarray(rest_vertices, f32).reshape(-1, 3)
        t = np.asarray(triangles, np.int64).reshape(-1, 3)
        if v.shape[0] < 4:
            raise ValueError("polyhedral cage requires at least 4 vertices")
        if t.shape[0] < 4:
            raise ValueError("polyhedral cage requires at least 4 triangles")
        for ti, tri in enumerate(t):
            if (tri >= v.shape[0]).any() or (tri < 0).any():
                raise ValueError(f"triangle {ti} references out-of-bounds vertex index {tri.tolist()}"
                                 f" (vertex count {v.shape[0]})")
            if tri[0] == tri[1] or tri[1] == tri[2] or tri[2] == tri[0]:
                raise ValueError(f"triangle {ti} is degenerate with repeated vertex {tri.tolist()}")
        return PolyCageMesh(v, t.astype(np.uint32))

    @property
    def num_vertices(self) -> int:
        return int(self.rest_vertices.shape[0])

    @property
    def num_triangles(self) -> int:
        return int(self.triangles.shape[0])

    # -- presets (mvc.rs:112-244) --------------------------------------------------
    @staticmethod
    def create_box_surface_cage(mn, mx) -> "PolyCageMesh":
        v = [[mn[0], mn[1], mn[2]], [mx[0], mn[1], mn[2]], [mx[0], mx[1], mn[2]],
             [mn[0], mx[1], mn[2]], [mn[0], mn[1], mx[2]], [mx[0], mn[1], mx[2]],
             [mx[0], mx[1], mx[2]], [mn[0], mx[1], mx[2]]]
        t = [[0, 2, 1], [0, 3, 2], [4, 5, 6], [4, 6, 7], [0, 1, 5], [0, 5, 4], [3, 7, 6],
             [3, 6, 2], [0, 4, 7], [0, 7, 3], [1, 2, 6], [1, 6, 5]]
        return PolyCageMesh(np.array(v, f32), np.array(t, np.uint32))

    @staticmethod
    def create_octahedron_cage(center, radius) -> "PolyCageMesh":
        c = np.asarray(center, f32)
        r = f32(max(abs(float(radius)), 1e-4))
        d = np.array([[r, 0, 0], [-r, 0, 0], [0, r, 0], [0, -r, 0], [0, 0, r], [0, 0, -r]], f32)
        t = [[0, 2, 4], [2, 1, 4], [1, 3, 4], [3, 0, 4], [2, 0, 5], [1, 2, 5], [3, 1, 5],
             [0, 3, 5]]
        return PolyCageMesh((c[None, :] + d).astype(f32), np.array(t, np.uint32))

    @staticmethod
    def create_icosahedron_cage(center, radius) -> "PolyCageMesh":
        c = np.asarray(center, f32)
        r = f32(max(abs(float(radius)), 1e-4))
        phi = (f32(1.0) + np.sqrt(f32(5.0))) * f32(0.5)
        raw = np.array([[-1, phi, 0], [1, phi, 0], [-1, -phi, 0], [1, -phi, 0], [0, -1, phi],
                        [0, 1, phi], [0, -1, -phi], [0, 1, -phi], [phi, 0, -1], [phi, 0, 1],
                        [-phi, 0, -1], [-phi, 0, 1]], f32)
        inv = f32(1.0) / np.sqrt((raw * raw).sum(1, dtype=f32)).astype(f32)
        v = c[None, :] + (raw * inv[:, None]).astype(f32) * r
        t = [[0, 11, 5], [0, 5, 1], [0, 1, 7], [0, 7, 10], [0, 10, 11], [1, 5, 9], [5, 11, 4],
             [11, 10, 2], [10, 7, 6], [7, 1, 8], [3, 9, 4], [3, 4, 2], [3, 2, 6], [3, 6, 8],
             [3, 8, 9], [4, 9, 5], [2, 4, 11], [6, 2, 10], [8, 6, 7], [9, 8, 1]]
        return PolyCageMesh(v.astype(f32), np.array(t, np.uint32))

    @staticmethod
    def icosphere(center, radius, level: int) -> "PolyCageMesh":
        """Icosahedron subdivided `level` times (each triangle into four, new
        vertices at edge midpoints pushed to the sphere): level 3 has 642
        vertices and 1,280 triangles. Vertex order: the 12 icosahedron
        vertices, then midpoints in order of first use."""
        base = PolyCageMesh.create_icosahedron_cage([0, 0, 0], 1.0)
        verts = [tuple(p) for p in base.rest_vertices.astype(np.float64)]
        tris = [tuple(int(x) for x in t) for t in base.triangles]
        for _ in range(level):
            mid = {}
            nt = []

            def midpoint(a, b):
                key = (min(a, b), max(a, b))
                if key not in mid:
                    p = np.add(verts[a], verts[b]) * 0.5
                    p = p / np.linalg.norm(p)
                    mid[key] = len(verts)
                    verts.append(tuple(p))
                return mid[key]

            for a, b, c in tris:
                ab, bc, ca = midpoint(a, b), midpoint(b, c), midpoint(c, a)
                nt += [(a, ab, ca), (b, bc, ab), (c, ca, bc), (ab, bc, ca)]
            tris = nt
        v = np.asarray(center, np.float64)[None, :] + np.array(verts) * float(radius)
        return PolyCageMesh(v.astype(f32), np.array(tris, np.uint32))

    def displace_sinusoids(self, amplitude: float = 0.1, waves: int = 8,
                           seed: int = 0) -> "PolyCageMesh":
        """Moves every vertex along its direction from the centroid by
        amplitude * f(v) / max|f|, f(v) = sum_k sin(k_k . v + phase_k) over
        `waves` wave vectors of random direction and length in [2, 4] with
        uniform phases (numpy PCG64 stream `seed`): a smooth random field whose
        largest displacement is `amplitude`."""
        rng = np.random.default_rng(seed)
        dirs = rng.normal(size=(waves, 3))
        dirs /= np.linalg.norm(dirs, axis=1, keepdims=True)
        k = dirs * rng.uniform(2.0, 4.0, size=(waves, 1))
        phase = rng.uniform(0.0, 2.0 * np.pi, size=waves)
        v = self.rest_vertices.astype(np.float64)
        c = v.mean(0)
        field = np.sin(v @ k.T + phase[None, :]).mean(1)
        field /= max(np.abs(field).max(), 1e-12)  # peak displacement = amplitude
        d = v - c
        d /= np.linalg.norm(d, axis=1, keepdims=True)
        return PolyCageMesh((v + amplitude * field[:, None] * d).astype(f32), self.triangles.copy())

    # -- checks (mvc.rs:315-337) ------------------------------------------------------
    def is_closed_manifold(self) -> bool:
        half = {}
        for a, b, c in self.triangles.tolist():
            for e in ((a, b), (b, c), (c, a)):
                half[e] = half.get(e, 0) + 1
                if half[e] > 1:
                    return False
        return len(self.triangles) > 0 and all((v, u) in half for (u, v) in half)

    def signed_volume(self) -> float:
        v = self.rest_vertices.astype(np.float64)
        a, b, c = (v[self.triangles[:, k]] for k in range(3))
        return float((a * np.cross(b, c)).sum() / 6.0)

    def winding_numbers(self, points) -> np.ndarray:
        """Generalised winding number of each point (mvc.rs:339-357), f64."""
        p = np.asarray(points, np.float64).reshape(-1, 3)
        v = self.rest_vertices.astype(np.float64)
        out = np.zeros(p.shape[0])
        on_vertex = np.zeros(p.shape[0], bool)
        for i0, i1, i2 in self.triangles:
            a, b, c = v[i0] - p, v[i1] - p, v[i2] - p
            la, lb, lc = (np.linalg.norm(x, axis=1) for x in (a, b, c))
            on_vertex |= (la < 1e-7) | (lb < 1e-7) | (lc < 1e-7)
            det = (a * np.cross(b, c)).sum(1)
            den = la * lb * lc + (a * b).sum(1) * lc + (b * c).sum(1) * la + (c * a).sum(1) * lb
            out += 2.0 * np.arctan2(det, den)
        out /= 4.0 * np.pi
        out[on_vertex] = 1.0  # a point on a cage vertex counts as inside (mvc.rs:347-349)
        return out

    @staticmethod
    def from_obj_str(obj: str) -> "PolyCageMesh":
        """from_obj_str (mvc.rs:247-306): `v` records and fanned `f` records."""
        verts, tris = [], []
        for line_no, raw in enumerate(obj.splitlines()):
            line = raw.split("#")[0].strip()
            if not line:
                continue
            parts = line.split()
            if parts[0] == "v":
                if len(parts) < 4:
                    raise ValueError(f"line {line_no + 1}: expected 3 coordinates for 'v'")
                verts.append([float(x) for x in parts[1:4]])
            elif parts[0] == "f":
                idx = []
                for tok in parts[1:]:
                    s = int(tok.split("/")[0])
                    if s > 0:
                        idx.append(s - 1)
                    elif s < 0:
                        r = len(verts) + s
                        if r < 0:
                            raise ValueError(f"line {line_no + 1}: negative face index {s} out of bounds")
                        idx.append(r)
                    else:
                        raise ValueError(f"line {line_no + 1}: 0 is not a valid OBJ index")
                if len(idx) < 3:
                    raise ValueError(f"line {line_no + 1}: face must have at least 3 vertices")
                for i in range(1, len(idx) - 1):
                    tris.append([idx[0], idx[i], idx[i + 1]])
        return PolyCageMesh.new(verts, tris)

    def vertex_faces(self):
        """Per-vertex incident faces in ascending face order, CSR:
        (offsets [V+1], entries face << 2 | corner)."""
        V = self.num_vertices
        lists = [[] for _ in range(V)]
        for f, tri in enumerate(self.triangles.tolist()):
            for c, v in enumerate(tri):
                lists[v].append((f << 2) | c)
        off = np.zeros(V + 1, np.uint32)
        off[1:] = np.cumsum([len(x) for x in lists])
        flat = np.array([e for x in lists for e in x], np.uint32)
        return off, flat
