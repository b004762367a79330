"""Camera and compositor uniform blocks (render/camera.rs, rasterizer/mod.rs)."""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

f32 = np.float32


def _normalize(v):
    v = np.asarray(v, f32)
    d = (v[0] * v[0] + v[1] * v[1]) + v[2] * v[2]
    return (v * (f32(1.0) / np.sqrt(d))).astype(f32)


def _cross(a, b):
    return np.array([a[1] * b[2] - b[1] * a[2], a[2] * b[0] - b[2] * a[0],
                     a[0] * b[1] - b[0] * a[1]], f32)


def _dot(a, b):
    return f32((a[0] * b[0] + a[1] * b[1]) + a[2] * b[2])


def look_at_lh(eye, target, up) -> np.ndarray:
    """glam Mat4::look_at_lh as a column-major [16] array: rows s, u, d with
    d = normalize(target - eye), s = normalize(up x d), u = d x s; camera z
    grows along the view direction (render/camera.rs:80)."""
    eye = np.asarray(eye, f32)
    d = _normalize(np.asarray(target, f32) - eye)
    f = (-d).astype(f32)  # look_to_rh's forward
    s = _normalize(_cross(f, np.asarray(up, f32)))
    u = _cross(s, f)
    cols = np.array([[s[0], u[0], -f[0], 0.0], [s[1], u[1], -f[1], 0.0], [s[2], u[2], -f[2], 0.0],
                     [-_dot(eye, s), -_dot(eye, u), _dot(eye, f), 1.0]], f32)
    return cols.ravel()


@dataclass
class CameraUniforms:
    """96-byte camera block: column-major view matrix + intrinsics (camera.rs:9-36)."""
    view_matrix: np.ndarray = field(default_factory=lambda: np.eye(4, dtype=f32).ravel())
    focal_x: float = 1.0
    focal_y: float = 1.0
    principal_x: float = 0.0
    principal_y: float = 0.0
    viewport_width: float = 1.0
    viewport_height: float = 1.0
    near_plane: float = 0.2

    @staticmethod
    def from_look_at(eye, target, up, fov_y_radians, viewport_width, viewport_height,
                     near_plane=0.2) -> "CameraUniforms":
        """CameraUniforms::from_look_at (camera.rs:71-96)."""
        fy = f32(0.5) * f32(viewport_height) / np.tan(f32(0.5) * f32(fov_y_radians))
        return CameraUniforms(look_at_lh(eye, target, up), float(fy), float(fy),
                              float(f32(0.5) * f32(viewport_width)),
                              float(f32(0.5) * f32(viewport_height)), float(viewport_width),
                              float(viewport_height), float(near_plane))

    def to_array(self) -> np.ndarray:
        a = np.zeros(24, f32)
        a[:16] = np.asarray(self.view_matrix, f32).ravel()
        a[16:23] = [self.focal_x, self.focal_y, self.principal_x, self.principal_y,
                    self.viewport_width, self.viewport_height, self.near_plane]
        return a

    def eye(self) -> np.ndarray:
        """World-space camera position (inverse of the rigid view transform)."""
        v = np.asarray(self.view_matrix, np.float64).reshape(4, 4).T  # row-major
        R, t = v[:3, :3], v[:3, 3]
        return (-R.T @ t).astype(f32)


@dataclass
class CompositorUniforms:
    """48-byte compositor block (rasterizer/mod.rs:16-37)."""
    screen_width: int
    screen_height: int
    background_color: tuple = (0.0, 0.0, 0.0, 1.0)
    camera_position: tuple = (0.0, 0.0, 0.0)
    sh_degree: int = 0

    @property
    def tiles_x(self) -> int:
        return (self.screen_width + 15) // 16

    @property
    def tiles_y(self) -> int:
        return (self.screen_height + 15) // 16


def orbit_camera(frame: int, frames: int, radius: float, width: int, height: int,
                 fov_deg: float = 60.0, height_y: float = 0.0) -> CameraUniforms:
    """Camera on a horizontal orbit of `radius` around the origin, looking at it."""
    ang = 2.0 * np.pi * frame / max(frames, 1)
    eye = (radius * np.sin(ang), height_y, radius * np.cos(ang))
    return CameraUniforms.from_look_at(eye, (0, 0, 0), (0, 1, 0), np.deg2rad(fov_deg), width,
                                       height, 0.2)
