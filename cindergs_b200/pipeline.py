"""GpuPipelineState: the reference's persistent four-stage GPU frame API
(render/gpu_state.rs:538-1343) on top of the sm_100a C library.

    state = GpuPipelineState()
    timings = state.execute_frame_gpu(scene, cages, camera, compositor,
                                      strain_split_threshold, mip_filter_3d_var,
                                      min_opacity, min_radius_px,
                                      profile_stages, force_stage3)
    rgba8 = state.readback_framebuffer_rgba8(width, height)

Residency rules follow GpuSceneState::sync_scene_and_cages
(gpu_state.rs:182-343): the rest scene is re-uploaded when its fingerprint
(array identities, size and a 64-sample value hash) changes, the cage
topology when the cage list or bindings change, and cage vertices every call
(the library skips Stage 1 when they are unchanged).
"""
from __future__ import annotations

import ctypes
import hashlib
from dataclasses import dataclass

import numpy as np

from . import _abi
from .camera import CameraUniforms, CompositorUniforms
from .cage import CageScene, TetMesh, UNBOUND
from .scene import GaussianSceneSoa, QuantizedGaussianSceneSoa

f32 = np.float32


@dataclass
class GpuStageTimings:
    """GpuStageTimings (gpu_state.rs:513-534)."""
    stage1_deform_ms: float = 0.0
    stage2_project_ms: float = 0.0
    stage3_bin_sort_ms: float = 0.0
    stage4_composite_ms: float = 0.0
    stage1_skipped: bool = False
    stage3_cached: bool = False
    used_hardware_timestamps: bool = False
    used_64bit_keys: bool = False
    active_gaussians: int = 0
    surviving_gaussians: int = 0
    total_tile_entries: int = 0

    @property
    def total_ms(self) -> float:
        return (self.stage1_deform_ms + self.stage2_project_ms + self.stage3_bin_sort_ms +
                self.stage4_composite_ms)


def scene_fingerprint(scene: GaussianSceneSoa) -> bytes:
    """Change detector of GpuSceneState (scene_fingerprint, gpu_state.rs:65-79):
    count, array identities and 64 evenly spaced samples (plus the last value)
    of each array, hashed with BLAKE2b."""
    h = hashlib.blake2b(digest_size=16)
    h.update(int(scene.count).to_bytes(8, "little"))
    arrays = (scene.fingerprint_arrays() if hasattr(scene, "fingerprint_arrays") else
              (scene.positions, scene.covariances_3d, scene.opacities, scene.sh_coeffs))
    for arr in arrays:
        h.update(int(arr.ctypes.data).to_bytes(8, "little"))
        flat = arr.reshape(-1)
        h.update(int(flat.size).to_bytes(8, "little"))
        step = max(flat.size // 64, 1)
        h.update(flat[::step].tobytes())
        if flat.size:
            h.update(flat[-1:].tobytes())
    return h.digest()


def _p(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


class GpuPipelineState:
    """Persistent GPU state: scene residency + frame arena, on one device."""

    def __init__(self, device: int = 0, stream: int | None = None):
        self._lib = _abi.load()
        self._ctx = ctypes.c_void_p()
        rc = self._lib.cgs_ctx_create(int(device), ctypes.c_void_p(stream or 0),
                                      ctypes.byref(self._ctx))
        if rc != _abi.CGS_OK:
            raise _abi.CgsError(rc, "cgs_ctx_create", "could not create a CUDA context")
        self.device = int(device)
        self._scene_hash = None
        self._scene_count = -1
        self._cage_key = None
        self._last = None
        self._mvc_V = 0
        self._device_springs = False
        self._num_cage_verts = 0

    # -- lifetime -------------------------------------------------------------
    def close(self) -> None:
        if self._ctx:
            self._lib.cgs_ctx_destroy(self._ctx)
            self._ctx = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc: int, fn: str) -> None:
        _abi.check(rc, fn, self._ctx)

    @property
    def handle(self) -> ctypes.c_void_p:
        return self._ctx

    # -- residency ------------------------------------------------------------
    def upload_scene(self, scene) -> None:
        """GaussianSceneSoa (f32 or f16 SH) or QuantizedGaussianSceneSoa."""
        if isinstance(scene, QuantizedGaussianSceneSoa):
            pos = np.ascontiguousarray(scene.positions, f32)
            cov = np.ascontiguousarray(scene.covariances_f16_packed, np.uint32)
            opa = np.ascontiguousarray(scene.opacities, f32)
            sh = np.ascontiguousarray(scene.sh_coeffs_f16_packed, np.uint32)
            self._check(self._lib.cgs_scene_upload_quantized(self._ctx, scene.count, _p(pos),
                                                             _p(cov), _p(opa), _p(sh),
                                                             int(scene.sh_degree)),
                        "cgs_scene_upload_quantized")
            self._scene_hash = scene_fingerprint(scene)
            self._scene_count = scene.count
            self._cage_key = None
            return
        pos = np.ascontiguousarray(scene.positions, f32)
        cov = np.ascontiguousarray(scene.covariances_3d, f32)
        opa = np.ascontiguousarray(scene.opacities, f32)
        if scene.sh_coeffs.dtype == np.float16:
            sh, fmt = np.ascontiguousarray(scene.sh_coeffs), _abi.CGS_SH_F16
        else:
            sh, fmt = np.ascontiguousarray(scene.sh_coeffs, f32), _abi.CGS_SH_F32
        self._check(self._lib.cgs_scene_upload(self._ctx, scene.count, _p(pos), _p(cov), _p(opa),
                                               _p(sh), fmt), "cgs_scene_upload")
        self._scene_hash = scene_fingerprint(scene)
        self._scene_count = scene.count
        self._cage_key = None

    def upload_cages(self, cages: CageScene | None) -> None:
        self._device_springs = False
        self._num_cage_verts = 0 if cages is None else sum(c.mesh.num_vertices for c in cages.cages)
        if cages is None or not cages.cages:
            self._check(self._lib.cgs_tet_cages_upload(self._ctx, 0, None, None, 0, None, None),
                        "cgs_tet_cages_upload")
            self._cage_key = ("none",)
            return
        elems, inv, nverts, bt, bw = cages.flatten()
        self._check(self._lib.cgs_tet_cages_upload(self._ctx, elems.shape[0], _p(elems), _p(inv),
                                                   nverts, _p(bt), _p(bw)),
                    "cgs_tet_cages_upload")
        self._cage_key = (id(cages), cages.bind_tet.ctypes.data, len(cages.cages),
                          tuple((id(c.mesh), c.mesh.num_tets, c.mesh.num_vertices)
                                for c in cages.cages))

    def sync_scene_and_cages(self, scene: GaussianSceneSoa, cages: CageScene | None) -> None:
        h = scene_fingerprint(scene)
        if h != self._scene_hash or scene.count != self._scene_count:
            self.upload_scene(scene)
        if cages is None or not cages.cages:
            if self._cage_key != ("none",):
                self.upload_cages(None)
            return
        key = (id(cages), cages.bind_tet.ctypes.data, len(cages.cages),
               tuple((id(c.mesh), c.mesh.num_tets, c.mesh.num_vertices) for c in cages.cages))
        if key != self._cage_key:
            self.upload_cages(cages)
        if self._device_springs:
            return  # the cage state lives on the device (springs_upload)
        v = np.ascontiguousarray(cages.flat_vertices(), f32)
        self._check(self._lib.cgs_cage_vertices_update(self._ctx, _p(v), v.shape[0]),
                    "cgs_cage_vertices_update")

    # -- cage springs on the device ------------------------------------------------
    def springs_upload(self, cages: CageScene) -> None:
        """Moves every cage's CageSpringSimulator state (rest, current,
        velocity, pins, stiffness / damping / mass, collision planes) to the
        device; frames then deform with the device state and the host stops
        uploading cage vertices (cgs_springs_upload). Upload the cages first."""
        specs, planes, first = [], [], 0
        for c in cages.cages:
            sim = c.simulator
            spec = _abi.CgsSpringCage(float(sim.stiffness), float(sim.damping), float(sim.mass),
                                      first, sim.rest_positions.shape[0], len(planes),
                                      len(sim.collision_planes), 0)
            for pl in sim.collision_planes:
                planes.append(_abi.CgsCollisionPlane((ctypes.c_float * 3)(*map(float, pl.normal)),
                                                     float(pl.offset), float(pl.restitution),
                                                     float(pl.friction)))
            specs.append(spec)
            first += sim.rest_positions.shape[0]
        rest = np.ascontiguousarray(np.concatenate([c.simulator.rest_positions for c in cages.cages]), f32)
        cur = np.ascontiguousarray(np.concatenate([c.simulator.current_positions for c in cages.cages]), f32)
        vel = np.ascontiguousarray(np.concatenate([c.simulator.velocities for c in cages.cages]), f32)
        pin = np.ascontiguousarray(np.concatenate([c.simulator.pinned for c in cages.cages]), np.uint8)
        spec_arr = (_abi.CgsSpringCage * len(specs))(*specs)
        plane_arr = (_abi.CgsCollisionPlane * max(len(planes), 1))(*planes)
        self._check(self._lib.cgs_springs_upload(self._ctx, len(specs), spec_arr, len(planes),
                                                 plane_arr if planes else None, rest.shape[0],
                                                 _p(rest), _p(cur), _p(vel), _p(pin)),
                    "cgs_springs_upload")
        self._device_springs = True

    def springs_step(self, dt: float, steps: int = 1) -> None:
        """Enqueues `steps` spring steps of `dt` on the device (cgs_springs_step)."""
        self._check(self._lib.cgs_springs_step(self._ctx, float(dt), int(steps)), "cgs_springs_step")

    def springs_impulse(self, magnitude: float) -> None:
        """trigger_jiggle_impulse on every device cage (cgs_springs_impulse)."""
        self._check(self._lib.cgs_springs_impulse(self._ctx, float(magnitude)), "cgs_springs_impulse")

    def springs_read(self) -> tuple[np.ndarray, np.ndarray]:
        """Device cage positions and velocities [V,3] (cgs_springs_read)."""
        n = self._num_cage_verts
        cur, vel = np.empty((n, 3), f32), np.empty((n, 3), f32)
        self._check(self._lib.cgs_springs_read(self._ctx, _p(cur), _p(vel)), "cgs_springs_read")
        return cur, vel

    def bind_tets(self, mesh: TetMesh, bounds=None):
        """GPU barycentric binding of the resident scene to `mesh`
        (TetMesh::bind_point). Returns (tet [N] u32, weights [N,4] f32)."""
        n = max(self._scene_count, 0)
        tets = np.zeros(n, np.uint32)
        w = np.zeros((n, 4), f32)
        elems = np.ascontiguousarray(mesh.elements, np.uint32)
        inv = np.ascontiguousarray(mesh.inv_dm, f32)
        rv = np.ascontiguousarray(mesh.rest_vertices, f32)
        if bounds is not None:
            bmin = np.ascontiguousarray(bounds[0], f32)
            bmax = np.ascontiguousarray(bounds[1], f32)
            ub, pmin, pmax = 1, _p(bmin), _p(bmax)
        else:
            ub, pmin, pmax = 0, None, None
        self._check(self._lib.cgs_bind_tets(self._ctx, mesh.num_tets, _p(elems), _p(inv),
                                            mesh.num_vertices, _p(rv), ub, pmin, pmax, _p(tets),
                                            _p(w)), "cgs_bind_tets")
        return tets, w

    # -- polygon cage (mean value coordinates) -----------------------------------
    def mvc_cage_upload(self, cage) -> None:
        """Uploads a PolyCageMesh (cindergs_b200.mvc) and drops earlier MVC bindings."""
        v = np.ascontiguousarray(cage.rest_vertices, f32)
        t = np.ascontiguousarray(cage.triangles, np.uint32)
        self._check(self._lib.cgs_mvc_cage_upload(self._ctx, v.shape[0], _p(v), t.shape[0], _p(t)),
                    "cgs_mvc_cage_upload")
        self._mvc_V = int(v.shape[0])

    def mvc_vertices_update(self, verts) -> None:
        v = np.ascontiguousarray(verts, f32).reshape(-1, 3)
        self._check(self._lib.cgs_mvc_vertices_update(self._ctx, _p(v), v.shape[0]),
                    "cgs_mvc_vertices_update")

    def mvc_bind(self) -> int:
        """PolyCageMesh::bind_gaussians (mvc.rs:498-541) for the resident scene
        on the GPU; returns how many Gaussians were bound."""
        nb = ctypes.c_uint32(0)
        self._check(self._lib.cgs_mvc_bind(self._ctx, ctypes.byref(nb)), "cgs_mvc_bind")
        return int(nb.value)

    def mvc_weights(self, points):
        """Exact MVC weights of points against the rest cage: a torch CUDA
        tensor [n, 3] -> [n, V] (device), or numpy -> numpy."""
        import torch
        host = not (isinstance(points, torch.Tensor) and points.is_cuda)
        pts = torch.as_tensor(np.asarray(points, f32) if host else points, dtype=torch.float32)
        pts = pts.reshape(-1, 3).contiguous().to(f"cuda:{self.device}")
        out = torch.empty((pts.shape[0], self._mvc_V), dtype=torch.float32, device=pts.device)
        torch.cuda.synchronize(pts.device)
        self._check(self._lib.cgs_mvc_weights(self._ctx, pts.shape[0], ctypes.c_void_p(pts.data_ptr()),
                                              ctypes.c_void_p(out.data_ptr())), "cgs_mvc_weights")
        return out.cpu().numpy() if host else out

    def mvc_read_bindings(self, max_slots: int | None = None):
        """(gaussian index [k] u32, wg [k, V, 4] f32) of the first k MVC bindings."""
        k = int(max_slots if max_slots is not None else 1 << 62)
        cnt = ctypes.c_uint64(0)
        self._check(self._lib.cgs_mvc_read_bindings(self._ctx, 0, None, None, ctypes.byref(cnt)),
                    "cgs_mvc_read_bindings")
        n = min(k, self._mvc_bound_hint()) if k else 0
        g = np.zeros(max(n, 1), np.uint32)
        wg = np.zeros((max(n, 1), self._mvc_V, 4), f32)
        self._check(self._lib.cgs_mvc_read_bindings(self._ctx, n, _p(g), _p(wg), ctypes.byref(cnt)),
                    "cgs_mvc_read_bindings")
        n = int(cnt.value)
        return g[:n], wg[:n]

    # -- learned MVC field -------------------------------------------------------
    def _dev_f32(self, a, cols: int):
        import torch
        host = not (isinstance(a, torch.Tensor) and a.is_cuda)
        t = torch.as_tensor(np.asarray(a, f32) if host else a, dtype=torch.float32)
        return t.reshape(-1, cols).contiguous().to(f"cuda:{self.device}"), host

    def mvc_field_create(self, seed: int = 0) -> None:
        """New seeded network for the uploaded polygon cage (drops learned bindings)."""
        self._check(self._lib.cgs_mvc_field_create(self._ctx, int(seed)), "cgs_mvc_field_create")

    def mvc_field_layout(self) -> tuple[dict, int, np.ndarray]:
        """({name: offset} for W1, b1, ... W5, b5, total floats, enc [c, 1/s])."""
        off = np.zeros(10, np.uint32)
        tot = ctypes.c_uint32(0)
        enc = np.zeros(4, f32)
        self._check(self._lib.cgs_mvc_field_layout(self._ctx, _p(off), ctypes.byref(tot), _p(enc)),
                    "cgs_mvc_field_layout")
        names = ["W1", "b1", "W2", "b2", "W3", "b3", "W4", "b4", "W5", "b5"]
        return dict(zip(names, (int(o) for o in off))), int(tot.value), enc

    def mvc_field_params(self, values=None) -> np.ndarray:
        """The fp32 parameter block; with `values`, loads it first (resets Adam)."""
        _, tot, _ = self.mvc_field_layout()
        src = None
        if values is not None:
            src = np.ascontiguousarray(values, f32).reshape(-1)
            if src.size != tot:
                raise ValueError(f"expected {tot} parameters, got {src.size}")
        out = np.zeros(tot, f32)
        self._check(self._lib.cgs_mvc_field_params(self._ctx, None, None if src is None else _p(src)),
                    "cgs_mvc_field_params")
        self._check(self._lib.cgs_mvc_field_params(self._ctx, _p(out), None), "cgs_mvc_field_params")
        return out

    def mvc_field_train(self, points, weights, steps: int, batch: int = 4096, lr: float = 1e-3,
                        lam: float = 1.0, seed: int = 1) -> tuple[float, float]:
        """Adam steps on (points [n, 3], exact weights [n, V]); returns the weight
        and residual loss terms averaged over the last tenth of the steps."""
        import torch
        pts, _ = self._dev_f32(points, 3)
        w, _ = self._dev_f32(weights, self._mvc_V)
        torch.cuda.synchronize(pts.device)
        loss = np.zeros(2, f32)
        self._check(self._lib.cgs_mvc_field_train(self._ctx, pts.shape[0],
                                                  ctypes.c_void_p(pts.data_ptr()),
                                                  ctypes.c_void_p(w.data_ptr()), int(steps),
                                                  int(batch), float(lr), float(lam), int(seed),
                                                  _p(loss)), "cgs_mvc_field_train")
        return float(loss[0]), float(loss[1])

    def mvc_field_grads(self, points, weights, lam: float = 1.0):
        """(gradient of the loss over all rows [total], (weight term, residual term))."""
        import torch
        pts, _ = self._dev_f32(points, 3)
        w, _ = self._dev_f32(weights, self._mvc_V)
        torch.cuda.synchronize(pts.device)
        _, tot, _ = self.mvc_field_layout()
        g = np.zeros(tot, f32)
        loss = np.zeros(2, f32)
        self._check(self._lib.cgs_mvc_field_grads(self._ctx, pts.shape[0],
                                                  ctypes.c_void_p(pts.data_ptr()),
                                                  ctypes.c_void_p(w.data_ptr()), float(lam), _p(g),
                                                  _p(loss)), "cgs_mvc_field_grads")
        return g, (float(loss[0]), float(loss[1]))

    def mvc_field_eval(self, points):
        """Network weights [n, V] of points [n, 3] (device tensor in, device out;
        numpy in, numpy out)."""
        import torch
        pts, host = self._dev_f32(points, 3)
        out = torch.empty((pts.shape[0], self._mvc_V), dtype=torch.float32, device=pts.device)
        torch.cuda.synchronize(pts.device)
        self._check(self._lib.cgs_mvc_field_eval(self._ctx, pts.shape[0],
                                                 ctypes.c_void_p(pts.data_ptr()),
                                                 ctypes.c_void_p(out.data_ptr())),
                    "cgs_mvc_field_eval")
        return out.cpu().numpy() if host else out

    def mvc_field_infer(self, points, rest: bool = False):
        """Fused inference: (positions [n, 3], gradients F [n, 3, 3]) on the
        current cage (rest cage with rest=True)."""
        import torch
        pts, host = self._dev_f32(points, 3)
        out = torch.empty((pts.shape[0], 12), dtype=torch.float32, device=pts.device)
        torch.cuda.synchronize(pts.device)
        self._check(self._lib.cgs_mvc_field_infer(self._ctx, pts.shape[0],
                                                  ctypes.c_void_p(pts.data_ptr()), int(rest),
                                                  ctypes.c_void_p(out.data_ptr())),
                    "cgs_mvc_field_infer")
        pos = out[:, :3]
        F = out[:, 3:].reshape(-1, 3, 3).transpose(1, 2)  # stored column-major
        if host:
            return pos.cpu().numpy(), F.cpu().numpy()
        return pos, F

    def mvc_bind_learned(self, threshold: float, per_frame: bool = False) -> tuple[int, int]:
        """Binds the polygon cage with the network where its linear-precision
        residual on the rest cage is at most threshold (relative to the cage
        half-extent); returns (bound, exact fallbacks). Frames apply the output
        layer to codes kept per Gaussian, or evaluate the whole network every
        frame with per_frame=True."""
        nb, nfb = ctypes.c_uint32(0), ctypes.c_uint32(0)
        flags = _abi.FIELD_PER_FRAME if per_frame else 0
        self._check(self._lib.cgs_mvc_bind_learned(self._ctx, float(threshold), flags,
                                                   ctypes.byref(nb), ctypes.byref(nfb)),
                    "cgs_mvc_bind_learned")
        return int(nb.value), int(nfb.value)

    def _mvc_bound_hint(self) -> int:
        cnt = ctypes.c_uint64(0)
        self._check(self._lib.cgs_mvc_read_bindings(self._ctx, 1 << 62, None, None,
                                                    ctypes.byref(cnt)), "cgs_mvc_read_bindings")
        return int(cnt.value)

    # -- frame ------------------------------------------------------------------
    def execute_frame_gpu(self, scene: GaussianSceneSoa, cages: CageScene | None,
                          camera: CameraUniforms, compositor: CompositorUniforms,
                          strain_split_threshold: float = 0.0, mip_filter_3d_var: float = 0.0,
                          min_opacity: float = 1.0 / 255.0, min_radius_px: float = 0.5,
                          profile_stages: bool = False, force_stage3: bool = False,
                          write_f32: bool = False, radix_bits: int = 0,
                          stage_timings: bool = True, entry_sort: int = 0,
                          tile_shape: int = 0) -> GpuStageTimings:
        """execute_frame_gpu (gpu_state.rs:613-1243). With stage_timings (the
        default) the call waits for the frame and returns its counts (and, with
        profile_stages, per-stage device ms); with stage_timings=False the frame
        is only enqueued (no host synchronisation), its kernel times still
        accumulate when profile_stages is set (read them with kernel_profile()),
        and the returned timings are all zero. radix_bits and entry_sort choose
        how the tile entries are sorted (include/cgs.h: CGS_SORT_*); every
        choice gives the same lists. tile_shape is the screen tile of Stages 3
        and 4 (CGS_TILE_*: the reference's 16x16 by default, 8x8 or 32x16)."""
        self.sync_scene_and_cages(scene, cages)
        cam = self._camera(camera)
        comp = self._compositor(compositor)
        params = _abi.CgsFrameParams(float(strain_split_threshold), float(mip_filter_3d_var),
                                     float(min_opacity), float(min_radius_px),
                                     int(bool(profile_stages)), int(bool(force_stage3)),
                                     int(bool(write_f32)), int(radix_bits), int(entry_sort),
                                     int(tile_shape))
        t = _abi.CgsStageTimings()
        tp = ctypes.byref(t) if stage_timings else None
        self._check(self._lib.cgs_execute_frame(self._ctx, ctypes.byref(cam), ctypes.byref(comp),
                                                ctypes.byref(params), tp),
                    "cgs_execute_frame")
        self._last = (compositor.screen_width, compositor.screen_height)
        return GpuStageTimings(t.stage1_deform_ms, t.stage2_project_ms, t.stage3_bin_sort_ms,
                               t.stage4_composite_ms, bool(t.stage1_skipped),
                               bool(t.stage3_cached), bool(t.used_hardware_timestamps),
                               bool(t.used_64bit_keys), int(t.active_gaussians),
                               int(t.surviving_gaussians), int(t.total_tile_entries))

    @staticmethod
    def _camera(camera: CameraUniforms) -> _abi.CgsCamera:
        cam = _abi.CgsCamera()
        arr = camera.to_array()
        for k in range(16):
            cam.view[k] = float(arr[k])
        (cam.focal_x, cam.focal_y, cam.principal_x, cam.principal_y, cam.viewport_width,
         cam.viewport_height, cam.near_plane) = (float(x) for x in arr[16:23])
        return cam

    def view_images(self, compositors) -> list:
        """Device RGBA8 images [H, W] (int32 words) for execute_views; keep and
        pass the same list every step so a captured graph can be replayed."""
        import torch
        return [torch.empty((int(c.screen_height), int(c.screen_width)), dtype=torch.int32,
                            device=f"cuda:{self.device}") for c in compositors]

    def execute_views(self, scene: GaussianSceneSoa, cages: CageScene | None, cameras,
                      compositors, images, use_graph: bool = True,
                      strain_split_threshold: float = 0.0, mip_filter_3d_var: float = 0.0,
                      min_opacity: float = 1.0 / 255.0, min_radius_px: float = 0.5,
                      radix_bits=0, entry_sort=0, tile_shape=0) -> dict:
        """One step of many views (cgs_execute_views): Stage 1 once, Stages 2-4
        per view into images[v] (from view_images). radix_bits, entry_sort and
        tile_shape are one value for every view or a list with one per view (see
        cindergs_b200.autotune). With use_graph the step is captured as a CUDA
        graph on the first call for a set of views and replayed afterwards.
        Returns the step's stats."""
        self.sync_scene_and_cages(scene, cages)
        n = len(cameras)
        cams = (_abi.CgsCamera * n)(*[self._camera(c) for c in cameras])
        comps = (_abi.CgsCompositor * n)(*[self._compositor(c) for c in compositors])
        outs = (ctypes.c_void_p * n)(*[ctypes.c_void_p(t.data_ptr()) for t in images])
        rbs = list(radix_bits) if hasattr(radix_bits, "__len__") else [radix_bits] * n
        ess = list(entry_sort) if hasattr(entry_sort, "__len__") else [entry_sort] * n
        tss = list(tile_shape) if hasattr(tile_shape, "__len__") else [tile_shape] * n
        params = (_abi.CgsFrameParams * n)(*[
            _abi.CgsFrameParams(float(strain_split_threshold), float(mip_filter_3d_var),
                                float(min_opacity), float(min_radius_px), 0, 1, 0, int(rbs[v]),
                                int(ess[v]), int(tss[v])) for v in range(n)])
        st = _abi.CgsViewsStats()
        self._check(self._lib.cgs_execute_views(self._ctx, n, cams, comps, params,
                                                outs, int(bool(use_graph)), ctypes.byref(st)),
                    "cgs_execute_views")
        return dict(ms=st.ms, total_tile_entries=int(st.total_tile_entries),
                    graph_replayed=bool(st.graph_replayed), graph_captured=bool(st.graph_captured),
                    views_rerendered=int(st.views_rerendered))

    @staticmethod
    def _compositor(c: CompositorUniforms) -> _abi.CgsCompositor:
        comp = _abi.CgsCompositor()
        comp.screen_width = int(c.screen_width)
        comp.screen_height = int(c.screen_height)
        comp.tiles_x = c.tiles_x
        comp.tiles_y = c.tiles_y
        for k in range(4):
            comp.background[k] = float(c.background_color[k])
        for k in range(3):
            comp.camera_position[k] = float(c.camera_position[k])
        comp.sh_degree = min(int(c.sh_degree), 3)
        return comp

    def readback_framebuffer_rgba8(self, width: int, height: int) -> np.ndarray:
        """Tight [H, W, 4] uint8 copy of the last frame (gpu_state.rs:1296-1328)."""
        out = np.empty((height, width, 4), np.uint8)
        self._check(self._lib.cgs_readback_rgba8(self._ctx, _p(out), width, height),
                    "cgs_readback_rgba8")
        return out

    def readback_framebuffer_rgba8_async(self, out: np.ndarray) -> int:
        """Starts copying the last frame's RGBA8 pixels into `out` ([H, W, 4]
        uint8, ideally page-locked) without waiting; returns a ticket for
        readback_wait (cgs_readback_rgba8_async). `out` must stay alive and
        untouched until then."""
        if out.dtype != np.uint8 or out.ndim != 3 or out.shape[2] != 4 or not out.flags.c_contiguous:
            raise ValueError("out must be a contiguous uint8 [H, W, 4] array")
        ticket = ctypes.c_uint64()
        self._check(self._lib.cgs_readback_rgba8_async(self._ctx, _p(out), out.shape[1], out.shape[0],
                                                        ctypes.byref(ticket)),
                    "cgs_readback_rgba8_async")
        return int(ticket.value)

    def readback_wait(self, ticket: int) -> None:
        """Waits until the copy `ticket` has arrived (cgs_readback_wait)."""
        self._check(self._lib.cgs_readback_wait(self._ctx, int(ticket)), "cgs_readback_wait")

    def readback_framebuffer_f32(self, width: int, height: int) -> np.ndarray:
        out = np.empty((height, width, 4), f32)
        self._check(self._lib.cgs_readback_rgba_f32(self._ctx, _p(out), width, height),
                    "cgs_readback_rgba_f32")
        return out

    def invalidate(self) -> None:
        self._check(self._lib.cgs_invalidate(self._ctx), "cgs_invalidate")
        self._scene_hash = None
        self._cage_key = None
        self._device_springs = False

    def invalidate_stage3(self) -> None:
        self._check(self._lib.cgs_invalidate_stage3(self._ctx), "cgs_invalidate_stage3")

    def synchronize(self) -> None:
        self._check(self._lib.cgs_ctx_synchronize(self._ctx), "cgs_ctx_synchronize")

    def device_bytes(self) -> int:
        v = ctypes.c_uint64()
        self._check(self._lib.cgs_ctx_device_bytes(self._ctx, ctypes.byref(v)),
                    "cgs_ctx_device_bytes")
        return int(v.value)

    def set_launch_shape(self, project_threads: int = 0, bin_blocks_per_sm: int = 0,
                         ranges_blocks: int = 0) -> None:
        """Block sizes of the frame's kernels (cgs_ctx_set_launch_shape; 0 =
        the library's default); chosen by cindergs_b200.autotune."""
        shp = _abi.CgsLaunchShape(int(project_threads), int(bin_blocks_per_sm), int(ranges_blocks), 0)
        self._check(self._lib.cgs_ctx_set_launch_shape(self._ctx, ctypes.byref(shp)),
                    "cgs_ctx_set_launch_shape")

    def set_device_budget(self, nbytes: int) -> None:
        """Caps the device memory of the scene residency and frame arena
        (cgs_ctx_set_device_budget; 0 = no cap). Growth past it raises
        CgsError with code CGS_E_OOM."""
        self._check(self._lib.cgs_ctx_set_device_budget(self._ctx, int(nbytes)),
                    "cgs_ctx_set_device_budget")

    def wait_drill(self, polls: int = 1 << 16) -> tuple:
        """Runs the bounded-wait drill (cgs_ctx_wait_drill); returns (status,
        mask of the waits that gave up). CGS_E_TIMEOUT is the expected status."""
        m = ctypes.c_uint32()
        rc = self._lib.cgs_ctx_wait_drill(self._ctx, int(polls), ctypes.byref(m))
        return int(rc), int(m.value)

    def kernel_profile(self) -> dict:
        """Per-kernel device ms, launches and algorithmic HBM bytes accumulated
        over the frames run with profile_stages=True since the last reset."""
        kp = _abi.CgsKernelProfile()
        self._check(self._lib.cgs_kernel_profile_read(self._ctx, ctypes.byref(kp)),
                    "cgs_kernel_profile_read")
        return {name: dict(ms=kp.ms[i], launches=int(kp.launches[i]),
                           alg_bytes=int(kp.alg_bytes[i]), alg_flops=int(kp.alg_flops[i]))
                for i, name in enumerate(_abi.KERNEL_NAMES)}

    def kernel_profile_reset(self) -> None:
        self._check(self._lib.cgs_kernel_profile_reset(self._ctx), "cgs_kernel_profile_reset")

    # -- SH coefficient rotation and the deformed-scene export -------------------
    def sh_rotate(self, sh, rotations, index=None, degree: int = 3):
        """Rotates [n, 48] SH coefficient blocks on the GPU: block i by
        rotations[index[i]] (or rotations[i % k]), rotations [k, 3, 3]
        indexed [k, row, col] (ShRotator::apply, sh_rotation.rs:389-471;
        cgs_sh_rotate). numpy in, numpy out; a CUDA tensor is rotated in
        place and returned."""
        import torch
        dev = f"cuda:{self.device}"
        on_device = isinstance(sh, torch.Tensor) and sh.is_cuda
        t = sh if on_device else torch.as_tensor(np.ascontiguousarray(sh, f32)).to(dev)
        if t.dtype != torch.float32 or not t.is_contiguous() or t.numel() % 48:
            raise ValueError("sh must be contiguous float32 [n, 48]")
        rot = torch.as_tensor(np.asarray(rotations, f32).reshape(-1, 3, 3)) if not (
            isinstance(rotations, torch.Tensor)) else rotations.float().reshape(-1, 3, 3)
        r9 = rot.transpose(1, 2).contiguous().to(dev)  # column-major per rotation
        idx = None
        if index is not None:
            idx = torch.as_tensor(np.asarray(index, np.uint32).astype(np.int32)).to(dev) if not (
                isinstance(index, torch.Tensor)) else index.to(dev, torch.int32).contiguous()
        n = t.numel() // 48
        self._check(self._lib.cgs_sh_rotate(self._ctx, n, ctypes.c_void_p(t.data_ptr()),
                                            int(r9.shape[0]), ctypes.c_void_p(r9.data_ptr()),
                                            ctypes.c_void_p(idx.data_ptr()) if idx is not None else None,
                                            int(degree)), "cgs_sh_rotate")
        return t if on_device else t.cpu().numpy().reshape(np.shape(sh))

    def export_deformed(self, sh_degree: int = 3) -> GaussianSceneSoa:
        """The last frame's deformed scene, SH coefficients rotated by each
        splat's tet or polygon-cage rotation, split children after the rest
        Gaussians (Timeline::deform_scene_at, app/timeline.rs:205-229;
        cgs_export_deformed)."""
        cnt = ctypes.c_uint64()
        self._check(self._lib.cgs_export_deformed(self._ctx, int(sh_degree), 0, None, None, None,
                                                  None, ctypes.byref(cnt)), "cgs_export_deformed")
        n = int(cnt.value)
        pos, cov = np.empty((n, 3), f32), np.empty((n, 6), f32)
        opa, sh = np.empty(n, f32), np.empty((n, 48), f32)
        self._check(self._lib.cgs_export_deformed(self._ctx, int(sh_degree), n, _p(pos), _p(cov),
                                                  _p(opa), _p(sh), ctypes.byref(cnt)),
                    "cgs_export_deformed")
        return GaussianSceneSoa(pos, cov, opa, sh)

    def export_deformed_ply_bytes(self, sh_degree: int = 3) -> bytes:
        """Binary PLY of the deformed scene (export_deformed_ply_bytes_at,
        app/timeline.rs:232-250)."""
        from .ply import write_binary_ply_bytes
        return write_binary_ply_bytes(self.export_deformed(sh_degree))

    def export_deformed_ply(self, path, sh_degree: int = 3) -> None:
        """Writes the deformed scene as binary PLY (export_deformed_ply_at,
        app/timeline.rs:253-272)."""
        from .ply import save_file
        save_file(path, self.export_deformed(sh_degree))

    def read_buffer(self, which: int, dtype) -> np.ndarray:
        """Intermediate buffer of the last frame (CGS_BUF_*), as a flat array."""
        nbytes = ctypes.c_uint64()
        self._check(self._lib.cgs_read_frame_buffer(self._ctx, which, None, 0,
                                                    ctypes.byref(nbytes)), "cgs_read_frame_buffer")
        out = np.empty(int(nbytes.value) // np.dtype(dtype).itemsize, dtype)
        self._check(self._lib.cgs_read_frame_buffer(self._ctx, which, _p(out), out.nbytes,
                                                    ctypes.byref(nbytes)), "cgs_read_frame_buffer")
        return out


# -- device-array primitives (render/kernels/scan.rs, radix_sort.rs) ---------------

def exclusive_scan_u32(state: GpuPipelineState, d_in: int, d_out: int, n: int) -> int:
    """gpu_exclusive_scan_total on raw device pointers; returns the total."""
    total = ctypes.c_uint64()
    _abi.check(state._lib.cgs_scan_u32(state.handle, ctypes.c_void_p(d_in),
                                       ctypes.c_void_p(d_out), n, ctypes.byref(total)),
               "cgs_scan_u32", state.handle)
    return int(total.value)


def radix_sort_u32_pairs(state: GpuPipelineState, d_keys: int, d_vals: int, n: int,
                         key_bits: int = 32, digit_bits: int = 0) -> None:
    """gpu_radix_sort_u32_pairs on raw device pointers (sorted in place)."""
    _abi.check(state._lib.cgs_sort_pairs_u32(state.handle, ctypes.c_void_p(d_keys),
                                             ctypes.c_void_p(d_vals), n, key_bits, digit_bits),
               "cgs_sort_pairs_u32", state.handle)


def radix_sort_u64_pairs(state: GpuPipelineState, d_tiles: int, d_depths: int, d_ids: int,
                         n: int, tile_bits: int, digit_bits: int = 0) -> None:
    """gpu_radix_sort_u64_pairs on raw device pointers (sorted in place)."""
    _abi.check(state._lib.cgs_sort_pairs_u64(state.handle, ctypes.c_void_p(d_tiles),
                                             ctypes.c_void_p(d_depths), ctypes.c_void_p(d_ids),
                                             n, tile_bits, digit_bits),
               "cgs_sort_pairs_u64", state.handle)
