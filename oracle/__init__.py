"""CPU oracle for the splat pipeline -- test infrastructure only.

ctypes bindings over ``oracle/_build/libcgs_oracle.so`` (built from
``cgs_oracle.cpp`` by ``oracle/Makefile``). Only the tests, the smoke check and
the CPU-baseline leg of ``bench.py`` use this module; the ``cindergs_b200``
package never imports it.

Two modes are exposed (see cgs_oracle.cpp): ``v2_*`` restates the reference's
GPU kernel semantics (the parity gates) and ``ref_*`` restates its Rayon CPU
backend (pinned by the reference's golden image hash).
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "libcgs_oracle.so")
_lib = None

_f32p = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")
_u32p = np.ctypeslib.ndpointer(dtype=np.uint32, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_u8p = np.ctypeslib.ndpointer(dtype=np.uint8, flags="C_CONTIGUOUS")
_c_u32 = ctypes.c_uint32
_c_u64 = ctypes.c_uint64
_c_f = ctypes.c_float
_vp = ctypes.c_void_p


def build() -> str:
    """Compiles the oracle library (make -C oracle) and returns its path."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        L.orc_set_threads.argtypes = [ctypes.c_int]
        L.orc_get_threads.restype = ctypes.c_int
        L.orc_tet_transforms.argtypes = [_c_u32, _f32p, _u32p, _f32p, _f32p, _f32p, _f32p]
        L.orc_deform_split.restype = _c_u32
        L.orc_deform_split.argtypes = [_c_u32, _c_u32, _f32p, _u32p, _f32p, _f32p, _u32p, _f32p,
                                       _f32p, _f32p, _f32p, _c_f, _c_f, _f32p, _f32p, _f32p, _u32p]
        L.orc_project_v2.restype = _c_u64
        L.orc_project_v2.argtypes = [_c_u32, _c_u32, _f32p, _f32p, _f32p, _f32p, _vp, _vp, _c_u32,
                                     _vp, _f32p, _f32p, _c_f, _c_f, _c_f, _c_u32, _c_u32, _f32p,
                                     _u32p]
        L.orc_count_tiles.restype = _c_u64
        L.orc_count_tiles.argtypes = [_c_u32, _f32p, _u32p, _c_u32, _c_u32, _u32p]
        L.orc_scan.restype = _c_u64
        L.orc_scan.argtypes = [_c_u64, _u32p, _u32p]
        L.orc_packed_key_bits.argtypes = [_c_u32, ctypes.POINTER(_c_u32), ctypes.POINTER(_c_u32)]
        L.orc_emit_keys32.argtypes = [_c_u32, _f32p, _u32p, _u32p, _c_u32, _c_u32, _c_f, _c_u32,
                                      _u32p, _u32p]
        L.orc_emit_keys64.argtypes = [_c_u32, _f32p, _u32p, _u32p, _c_u32, _c_u32, _u32p, _u32p,
                                      _u32p]
        L.orc_sort_pairs32.argtypes = [_c_u64, _u32p, _u32p, _c_u32]
        L.orc_sort_triples64.argtypes = [_c_u64, _u32p, _u32p, _u32p]
        L.orc_tile_ranges.argtypes = [_c_u64, _u32p, _c_u32, _c_u32, _u32p]
        L.orc_composite_v2.argtypes = [_c_u32, _c_u32, _f32p, _u32p, _u32p, _f32p, _vp, _vp]
        L.orc_detmath.restype = _c_f
        L.orc_detmath.argtypes = [ctypes.c_int, _c_f, _c_f]
        L.orc_bind_points.argtypes = [_c_u32, _f32p, _c_u32, _f32p, _f32p, ctypes.c_int, _vp, _vp,
                                      _u32p, _f32p]
        L.orc_fibonacci_cluster.argtypes = [_c_u32, _c_f, _f32p, _f32p, _f32p, _f32p, _f32p]
        L.orc_ref_project_scene.argtypes = [_c_u32, _f32p, _f32p, _f32p, _f32p, _f32p, _i32p,
                                            _f32p]
        L.orc_ref_bin_and_sort.restype = _c_u64
        L.orc_ref_bin_and_sort.argtypes = [_c_u32, _f32p, _f32p, _i32p, _c_u32, _c_u32, _vp, _vp,
                                           _vp, _vp]
        L.orc_ref_rasterize.argtypes = [_c_u32, _c_u32, _f32p, _f32p, _f32p, _f32p, _f32p, _u32p,
                                        _u32p, _f32p, _f32p, _c_u32, _vp, _vp]
        L.orc_mvc_winding.restype = _c_f
        L.orc_mvc_winding.argtypes = [_c_u32, _f32p, _u32p, _f32p]
        L.orc_mvc_weights.argtypes = [_c_u32, _f32p, _c_u32, _f32p, _c_u32, _u32p, _f32p]
        L.orc_mvc_step.restype = _c_f
        L.orc_mvc_step.argtypes = [_c_u32, _f32p]
        L.orc_mvc_bind.argtypes = [_c_u32, _f32p, _c_u32, _f32p, _c_u32, _u32p, _u8p, _f32p]
        L.orc_mvc_deform.restype = _c_u32
        L.orc_mvc_deform.argtypes = [_c_u32, _f32p, _f32p, _f32p, _u8p, _f32p, _c_u32, _f32p, _c_f,
                                     _c_f, _f32p, _f32p, _f32p, _u32p, _f32p]
        L.orc_pixel_hash.restype = _c_u64
        L.orc_pixel_hash.argtypes = [_c_u64, _u8p]
        L.orc_ref_render_scene.restype = _c_u64
        L.orc_ref_render_scene.argtypes = [_c_u32, _f32p, _f32p, _f32p, _f32p, _f32p, _c_u32,
                                           _c_u32, _f32p, _f32p, _c_u32, _vp, _vp]
        L.orc_ellipse_tile.restype = ctypes.c_int
        L.orc_ellipse_tile.argtypes = [_c_f] * 6 + [_c_u32] * 4
        L.orc_conic_extents.restype = ctypes.c_int
        L.orc_conic_extents.argtypes = [_c_f] * 4 + [_f32p, _i32p]
        L.orc_ref_tet_transforms.argtypes = [_c_u32, _f32p, _u32p, _f32p, _f32p, _f32p, _f32p]
        L.orc_ref_sh_rotate.argtypes = [_c_u32, _f32p, _f32p, _c_u32]
        L.orc_sh_rotation_matrix.argtypes = [_f32p, _c_u32, _f32p]
        L.orc_set_tile_shape.argtypes = [_c_u32, _c_u32]
        L.orc_spring_frame_damping.restype = _c_f
        L.orc_spring_frame_damping.argtypes = [_c_f, _c_f]
        L.orc_spring_step.argtypes = [_c_u32, _f32p, _f32p, _f32p, _vp, _c_f, _c_f, _c_f, _c_u32,
                                      _vp, _c_f]
        L.orc_spring_impulse.argtypes = [_c_u32, _f32p, _f32p, _vp, _c_f]
        L.orc_ref_frame.restype = _c_u64
        L.orc_ref_frame.argtypes = [_c_u32, _f32p, _f32p, _f32p, _f32p, _c_u32, _vp, _vp, _vp, _vp,
                                    _vp, _f32p, _c_u32, _c_u32, _f32p, _f32p, _c_u32, _c_f, _c_f,
                                    _u8p, ctypes.POINTER(_c_u32)]
        L.orc_ref_ellipse_tile.restype = ctypes.c_int
        L.orc_ref_ellipse_tile.argtypes = [_c_f] * 6 + [_c_u32] * 4
        L.orc_ref_tile_bounds_xy.restype = ctypes.c_int
        L.orc_ref_tile_bounds_xy.argtypes = [_c_f] * 4 + [_c_u32] * 4 + [_u32p]
        L.orc_pack_depth.restype = _c_u32
        L.orc_pack_depth.argtypes = [_c_f, _c_f, _c_u32]
        L.orc_ref_deform.restype = _c_u32
        L.orc_ref_deform.argtypes = [_c_u32, _f32p, _f32p, _f32p, _f32p, _c_u32, _f32p, _u32p,
                                     _f32p, _u32p, _f32p, _c_u32, _c_f, _c_f, _f32p, _f32p, _f32p,
                                     _f32p]
        _lib = L
    return _lib


def _ptr(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def _u32(a):
    return np.ascontiguousarray(a, dtype=np.uint32)


def set_threads(n: int) -> None:
    lib().orc_set_threads(int(n))


def threads() -> int:
    return int(lib().orc_get_threads())


def detmath(which: str, x: float, y: float = 0.0) -> float:
    code = {"log": 0, "exp": 1, "acos": 2, "cos": 3, "pow": 4}[which]
    return float(lib().orc_detmath(code, x, y))


# ------------------------------------------------------------------ v2 mode

def v2_tet_transforms(verts, elems, inv_dm):
    verts, elems, inv_dm = _f32(verts).ravel(), _u32(elems).ravel(), _f32(inv_dm).ravel()
    T = elems.size // 4
    J = np.zeros(T * 9, np.float32)
    R = np.zeros(T * 9, np.float32)
    S = np.zeros(T, np.float32)
    lib().orc_tet_transforms(T, verts, elems, inv_dm, J, R, S)
    return J, R, S


def v2_deform_split(verts, elems, J, stretch, bind_tet, bind_w, pos, cov, opa, split_thr, mip):
    n = int(np.asarray(opa).size)
    T = int(np.asarray(elems).size // 4)
    out_pos = np.zeros(2 * n * 3, np.float32)
    out_cov = np.zeros(2 * n * 6, np.float32)
    out_opa = np.zeros(2 * n, np.float32)
    meta = np.zeros(2 * n, np.uint32)
    k = lib().orc_deform_split(n, T, _f32(verts).ravel(), _u32(elems).ravel(), _f32(J).ravel(),
                               _f32(stretch).ravel(), _u32(bind_tet).ravel(),
                               _f32(bind_w).ravel(), _f32(pos).ravel(), _f32(cov).ravel(),
                               _f32(opa).ravel(), split_thr, mip, out_pos, out_cov, out_opa, meta)
    m = n + int(k)
    return out_pos[: 3 * m], out_cov[: 6 * m], out_opa[:m], meta[: 2 * int(k)], int(k)


def v2_project(pos, cov, opa, sh, cam24, cam_pos, mip, min_opa, min_rad, sh_degree, n_rest=None,
               bind_tet=None, tet_R=None, num_tets=0, split_meta=None):
    pos, cov, opa, sh = _f32(pos).ravel(), _f32(cov).ravel(), _f32(opa).ravel(), _f32(sh).ravel()
    active = opa.size
    n_rest = active if n_rest is None else int(n_rest)
    has_def = 1 if (bind_tet is not None and tet_R is not None) else 0
    bt = None if bind_tet is None else _u32(bind_tet).ravel()
    tr = None if tet_R is None else _f32(tet_R).ravel()
    sm = None if split_meta is None else _u32(split_meta).ravel()
    attrs = np.zeros(active * 10, np.float32)
    ext = np.zeros(active, np.uint32)
    surv = lib().orc_project_v2(active, n_rest, pos, cov, opa, sh, _ptr(bt), _ptr(tr),
                                int(num_tets), _ptr(sm), _f32(cam24).ravel(),
                                _f32(cam_pos).ravel(), mip, min_opa, min_rad, int(sh_degree),
                                has_def, attrs, ext)
    return attrs, ext, int(surv)


def v2_count_tiles(attrs, ext, W, H):
    ext = _u32(ext).ravel()
    counts = np.zeros(ext.size, np.uint32)
    total = lib().orc_count_tiles(ext.size, _f32(attrs).ravel(), ext, W, H, counts)
    return counts, int(total)


def scan(x):
    x = _u32(x).ravel()
    out = np.zeros_like(x)
    total = lib().orc_scan(x.size, x, out)
    return out, int(total)


def packed_key_bits(total_tiles):
    tb, db = _c_u32(), _c_u32()
    lib().orc_packed_key_bits(int(total_tiles), ctypes.byref(tb), ctypes.byref(db))
    return int(tb.value), int(db.value)


def v2_emit_keys32(attrs, ext, offsets, total, W, H, near_plane, depth_bits):
    keys = np.zeros(total, np.uint32)
    ids = np.zeros(total, np.uint32)
    ext = _u32(ext).ravel()
    lib().orc_emit_keys32(ext.size, _f32(attrs).ravel(), ext, _u32(offsets).ravel(), W, H,
                          near_plane, depth_bits, keys, ids)
    return keys, ids


def v2_emit_keys64(attrs, ext, offsets, total, W, H):
    t = np.zeros(total, np.uint32)
    d = np.zeros(total, np.uint32)
    ids = np.zeros(total, np.uint32)
    ext = _u32(ext).ravel()
    lib().orc_emit_keys64(ext.size, _f32(attrs).ravel(), ext, _u32(offsets).ravel(), W, H, t, d,
                          ids)
    return t, d, ids


def sort_pairs32(keys, vals, key_bits=32):
    k, v = _u32(keys).copy(), _u32(vals).copy()
    lib().orc_sort_pairs32(k.size, k, v, int(key_bits))
    return k, v


def sort_triples64(tiles, depths, ids):
    t, d, i = _u32(tiles).copy(), _u32(depths).copy(), _u32(ids).copy()
    lib().orc_sort_triples64(t.size, t, d, i)
    return t, d, i


def tile_ranges(sorted_words, shift, total_tiles):
    s = _u32(sorted_words).ravel()
    ranges = np.zeros(2 * total_tiles, np.uint32)
    lib().orc_tile_ranges(s.size, s, int(shift), int(total_tiles), ranges)
    return ranges


def v2_composite(W, H, attrs, sorted_ids, ranges, bg):
    rgba8 = np.zeros(W * H * 4, np.uint8)
    f = np.zeros(W * H * 4, np.float32)
    lib().orc_composite_v2(W, H, _f32(attrs).ravel(), _u32(sorted_ids).ravel(),
                           _u32(ranges).ravel(), _f32(bg).ravel(), _ptr(rgba8), _ptr(f))
    return rgba8.reshape(H, W, 4), f.reshape(H, W, 4)


def v2_frame(scene, cam24, comp, *, mip=0.0, min_opa=1.0 / 255.0, min_rad=0.5, split_thr=0.0,
             cage=None, tile=(16, 16)):
    """Whole v2 frame on the CPU. ``scene`` = dict(pos, cov, opa, sh);
    ``comp`` = dict(width, height, bg, cam_pos, sh_degree); ``cage`` =
    dict(verts, elems, inv_dm, bind_tet, bind_w) or None; ``tile`` = the
    screen tile (width, height) of Stages 3 and 4. Returns a dict with every
    intermediate (the same buffers the GPU frame exposes)."""
    lib().orc_set_tile_shape(int(tile[0]), int(tile[1]))
    try:
        return _v2_frame(scene, cam24, comp, mip, min_opa, min_rad, split_thr, cage, tile)
    finally:
        lib().orc_set_tile_shape(16, 16)


def _v2_frame(scene, cam24, comp, mip, min_opa, min_rad, split_thr, cage, tile):
    W, H = int(comp["width"]), int(comp["height"])
    out = {}
    n = int(np.asarray(scene["opa"]).size)
    if cage is not None:
        J, R, S = v2_tet_transforms(cage["verts"], cage["elems"], cage["inv_dm"])
        pos, cov, opa, meta, k = v2_deform_split(cage["verts"], cage["elems"], J, S,
                                                 cage["bind_tet"], cage["bind_w"], scene["pos"],
                                                 scene["cov"], scene["opa"], split_thr, mip)
        out.update(J=J, R=R, stretch=S, def_pos=pos, def_cov=cov, def_opa=opa, meta=meta,
                   splits=k)
        attrs, ext, surv = v2_project(pos, cov, opa, scene["sh"], cam24, comp["cam_pos"], 0.0,
                                      min_opa, min_rad, comp["sh_degree"], n_rest=n,
                                      bind_tet=cage["bind_tet"], tet_R=R,
                                      num_tets=np.asarray(cage["elems"]).size // 4,
                                      split_meta=meta)
    else:
        attrs, ext, surv = v2_project(scene["pos"], scene["cov"], scene["opa"], scene["sh"],
                                      cam24, comp["cam_pos"], mip, min_opa, min_rad,
                                      comp["sh_degree"])
    counts, total = v2_count_tiles(attrs, ext, W, H)
    offsets, total2 = scan(counts)
    assert total == total2
    tw, th = int(tile[0]), int(tile[1])
    tiles = ((W + tw - 1) // tw) * ((H + th - 1) // th)
    out.update(attrs=attrs, ext=ext, surviving=surv, counts=counts, offsets=offsets,
               entries=total, total_tiles=tiles)
    if tiles <= 65535:
        tb, db = packed_key_bits(tiles)
        keys, ids = v2_emit_keys32(attrs, ext, offsets, total, W, H, float(cam24[22]), db)
        sk, si = sort_pairs32(keys, ids, min(tb + db, 32))
        ranges = tile_ranges(sk, db, tiles)
        out.update(keys=keys, sorted_keys=sk, sorted_ids=si, tile_bits=tb, depth_bits=db)
    else:
        t, d, ids = v2_emit_keys64(attrs, ext, offsets, total, W, H)
        st, sd, si = sort_triples64(t, d, ids)
        ranges = tile_ranges(st, 0, tiles)
        out.update(sorted_tiles=st, sorted_depths=sd, sorted_ids=si)
    rgba8, f = v2_composite(W, H, attrs, out["sorted_ids"], ranges, comp["bg"])
    out.update(ranges=ranges, rgba8=rgba8, rgba_f32=f)
    return out


def bind_points(points, rest_verts, elems, inv_dm, bounds=None):
    """TetMesh::bind_point for every point; returns (tet [N], weights [N,4])."""
    pts = _f32(points).reshape(-1, 3)
    elems = _u32(elems).reshape(-1, 4)
    rv = _f32(rest_verts).reshape(-1, 3)
    x0 = np.ascontiguousarray(rv[elems[:, 0].astype(np.int64)], np.float32)
    n = pts.shape[0]
    tet = np.zeros(n, np.uint32)
    w = np.zeros((n, 4), np.float32)
    if bounds is not None:
        bmin, bmax = _f32(bounds[0]), _f32(bounds[1])
        lib().orc_bind_points(n, pts.ravel(), elems.shape[0], x0.ravel(), _f32(inv_dm).ravel(), 1,
                              _ptr(bmin), _ptr(bmax), tet, w)
    else:
        lib().orc_bind_points(n, pts.ravel(), elems.shape[0], x0.ravel(), _f32(inv_dm).ravel(), 0,
                              None, None, tet, w)
    return tet, w


# ------------------------------------------------------------------ ref mode

def fibonacci_cluster(count, radius, center):
    pos = np.zeros(count * 3, np.float32)
    cov = np.zeros(count * 6, np.float32)
    opa = np.zeros(count, np.float32)
    sh = np.zeros(count * 48, np.float32)
    lib().orc_fibonacci_cluster(count, radius, _f32(center), pos, cov, opa, sh)
    return dict(pos=pos, cov=cov, opa=opa, sh=sh)


def ref_render_scene(scene, cam24, W, H, bg, cam_pos, sh_degree):
    n = int(np.asarray(scene["opa"]).size)
    rgba8 = np.zeros(W * H * 4, np.uint8)
    f = np.zeros(W * H * 4, np.float32)
    entries = lib().orc_ref_render_scene(n, _f32(scene["pos"]).ravel(), _f32(scene["cov"]).ravel(),
                                         _f32(scene["opa"]).ravel(), _f32(scene["sh"]).ravel(),
                                         _f32(cam24).ravel(), W, H, _f32(bg), _f32(cam_pos),
                                         int(sh_degree), _ptr(rgba8), _ptr(f))
    return rgba8.reshape(H, W, 4), f.reshape(H, W, 4), int(entries)


def pixel_hash(rgba8) -> int:
    b = np.ascontiguousarray(rgba8, dtype=np.uint8).ravel()
    return int(lib().orc_pixel_hash(b.size, b))


def ref_ellipse_tile(mu_x, mu_y, conic, alpha, tx, ty, W, H) -> bool:
    """ellipse_intersects_tile (render/tiles/mod.rs:139-184), glibc logf cutoff."""
    return bool(lib().orc_ref_ellipse_tile(mu_x, mu_y, conic[0], conic[1], conic[2], alpha, tx,
                                           ty, W, H))


def ref_tile_bounds_xy(cx, cy, ex, ey, tiles_x, tiles_y, W, H):
    """compute_gaussian_tile_bounds_xy (render/tiles/mod.rs:97-130): None or
    (tx0, tx1, ty0, ty1)."""
    box = np.zeros(4, np.uint32)
    ok = lib().orc_ref_tile_bounds_xy(cx, cy, ex, ey, tiles_x, tiles_y, W, H, box)
    return tuple(int(v) for v in box) if ok else None


def pack_depth(tz, near_plane, depth_bits) -> int:
    """pack_relative_depth_bits (render/kernels/binning.rs:25-31)."""
    return int(lib().orc_pack_depth(float(tz), float(near_plane), int(depth_bits)))


def ref_deform(scene, cage, sh_degree=3, split_thr=0.0, mip=0.0):
    """deform_cage_scene_cpu restated (ref mode, cpu_reference.rs:157-404):
    dict(pos [m,3], cov [m,6], opa [m], sh [m,48]) with split children
    appended in parent order. ``cage`` = dict(verts, elems, inv_dm, bind_tet,
    bind_w) with global tet indices."""
    n = int(np.asarray(scene["opa"]).size)
    elems = _u32(cage["elems"]).ravel()
    op = np.zeros(2 * n * 3, np.float32)
    oc = np.zeros(2 * n * 6, np.float32)
    oa = np.zeros(2 * n, np.float32)
    osh = np.zeros(2 * n * 48, np.float32)
    m = lib().orc_ref_deform(n, _f32(scene["pos"]).ravel(), _f32(scene["cov"]).ravel(),
                             _f32(scene["opa"]).ravel(), _f32(scene["sh"]).ravel(),
                             elems.size // 4, _f32(cage["verts"]).ravel(), elems,
                             _f32(cage["inv_dm"]).ravel(), _u32(cage["bind_tet"]).ravel(),
                             _f32(cage["bind_w"]).ravel(), int(sh_degree), float(split_thr),
                             float(mip), op, oc, oa, osh)
    m = int(m)
    return dict(pos=op[:3 * m].reshape(m, 3), cov=oc[:6 * m].reshape(m, 6), opa=oa[:m],
                sh=osh[:48 * m].reshape(m, 48))


def ref_tet_transforms(verts, elems, inv_dm):
    """Reference CPU tet transforms (glam polar, f64 Jacobi stretch)."""
    elems = _u32(elems).ravel()
    T = elems.size // 4
    J = np.zeros(T * 9, np.float32)
    R = np.zeros(T * 9, np.float32)
    S = np.zeros(T, np.float32)
    lib().orc_ref_tet_transforms(T, _f32(verts).ravel(), elems, _f32(inv_dm).ravel(), J, R, S)
    return J, R, S


def ref_sh_rotate(sh, R9, degree):
    """ShRotator::new(R, degree).apply on every 48-coefficient block of `sh`
    (render/rasterizer/sh_rotation.rs:389-440); R9 column-major."""
    out = _f32(sh).copy().ravel()
    lib().orc_ref_sh_rotate(out.size // 48, out, _f32(R9).ravel(), int(degree))
    return out


def sh_rotation_matrix(R9, band):
    """sh_rotation_matrix(R, band) (sh_rotation.rs:367-385): row-major
    (2 band + 1)^2 float32 matrix; R9 column-major."""
    n = 2 * int(band) + 1
    out = np.zeros(n * n, np.float32)
    lib().orc_sh_rotation_matrix(_f32(R9).ravel(), int(band), out)
    return out.reshape(n, n)


def spring_frame_damping(damping, dt) -> float:
    """CageSpringSimulator::frame_damping (deformation/dynamics.rs:137-148)."""
    return float(lib().orc_spring_frame_damping(float(damping), float(dt)))


def spring_step(rest, cur, vel, pinned, stiffness, damping, mass, planes, dt):
    """One CageSpringSimulator::step (dynamics.rs:249-277) of one cage; returns
    new (current, velocity) [V,3]. planes [P,8]: nx ny nz offset restitution
    friction pad pad."""
    rest = _f32(rest).reshape(-1, 3)
    c = _f32(cur).reshape(-1, 3).copy()
    v = _f32(vel).reshape(-1, 3).copy()
    pin = np.ascontiguousarray(pinned, np.uint8) if pinned is not None else None
    pl = np.ascontiguousarray(planes, np.float32).reshape(-1, 8) if planes is not None and len(
        planes) else None
    lib().orc_spring_step(rest.shape[0], rest.ravel(), c.ravel(), v.ravel(),
                          _ptr(pin) if pin is not None else None, float(stiffness), float(damping),
                          float(mass), 0 if pl is None else pl.shape[0],
                          _ptr(pl) if pl is not None else None, float(dt))
    return c, v


def spring_impulse(rest, vel, pinned, magnitude):
    """CageSpringSimulator::trigger_jiggle_impulse (dynamics.rs:280-305)."""
    rest = _f32(rest).reshape(-1, 3)
    v = _f32(vel).reshape(-1, 3).copy()
    pin = np.ascontiguousarray(pinned, np.uint8) if pinned is not None else None
    lib().orc_spring_impulse(rest.shape[0], rest.ravel(), v.ravel(),
                             _ptr(pin) if pin is not None else None, float(magnitude))
    return v


def ref_frame(scene, cam24, W, H, bg, cam_pos, sh_degree, cage=None, split_thr=0.0, mip=0.0):
    """execute_cpu_reference_with_options restated (ref CPU mode). Returns
    (rgba8 [H,W,4], tile entries, split children)."""
    n = int(np.asarray(scene["opa"]).size)
    rgba8 = np.zeros(W * H * 4, np.uint8)
    splits = _c_u32()
    if cage is not None:
        verts, elems = _f32(cage["verts"]).ravel(), _u32(cage["elems"]).ravel()
        inv, bt, bw = _f32(cage["inv_dm"]).ravel(), _u32(cage["bind_tet"]).ravel(), \
            _f32(cage["bind_w"]).ravel()
        T = elems.size // 4
        args = (T, _ptr(verts), _ptr(elems), _ptr(inv), _ptr(bt), _ptr(bw))
    else:
        args = (0, None, None, None, None, None)
    e = lib().orc_ref_frame(n, _f32(scene["pos"]).ravel(), _f32(scene["cov"]).ravel(),
                            _f32(scene["opa"]).ravel(), _f32(scene["sh"]).ravel(), *args,
                            _f32(cam24).ravel(), W, H, _f32(bg), _f32(cam_pos), int(sh_degree),
                            split_thr, mip, rgba8, ctypes.byref(splits))
    return rgba8.reshape(H, W, 4), int(e), int(splits.value)


def ellipse_tile(mu_x, mu_y, conic, alpha, tx, ty, W, H) -> bool:
    return bool(lib().orc_ellipse_tile(mu_x, mu_y, conic[0], conic[1], conic[2], alpha, tx, ty,
                                       W, H))


def conic_extents(sxx, sxy, syy, alpha):
    """compute_conic_and_extents; None when culled, else (conic[3], ext[2])."""
    c = np.zeros(3, np.float32)
    e = np.zeros(2, np.int32)
    ok = lib().orc_conic_extents(sxx, sxy, syy, alpha, c, e)
    return (c, e) if ok else None


def ref_project(pos, cov, cam24):
    """project_scene_cpu: (xy [N,2], depth [N], radius [N], conic [N,3])."""
    pos, cov = _f32(pos).reshape(-1, 3), _f32(cov).reshape(-1, 6)
    n = pos.shape[0]
    xy = np.zeros(2 * n, np.float32)
    d = np.zeros(n, np.float32)
    r = np.zeros(n, np.int32)
    c = np.zeros(3 * n, np.float32)
    lib().orc_ref_project_scene(n, pos.ravel(), cov.ravel(), _f32(cam24), xy, d, r, c)
    return xy.reshape(n, 2), d, r, c.reshape(n, 3)


def ref_bin_and_sort(xy, depths, radii, W, H):
    """bin_and_sort_gaussians_cpu: (tiles, depth_bits, ids, ranges [T,2])."""
    xy = _f32(xy).ravel()
    depths = _f32(depths).ravel()
    radii = np.ascontiguousarray(radii, np.int32).ravel()
    n = radii.size
    total = lib().orc_ref_bin_and_sort(n, xy, depths, radii, W, H, None, None, None, None)
    tiles = ((W + 15) // 16) * ((H + 15) // 16)
    t = np.zeros(total, np.uint32)
    d = np.zeros(total, np.uint32)
    i = np.zeros(total, np.uint32)
    rg = np.zeros(2 * tiles, np.uint32)
    lib().orc_ref_bin_and_sort(n, xy, depths, radii, W, H, _ptr(t), _ptr(d), _ptr(i), _ptr(rg))
    return t, d, i, rg.reshape(tiles, 2)


def ref_rasterize(W, H, xy, conics, opa, sh, pos, sorted_ids, ranges, bg, cam_pos, sh_degree):
    """rasterize_scene_cpu: (rgba8 [H,W,4], rgba_f32 [H,W,4])."""
    rgba8 = np.zeros(W * H * 4, np.uint8)
    f = np.zeros(W * H * 4, np.float32)
    lib().orc_ref_rasterize(W, H, _f32(xy).ravel(), _f32(conics).ravel(), _f32(opa).ravel(),
                            _f32(sh).ravel(), _f32(pos).ravel(), _u32(sorted_ids).ravel(),
                            _u32(ranges).ravel(), _f32(bg), _f32(cam_pos), int(sh_degree),
                            _ptr(rgba8), _ptr(f))
    return rgba8.reshape(H, W, 4), f.reshape(H, W, 4)


# ---------------------------------------------------------------- MVC (ref)
def mvc_winding(verts, tris, point) -> float:
    """PolyCageMesh::winding_number (deformation/mvc.rs:339-357)."""
    return float(lib().orc_mvc_winding(int(np.asarray(tris).reshape(-1, 3).shape[0]),
                                       _f32(verts), _u32(tris), _f32(point)))


def mvc_weights(points, verts, tris):
    """compute_mvc_weights (deformation/mvc.rs:366-471) for each point: [n, V]."""
    pts = _f32(points).reshape(-1, 3)
    v = _f32(verts).reshape(-1, 3)
    t = _u32(tris).reshape(-1, 3)
    out = np.zeros((pts.shape[0], v.shape[0]), np.float32)
    lib().orc_mvc_weights(pts.shape[0], pts, v.shape[0], v, t.shape[0], t, out)
    return out


def mvc_step(verts) -> float:
    """jacobian_step_size (deformation/mvc.rs:484-494)."""
    v = _f32(verts).reshape(-1, 3)
    return float(lib().orc_mvc_step(v.shape[0], v))


def mvc_bind(points, verts, tris):
    """bind_gaussians (deformation/mvc.rs:498-541): (inside [n] bool, wg [n, V, 4]) with
    wg[..., 0] the weights and wg[..., 1:] the central-difference gradients."""
    pts = _f32(points).reshape(-1, 3)
    v = _f32(verts).reshape(-1, 3)
    t = _u32(tris).reshape(-1, 3)
    inside = np.zeros(pts.shape[0], np.uint8)
    wg = np.zeros((pts.shape[0], v.shape[0], 4), np.float32)
    lib().orc_mvc_bind(pts.shape[0], pts, v.shape[0], v, t.shape[0], t, inside, wg)
    return inside.astype(bool), wg


def mvc_deform(pos, cov, opa, inside, wg, deformed_verts, split_thr=0.0, mip=0.0):
    """deform_scene_cpu (deformation/mvc.rs:564-749) without SH coefficient
    rotation; returns dict(pos, cov, opa, parent, R) with children appended."""
    pos = _f32(pos).reshape(-1, 3)
    n = pos.shape[0]
    V = np.asarray(deformed_verts).reshape(-1, 3).shape[0]
    op = np.zeros((2 * n, 3), np.float32)
    oc = np.zeros((2 * n, 6), np.float32)
    oa = np.zeros(2 * n, np.float32)
    par = np.zeros(max(n, 1), np.uint32)
    R = np.zeros((n, 9), np.float32)
    total = lib().orc_mvc_deform(n, pos, _f32(cov).reshape(-1, 6), _f32(opa),
                                 np.ascontiguousarray(inside, np.uint8),
                                 _f32(wg).reshape(-1), V, _f32(deformed_verts).reshape(-1, 3),
                                 float(split_thr), float(mip), op, oc, oa, par, R)
    return dict(pos=op[:total], cov=oc[:total], opa=oa[:total], parent=par[:total - n], R=R)
