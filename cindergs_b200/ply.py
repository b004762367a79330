"""3DGS binary PLY files: header parsing, vertex decoding and activation into
GaussianSceneSoa, and the canonical 62-float little-endian writer used to
export deformed scenes (scene/ply_loader.rs:1-712, scene/raw_vertex.rs,
GaussianSceneSoa::push_raw / to_raw_vertices, scene/soa.rs:113-329).

A raw vertex is 62 float32 values (raw_vertex.rs:16-42): x y z, nx ny nz,
f_dc_0..2, f_rest_0..44 (channel-major), opacity (logit), scale_0..2
(log), rot_0..3 (w x y z). Files may declare the properties in any order,
with any scalar type for the ignored ones, big- or little-endian, and 0, 9,
24 or 45 f_rest values (SH degree 0..3; compact layouts are scattered into
the 15-per-channel stride). Decoding is vectorised over the vertices.
"""
from __future__ import annotations

import os
import re
from dataclasses import dataclass, field

import numpy as np

from .scene import (MIN_SCALE, GaussianSceneSoa, activate_opacity, activate_rotation,
                    activate_scale, compute_covariance_3d)

f32 = np.float32
RAW_FLOATS = 62
RAW_BYTES = RAW_FLOATS * 4

# PlyScalarType::parse / size (ply_loader.rs:34-78): token -> (kind, bytes)
_SCALAR = {
    "char": ("i1", 1), "int8": ("i1", 1), "uchar": ("u1", 1), "uint8": ("u1", 1),
    "short": ("i2", 2), "int16": ("i2", 2), "ushort": ("u2", 2), "uint16": ("u2", 2),
    "int": ("i4", 4), "int32": ("i4", 4), "uint": ("u4", 4), "uint32": ("u4", 4),
    "float": ("f4", 4), "float32": ("f4", 4), "double": ("f8", 8), "float64": ("f8", 8),
}
_REQUIRED = ("x", "y", "z", "f_dc_0", "f_dc_1", "f_dc_2", "opacity", "scale_0", "scale_1",
             "scale_2", "rot_0", "rot_1", "rot_2", "rot_3")


class PlyError(ValueError):
    """PlyError (ply_loader.rs:156-222); `kind` names the reference variant."""

    def __init__(self, kind: str, message: str, **fields):
        super().__init__(message)
        self.kind = kind
        self.fields = fields


@dataclass
class PlyProperty:
    name: str
    ty: str        # numpy kind: i1 u1 i2 u2 i4 u4 f4 f8
    offset: int    # bytes from the start of the record

    @property
    def is_float(self) -> bool:
        return self.ty in ("f4", "f8")


@dataclass
class PlyHeader:
    format: str               # "binary_little_endian" or "binary_big_endian"
    vertex_count: int
    vertex_stride: int
    properties: list = field(default_factory=list)
    payload_offset: int = 0
    sh_degree: int = 0

    @property
    def payload_len(self) -> int:
        return self.vertex_count * self.vertex_stride

    @property
    def little_endian(self) -> bool:
        return self.format == "binary_little_endian"

    def property(self, name: str):  # defined last: the name shadows the builtin below it
        """The first property of that name (PlyHeader::property)."""
        for p in self.properties:
            if p.name == name:
                return p
        return None


def find_end_header(data: bytes) -> int:
    """Offset of the payload: after the first `end_header` that starts a line
    and ends with LF or CRLF, else after the first `end_header` anywhere
    that does (find_end_header, ply_loader.rs:234-271)."""
    marker = b"end_header"

    def after_newline(pos: int):
        after = pos + len(marker)
        if after < len(data):
            if data.startswith(b"\r\n", after):
                return after + 2
            if data.startswith(b"\n", after):
                return after + 1
        return None

    pos = data.find(marker)
    while pos >= 0:
        if pos == 0 or data[pos - 1] in (0x0A, 0x0D):
            end = after_newline(pos)
            if end is not None:
                return end
        pos = data.find(marker, pos + 1)
    pos = data.find(marker)
    if pos >= 0:
        end = after_newline(pos)
        if end is not None:
            return end
    raise PlyError("MissingEndHeader", "PLY header marker 'end_header' not found")


def _lines(text: str):
    """str::lines: split on LF, drop one trailing CR, no final empty line."""
    parts = text.split("\n")
    if parts and parts[-1] == "":
        parts.pop()
    return [p[:-1] if p.endswith("\r") else p for p in parts]


_USIZE = re.compile(r"\+?[0-9]+")


def parse_element_vertex_count(header: str):
    """Declared `element vertex N` count or None (ply_loader.rs:274-287)."""
    for line in _lines(header):
        parts = line.split()
        if len(parts) >= 3 and parts[0] == "element" and parts[1] == "vertex":
            return int(parts[2]) if _USIZE.fullmatch(parts[2]) else None
    return None


def parse_header(data: bytes) -> PlyHeader:
    """Parses and validates the ASCII header (parse_header, ply_loader.rs:290-462)."""
    if not (data.startswith(b"ply\n") or data.startswith(b"ply\r\n")):
        raise PlyError("InvalidMagic", "Not a valid PLY file (missing leading 'ply' magic header)")
    payload_offset = find_end_header(data)
    try:
        text = data[:payload_offset].decode("utf-8")
    except UnicodeDecodeError:
        raise PlyError("InvalidHeaderUtf8", "PLY header is not valid UTF-8") from None

    fmt = None
    elements: list[tuple[str, int]] = []
    props: list[PlyProperty] = []
    stride = 0
    current = None
    for raw_line in _lines(text):
        line = raw_line.strip()
        if not line or line.startswith("comment") or line.startswith("obj_info"):
            continue
        parts = line.split()
        head = parts[0]
        if head == "format":
            token = parts[1] if len(parts) > 1 else ""
            if token == "ascii":
                raise PlyError("UnsupportedFormat",
                               "unsupported PLY format 'ascii (re-export the scene as "
                               "binary_little_endian or binary_big_endian)'")
            if token not in ("binary_little_endian", "binary_big_endian"):
                raise PlyError("UnsupportedFormat", f"unsupported PLY format '{token}'")
            fmt = token
        elif head == "element":
            name = parts[1] if len(parts) > 1 else ""
            if len(parts) < 3 or not _USIZE.fullmatch(parts[2]):
                raise PlyError("UnsupportedLayout", f"unsupported vertex layout: element '{name}' has no count")
            count = int(parts[2])
            if name == "vertex":
                current = name
            elif current == "vertex":
                current = None  # later properties belong to the new element
            elements.append((name, count))
        elif head == "property":
            if current != "vertex":
                continue
            maybe_list = parts[1] if len(parts) > 1 else ""
            if maybe_list == "list":
                name = parts[4] if len(parts) > 4 else "property"
                raise PlyError("UnsupportedListProperty",
                               f"unsupported list property '{name}': PLY lists are not valid in a "
                               "3DGS vertex record", name=name)
            if maybe_list not in _SCALAR:
                raise PlyError("UnsupportedLayout",
                               f"unsupported vertex layout: unknown property type '{maybe_list}'")
            name = parts[2] if len(parts) > 2 else ""
            if not name:
                raise PlyError("UnsupportedLayout",
                               "unsupported vertex layout: property declaration without a name")
            ty, size = _SCALAR[maybe_list]
            props.append(PlyProperty(name, ty, stride))
            stride += size

    if fmt is None:
        raise PlyError("MissingFormat", "PLY header declares no 'format' line")
    counts = [c for n, c in elements if n == "vertex"]
    if not counts:
        raise PlyError("MissingVertexElement", "PLY header declares no 'element vertex' count")
    vertex_count = counts[0]
    for name, count in elements:
        if name != "vertex" and count > 0:
            raise PlyError("UnsupportedElement",
                           f"unsupported PLY element '{name}' with {count} records",
                           name=name, count=count)
    header = PlyHeader(fmt, vertex_count, stride, props, payload_offset, 0)
    if vertex_count == 0:
        return header
    if not props:
        raise PlyError("UnsupportedLayout", "unsupported vertex layout: vertex element has no properties")
    for name in _REQUIRED:
        p = header.property(name)
        if p is None:
            raise PlyError("MissingProperty", f"vertex property '{name}' is required but missing",
                           name=name)
        if not p.is_float:
            raise PlyError("InvalidPropertyType", f"vertex property '{name}' must be a float",
                           name=name, ty=p.ty)
    rest = 0
    while True:
        p = header.property(f"f_rest_{rest}")
        if p is None:
            break
        if not p.is_float:
            raise PlyError("InvalidPropertyType", f"vertex property '{p.name}' must be a float",
                           name=p.name, ty=p.ty)
        rest += 1
    degrees = {0: 0, 9: 1, 24: 2, 45: 3}
    if rest not in degrees:
        raise PlyError("UnsupportedShLayout",
                       f"spherical harmonics layout with {rest} f_rest properties is unsupported "
                       "(expected 0, 9, 24, or 45)", count=rest)
    header.sh_degree = degrees[rest]
    return header


def _column(rows: np.ndarray, prop: PlyProperty, little: bool) -> np.ndarray:
    """One property of every record as float32 (PlyScalarType::read_f32)."""
    size = np.dtype(prop.ty).itemsize
    raw = np.ascontiguousarray(rows[:, prop.offset:prop.offset + size])
    dt = np.dtype(prop.ty).newbyteorder("<" if little else ">")
    return raw.view(dt).reshape(-1).astype(f32)


def parse_vertex_payload(header: PlyHeader, payload: bytes) -> np.ndarray:
    """Raw vertices [N, 62] float32 from any declared layout
    (parse_vertex_payload, ply_loader.rs:523-583)."""
    needed = header.payload_len
    if len(payload) < needed:
        raise PlyError("TruncatedPayload",
                       f"vertex payload is truncated: need {needed} bytes, file provides {len(payload)}",
                       needed=needed, available=len(payload))
    n = header.vertex_count
    out = np.zeros((n, RAW_FLOATS), f32)
    if n == 0:
        return out
    rows = np.frombuffer(payload, np.uint8, count=needed).reshape(n, header.vertex_stride)
    le = header.little_endian

    def put(col: int, name: str, required: bool = True):
        p = header.property(name)
        if p is None:
            if required:
                raise PlyError("MissingProperty", f"vertex property '{name}' is required but missing",
                               name=name)
            return
        out[:, col] = _column(rows, p, le)

    for k, name in enumerate(("x", "y", "z")):
        put(k, name)
    for k, name in enumerate(("nx", "ny", "nz")):
        put(3 + k, name, required=False)
    for k in range(3):
        put(6 + k, f"f_dc_{k}")
    per_channel = {0: 0, 1: 3, 2: 8, 3: 15}[header.sh_degree]
    for ch in range(3):
        for k in range(per_channel):
            put(9 + 15 * ch + k, f"f_rest_{ch * per_channel + k}")
    put(54, "opacity")
    for k in range(3):
        put(55 + k, f"scale_{k}")
    for k in range(4):
        put(58 + k, f"rot_{k}")
    return out


def scene_from_raw_vertices(raw: np.ndarray) -> GaussianSceneSoa:
    """Activated scene from raw vertices (GaussianSceneSoa::from_raw_vertices_par,
    soa.rs:137-188): covariance from exp scales and the normalised quaternion,
    sigmoid opacity, SH copied."""
    raw = np.asarray(raw, f32).reshape(-1, RAW_FLOATS)
    cov = compute_covariance_3d(activate_scale(raw[:, 55:58]), activate_rotation(raw[:, 58:62]))
    return GaussianSceneSoa(np.ascontiguousarray(raw[:, 0:3]), cov.astype(f32),
                            activate_opacity(raw[:, 54]), np.ascontiguousarray(raw[:, 6:54]))


def load_from_bytes(data: bytes) -> GaussianSceneSoa:
    """PlyLoader::load_from_bytes (ply_loader.rs:610-642)."""
    header = parse_header(data)
    if header.vertex_count == 0:
        e = np.zeros((0,), f32)
        return GaussianSceneSoa(e.reshape(0, 3), e.reshape(0, 6), e, e.reshape(0, 48))
    payload = memoryview(data)[header.payload_offset:]
    if len(payload) < header.payload_len:
        raise PlyError("TruncatedPayload",
                       f"vertex payload is truncated: need {header.payload_len} bytes, file provides "
                       f"{len(payload)}", needed=header.payload_len, available=len(payload))
    return scene_from_raw_vertices(parse_vertex_payload(header, payload))


def load_file(path) -> GaussianSceneSoa:
    """PlyLoader::load_file (ply_loader.rs:595-605)."""
    with open(path, "rb") as fh:
        return load_from_bytes(fh.read())


def _symmetric_eigen_3x3(cov: np.ndarray):
    """symmetric_eigen_3x3 (math/covariance.rs:181-262) over [N,6] packed
    covariances: f64 cyclic Jacobi, 12 sweeps over (0,1), (0,2), (1,2),
    eigenvalues descending (stable, total order), unit eigenvector columns
    made right-handed. Returns (evals [N,3] f32, basis [N,3 cols,3] f32)."""
    c = cov.astype(np.float64)
    n = c.shape[0]
    a = np.empty((n, 3, 3))
    a[:, 0, 0], a[:, 0, 1], a[:, 0, 2] = c[:, 0], c[:, 1], c[:, 2]
    a[:, 1, 0], a[:, 1, 1], a[:, 1, 2] = c[:, 1], c[:, 3], c[:, 4]
    a[:, 2, 0], a[:, 2, 1], a[:, 2, 2] = c[:, 2], c[:, 4], c[:, 5]
    v = np.broadcast_to(np.eye(3), (n, 3, 3)).copy()
    with np.errstate(divide="ignore", invalid="ignore"):
        for _ in range(12):
            for p, q in ((0, 1), (0, 2), (1, 2)):
                apq = a[:, p, q].copy()
                on = ~(np.abs(apq) <= 1e-15)
                if not on.any():
                    continue
                tau = (a[:, q, q] - a[:, p, p]) / (2.0 * apq)
                root = np.sqrt(1.0 + tau * tau)
                t = np.where(tau >= 0.0, 1.0 / (tau + root), -1.0 / (-tau + root))
                cs = 1.0 / np.sqrt(1.0 + t * t)
                sn = t * cs
                app, aqq = a[:, p, p].copy(), a[:, q, q].copy()
                a[:, p, p] = np.where(on, app - t * apq, app)
                a[:, q, q] = np.where(on, aqq + t * apq, aqq)
                a[:, p, q] = np.where(on, 0.0, a[:, p, q])
                a[:, q, p] = np.where(on, 0.0, a[:, q, p])
                r = 3 - p - q
                arp, arq = a[:, r, p].copy(), a[:, r, q].copy()
                nrp = np.where(on, cs * arp - sn * arq, arp)
                nrq = np.where(on, sn * arp + cs * arq, arq)
                a[:, r, p] = nrp
                a[:, p, r] = nrp
                a[:, r, q] = nrq
                a[:, q, r] = nrq
                vp, vq = v[:, :, p].copy(), v[:, :, q].copy()
                v[:, :, p] = np.where(on[:, None], cs[:, None] * vp - sn[:, None] * vq, vp)
                v[:, :, q] = np.where(on[:, None], sn[:, None] * vp + cs[:, None] * vq, vq)
    ev = np.stack([a[:, 0, 0], a[:, 1, 1], a[:, 2, 2]], axis=1)
    vec = np.empty((n, 3, 3))  # [n, eigen index, component]
    for k in range(3):
        x, y, z = v[:, 0, k], v[:, 1, k], v[:, 2, k]
        inv = 1.0 / np.sqrt((x * x + y * y) + z * z)  # DVec3::normalize
        vec[:, k, 0], vec[:, k, 1], vec[:, k, 2] = x * inv, y * inv, z * inv
    # stable descending order under f64 total_cmp
    bits = ev.view(np.int64)
    key = np.where(bits < 0, bits ^ np.int64(0x7FFFFFFFFFFFFFFF), bits)
    order = np.tile(np.arange(3), (n, 1))
    rows = np.arange(n)
    for i in (1, 2):
        for j in range(i, 0, -1):
            swap = key[rows, order[:, j - 1]] < key[rows, order[:, j]]
            lo, hi = order[:, j - 1].copy(), order[:, j].copy()
            order[:, j - 1] = np.where(swap, hi, lo)
            order[:, j] = np.where(swap, lo, hi)
    evals = np.take_along_axis(ev, order, axis=1).astype(f32)
    basis = np.take_along_axis(vec, order[:, :, None], axis=1).astype(f32)  # [n, col, comp]
    # Mat3::determinant = z . (x cross y), float32
    c0, c1, c2 = basis[:, 0], basis[:, 1], basis[:, 2]
    cx = c0[:, 1] * c1[:, 2] - c1[:, 1] * c0[:, 2]
    cy = c0[:, 2] * c1[:, 0] - c1[:, 2] * c0[:, 0]
    cz = c0[:, 0] * c1[:, 1] - c1[:, 0] * c0[:, 1]
    det = (c2[:, 0] * cx + c2[:, 1] * cy) + c2[:, 2] * cz
    basis[det < 0, 2] *= f32(-1.0)
    return evals, basis


def _quat_from_basis(basis: np.ndarray) -> np.ndarray:
    """Unit quaternion (x, y, z, w) of rotation matrices given as columns
    [N, col, comp], by the branch on the largest of 4x^2, 4y^2, 4z^2, 4w^2
    read off the diagonal (Day, "Converting a Rotation Matrix to a
    Quaternion", 2015; glam's Quat::from_mat3), then normalised."""
    m = basis.astype(f32)
    m00, m01, m02 = m[:, 0, 0], m[:, 0, 1], m[:, 0, 2]
    m10, m11, m12 = m[:, 1, 0], m[:, 1, 1], m[:, 1, 2]
    m20, m21, m22 = m[:, 2, 0], m[:, 2, 1], m[:, 2, 2]
    one, half = f32(1.0), f32(0.5)
    q = np.empty((m.shape[0], 4), f32)
    with np.errstate(divide="ignore", invalid="ignore"):
        dif10, omm22 = m11 - m00, one - m22
        sum10, opm22 = m11 + m00, one + m22
        fx = omm22 - dif10
        fy = omm22 + dif10
        fz = opm22 - sum10
        fw = opm22 + sum10
        cand = {
            "x": (fx, lambda i: (fx * i, (m01 + m10) * i, (m02 + m20) * i, (m12 - m21) * i)),
            "y": (fy, lambda i: ((m01 + m10) * i, fy * i, (m12 + m21) * i, (m20 - m02) * i)),
            "z": (fz, lambda i: ((m02 + m20) * i, (m12 + m21) * i, fz * i, (m01 - m10) * i)),
            "w": (fw, lambda i: ((m12 - m21) * i, (m20 - m02) * i, (m01 - m10) * i, fw * i)),
        }
        low = m22 <= 0
        pick = np.where(low, np.where(dif10 <= 0, 0, 1), np.where(sum10 <= 0, 2, 3))
        for k, key in enumerate("xyzw"):
            sel = pick == k
            if not sel.any():
                continue
            f, build = cand[key]
            inv = (half / np.sqrt(f)).astype(f32)
            comps = build(inv)
            for j in range(4):
                q[sel, j] = np.asarray(comps[j], f32)[sel]
    norm = np.sqrt(((q[:, 0] * q[:, 0] + q[:, 1] * q[:, 1]) + q[:, 2] * q[:, 2]) + q[:, 3] * q[:, 3])
    return (q * (one / norm)[:, None]).astype(f32)


def to_raw_vertices(scene: GaussianSceneSoa) -> np.ndarray:
    """Raw vertices [N, 62] for serialising a scene (to_raw_vertices,
    soa.rs:304-328): logit opacity, log scales and quaternion from the
    covariance's eigen-decomposition, SH copied, normals zero."""
    n = scene.count
    out = np.zeros((n, RAW_FLOATS), f32)
    if n == 0:
        return out
    out[:, 0:3] = scene.positions
    # inverse_activate_opacity (covariance.rs:163-166)
    a = np.clip(scene.opacities.astype(f32), f32(1e-6), f32(1.0) - f32(1e-6))
    out[:, 54] = np.log(a / (f32(1.0) - a)).astype(f32)
    # decompose_covariance_3d (covariance.rs:272-284) + inverse_activate_scale
    evals, basis = _symmetric_eigen_3x3(np.asarray(scene.covariances_3d, f32))
    min_var = MIN_SCALE * MIN_SCALE
    scale = np.sqrt(np.maximum(evals, min_var)).astype(f32)
    out[:, 55:58] = np.log(np.maximum(scale, MIN_SCALE)).astype(f32)
    q = _quat_from_basis(basis)
    out[:, 58] = q[:, 3]
    out[:, 59:62] = q[:, 0:3]
    sh = np.asarray(scene.sh_coeffs, f32)
    out[:, 6:54] = sh
    return out


def write_binary_ply_bytes(scene: GaussianSceneSoa) -> bytes:
    """Canonical binary little-endian 3DGS PLY (write_binary_ply_bytes,
    ply_loader.rs:673-702)."""
    raw = to_raw_vertices(scene)
    names = (["x", "y", "z", "nx", "ny", "nz"] + [f"f_dc_{i}" for i in range(3)]
             + [f"f_rest_{i}" for i in range(45)] + ["opacity"]
             + [f"scale_{i}" for i in range(3)] + [f"rot_{i}" for i in range(4)])
    header = f"ply\nformat binary_little_endian 1.0\nelement vertex {raw.shape[0]}\n"
    header += "".join(f"property float {n}\n" for n in names) + "end_header\n"
    return header.encode("ascii") + raw.astype("<f4").tobytes()


def save_file(path, scene: GaussianSceneSoa) -> None:
    """PlyLoader::save_file (ply_loader.rs:704-710)."""
    data = write_binary_ply_bytes(scene)
    with open(os.fspath(path), "wb") as fh:
        fh.write(data)
