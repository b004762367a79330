"""3DGS PLY reader/writer against the cases of the reference's loader tests
(scene/ply_loader.rs:714-1080): LF/CRLF/comment header ends, vertex-count
parsing, the canonical 62-float round trip, ASCII and list rejection,
missing properties, reordered and extra properties, big-endian payloads, SH
degree detection and the compact degree-1 scatter, unsupported SH layouts,
truncated payloads, extra elements, and the writer's round trip."""
import struct

import numpy as np
import pytest

from cindergs_b200 import ply
from cindergs_b200.scene import (GaussianSceneSoa, activate_opacity, random_scene)

f32 = np.float32
STANDARD = ["x", "y", "z", "f_dc_0", "f_dc_1", "f_dc_2", "opacity", "scale_0", "scale_1",
            "scale_2", "rot_0", "rot_1", "rot_2", "rot_3"]


def header(fmt, count, props):
    text = f"ply\nformat {fmt}\nelement vertex {count}\n"
    text += "".join(f"property {ty} {name}\n" for ty, name in props)
    return text + "end_header\n"


def floats(props):
    return [("float", n) for n in props]


def test_end_of_header_offsets():
    lf = b"ply\nformat binary_little_endian 1.0\nelement vertex 2\nend_header\n"
    assert ply.find_end_header(lf) == len(lf)
    crlf = b"ply\r\nformat binary_little_endian 1.0\r\nelement vertex 2\r\nend_header\r\n"
    assert ply.find_end_header(crlf) == len(crlf)
    comments = (b"ply\ncomment author: test\ncomment end_header in comment\n"
                b"element vertex 10\nend_header\n")
    assert ply.find_end_header(comments) == len(comments)
    with pytest.raises(ply.PlyError) as e:
        ply.find_end_header(b"ply\nformat binary_little_endian 1.0\nelement vertex 2\n")
    assert e.value.kind == "MissingEndHeader"


def test_vertex_count_parsing():
    assert ply.parse_element_vertex_count(
        "ply\nformat binary_little_endian 1.0\nelement vertex 14205\nproperty float x\nend_header\n"
    ) == 14205
    assert ply.parse_element_vertex_count("ply\nformat binary_little_endian 1.0\nend_header\n") is None


def test_canonical_round_trip_through_a_file(tmp_path):
    raw = np.zeros(62, f32)
    raw[0:3] = [10.0, -5.0, 3.5]
    raw[6:9] = [0.5, 0.6, 0.7]
    raw[54] = 2.0
    raw[55:58] = [-0.5, 0.0, 1.2]
    raw[58:62] = [1.0, 0.0, 0.0, 0.0]
    names = (["x", "y", "z", "nx", "ny", "nz"] + [f"f_dc_{i}" for i in range(3)]
             + [f"f_rest_{i}" for i in range(45)] + ["opacity"] + [f"scale_{i}" for i in range(3)]
             + [f"rot_{i}" for i in range(4)])
    data = header("binary_little_endian 1.0", 1, floats(names)).encode() + raw.tobytes()
    path = tmp_path / "one.ply"
    path.write_bytes(data)
    scene = ply.load_file(path)
    assert scene.count == 1
    np.testing.assert_array_equal(scene.positions[0], [10.0, -5.0, 3.5])
    np.testing.assert_array_equal(scene.sh_coeffs[0, :3], np.array([0.5, 0.6, 0.7], f32))
    h = ply.parse_header(data)
    np.testing.assert_array_equal(ply.parse_vertex_payload(h, data[h.payload_offset:])[0], raw)
    # identity rotation: the covariance is diag(exp(2 s))
    np.testing.assert_allclose(scene.covariances_3d[0], [np.exp(-1.0), 0, 0, 1.0, 0, np.exp(2.4)],
                               rtol=1e-6)


@pytest.mark.parametrize("text,kind", [
    (b"ply\nformat ascii 1.0\nelement vertex 1\nproperty float x\nend_header\n", "UnsupportedFormat"),
    (b"ply\nformat binary_little_endian 1.0\nelement vertex 1\nproperty float x\n"
     b"property list uchar int vertex_indices\nend_header\n", "UnsupportedListProperty"),
    (b"plx\nformat binary_little_endian 1.0\nend_header\n", "InvalidMagic"),
    (b"ply\nelement vertex 1\nproperty float x\nend_header\n", "MissingFormat"),
    (b"ply\nformat binary_little_endian 1.0\nelement face 0\nend_header\n", "MissingVertexElement"),
    (b"ply\nformat binary_little_endian 1.0\nelement vertex 1\nproperty float x\n"
     b"element face 2\nend_header\n", "UnsupportedElement"),
    (b"ply\nformat binary_little_endian 1.0\nelement vertex 1\nproperty half x\nend_header\n",
     "UnsupportedLayout"),
])
def test_rejections(text, kind):
    with pytest.raises(ply.PlyError) as e:
        ply.parse_header(text)
    assert e.value.kind == kind
    if kind == "UnsupportedFormat":
        assert "ascii" in str(e.value)


def test_missing_required_property():
    with pytest.raises(ply.PlyError) as e:
        ply.parse_header(header("binary_little_endian 1.0", 1, floats(["x", "y", "z"])).encode())
    assert e.value.kind == "MissingProperty" and e.value.fields["name"] == "f_dc_0"


def test_integer_required_property_is_rejected():
    props = floats(STANDARD)
    props[6] = ("uchar", "opacity")
    with pytest.raises(ply.PlyError) as e:
        ply.parse_header(header("binary_little_endian 1.0", 1, props).encode())
    assert e.value.kind == "InvalidPropertyType" and e.value.fields["name"] == "opacity"


def test_reordered_and_extra_properties():
    props = floats(["scale_0", "scale_1", "scale_2", "rot_0", "rot_1", "rot_2", "rot_3", "opacity",
                    "f_dc_0", "f_dc_1", "f_dc_2"]) + [("int", "cluster_id")] + floats(["x", "y", "z"])
    body = struct.pack("<11f", 0, 0, 0, 1, 0, 0, 0, 3.0, 0.1, 0.2, 0.3) + struct.pack("<i", 7)
    body += struct.pack("<3f", 1.5, -2.0, 0.25)
    scene = ply.load_from_bytes(header("binary_little_endian 1.0", 1, props).encode() + body)
    assert scene.count == 1
    np.testing.assert_array_equal(scene.positions[0], [1.5, -2.0, 0.25])
    assert abs(scene.opacities[0] - activate_opacity(np.array([3.0], f32))[0]) < 1e-6
    assert abs(scene.sh_coeffs[0, 0] - 0.1) < 1e-6


def test_big_endian_and_double_payloads():
    vals = [1.0, 2.0, 3.0, 0.1, 0.2, 0.3, 0.5, -1.0, 0.0, 1.0, 1.0, 0.0, 0.0, 0.0]
    data = header("binary_big_endian 1.0", 1, floats(STANDARD)).encode() + struct.pack(">14f", *vals)
    scene = ply.load_from_bytes(data)
    np.testing.assert_array_equal(scene.positions[0], [1.0, 2.0, 3.0])
    np.testing.assert_array_equal(scene.sh_coeffs[0, :3], np.array([0.1, 0.2, 0.3], f32))
    dbl = [("double", n) for n in STANDARD]
    data = header("binary_little_endian 1.0", 1, dbl).encode() + struct.pack("<14d", *vals)
    scene2 = ply.load_from_bytes(data)
    np.testing.assert_array_equal(scene2.positions, scene.positions)
    np.testing.assert_array_equal(scene2.covariances_3d, scene.covariances_3d)


@pytest.mark.parametrize("rest,degree", [(0, 0), (9, 1), (24, 2), (45, 3)])
def test_sh_degree_detection(rest, degree):
    props = floats(STANDARD + [f"f_rest_{i}" for i in range(rest)])
    assert ply.parse_header(header("binary_little_endian 1.0", 1, props).encode()).sh_degree == degree


def test_compact_degree_one_is_scattered_per_channel():
    props = floats(STANDARD + [f"f_rest_{i}" for i in range(9)])
    vals = [1.0, 2.0, 3.0, 0.1, 0.2, 0.3, 0.5, -1.0, 0.0, 1.0, 1.0, 0.0, 0.0, 0.0]
    data = header("binary_little_endian 1.0", 1, props).encode()
    data += struct.pack("<14f", *vals) + struct.pack("<9f", *range(1, 10))
    sh = ply.load_from_bytes(data).sh_coeffs[0]
    np.testing.assert_array_equal(sh[:3], np.array([0.1, 0.2, 0.3], f32))
    np.testing.assert_array_equal(sh[3:6], [1, 2, 3])
    np.testing.assert_array_equal(sh[18:21], [4, 5, 6])
    np.testing.assert_array_equal(sh[33:36], [7, 8, 9])
    assert not sh[6:18].any() and not sh[21:33].any() and not sh[36:].any()


def test_unsupported_sh_layout():
    props = floats(STANDARD + ["f_rest_0", "f_rest_1"])
    with pytest.raises(ply.PlyError) as e:
        ply.parse_header(header("binary_little_endian 1.0", 1, props).encode())
    assert e.value.kind == "UnsupportedShLayout" and e.value.fields["count"] == 2


def test_truncated_payload():
    data = header("binary_little_endian 1.0", 2, floats(STANDARD)).encode() + bytes(8)
    with pytest.raises(ply.PlyError) as e:
        ply.load_from_bytes(data)
    assert e.value.kind == "TruncatedPayload"
    assert e.value.fields == {"needed": 2 * 14 * 4, "available": 8}


def test_empty_vertex_element():
    scene = ply.load_from_bytes(b"ply\nformat binary_little_endian 1.0\nelement vertex 0\nend_header\n")
    assert scene.count == 0


def test_writer_round_trip_of_the_reference_pair():
    sh0 = np.zeros(48, f32)
    sh0[[0, 1, 2, 3, 18, 33]] = [0.5, -0.25, 0.75, 0.1, -0.15, 0.2]
    scene = GaussianSceneSoa(np.array([[0.25, -0.5, 1.25], [-1.0, 2.0, 0.5]], f32),
                             np.array([[0.04, 0, 0, 0.09, 0, 0.02],
                                       [0.01, 0.002, 0, 0.02, -0.001, 0.03]], f32),
                             np.array([0.85, 0.35], f32), np.stack([sh0, np.full(48, 0.12, f32)]))
    data = ply.write_binary_ply_bytes(scene)
    assert data.startswith(b"ply\nformat binary_little_endian 1.0\nelement vertex 2\nproperty float x\n")
    h = ply.parse_header(data)
    assert h.vertex_stride == 248 and len(h.properties) == 62 and h.sh_degree == 3
    loaded = ply.load_from_bytes(data)
    assert np.abs(loaded.positions - scene.positions).max() < 1e-4
    assert np.abs(loaded.covariances_3d - scene.covariances_3d).max() < 1e-3
    assert np.abs(loaded.opacities - scene.opacities).max() < 1e-4
    np.testing.assert_array_equal(loaded.sh_coeffs, scene.sh_coeffs)


def test_writer_round_trip_of_a_random_scene():
    """Covariance -> (log scale, quaternion) -> covariance is the identity up
    to float32 rounding, for anisotropic random Gaussians."""
    scene = random_scene(2000, seed=5)
    loaded = ply.load_from_bytes(ply.write_binary_ply_bytes(scene))
    np.testing.assert_array_equal(loaded.positions, scene.positions)
    np.testing.assert_array_equal(loaded.sh_coeffs, scene.sh_coeffs)
    rel = np.abs(loaded.covariances_3d - scene.covariances_3d).max(axis=1) / \
        np.abs(scene.covariances_3d).max(axis=1)
    assert rel.max() < 1e-4
    assert np.abs(loaded.opacities - scene.opacities).max() < 1e-5
    # a second write reproduces the first quaternion up to sign
    raw1 = ply.to_raw_vertices(scene)
    raw2 = ply.to_raw_vertices(loaded)
    q1, q2 = raw1[:, 58:62], raw2[:, 58:62]
    dots = np.abs(np.sum(q1.astype(np.float64) * q2, axis=1))
    assert np.quantile(dots, 0.99) > 1 - 1e-5
