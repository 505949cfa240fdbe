"""3DGS PLY scenes: the header rules and the writer (src/ply.rs tests,
:183-321) on the host, and the numpy parse restatement in oracle/ply.py
pinned against the reference's layout test. No GPU."""
import numpy as np
import pytest

import splatfield_b200 as sf
from oracle import ply as oply

BASE_PROPS = ["x", "y", "z", "rot_0", "rot_1", "rot_2", "rot_3", "scale_0", "scale_1", "scale_2", "opacity",
              "f_dc_0", "f_dc_1", "f_dc_2"]


def synthetic_ply(n, extra=()):
    """ply.rs:189-210: value (i * 31 + j) * 0.25 - 8 at row i, column j."""
    props = "".join(f"property float {p}\n" for p in BASE_PROPS + list(extra))
    head = f"ply\nformat binary_little_endian 1.0\nelement vertex {n}\n{props}end_header\n".encode()
    stride = len(BASE_PROPS) + len(extra)
    vals = np.array([(i * 31 + j) * 0.25 - 8.0 for i in range(n) for j in range(stride)], np.float32)
    return head + vals.tobytes()


def test_oracle_parse_layout_matches_reference_test():
    """ply.rs:212-249: field-major planes, rest sorted by number."""
    data = synthetic_ply(3, ["f_rest_0", "f_rest_2", "f_rest_1"])
    attr, sh = oply.parse_ply(data)
    assert attr.size == 3 * 11 and sh.size == 3 * 6
    off = data.index(b"end_header") + 11
    stride = 17

    def file(i, j):
        return np.frombuffer(data, np.float32, 1, off + (i * stride + j) * 4)[0]

    assert attr[0] == file(0, 0) and attr[3] == file(0, 1) and attr[6] == file(0, 2)
    assert attr[7 * 3] == file(0, 7) and attr[8 * 3] == file(0, 8) and attr[9 * 3] == file(0, 9)
    assert attr[10 * 3] == file(0, 10)
    for i in range(3):
        for c, rest in enumerate([14, 16, 15]):
            assert sh[c * 3 + i] == file(i, 11 + c)
            assert sh[(3 + c) * 3 + i] == file(i, rest)


def test_inspect_reports_count_and_coefficients(built_lib):
    assert sf.ply_inspect(synthetic_ply(3, ["f_rest_0", "f_rest_2", "f_rest_1"])) == (3, 2)
    assert sf.ply_inspect(synthetic_ply(5, [f"f_rest_{j}" for j in range(45)])) == (5, 16)
    assert sf.ply_inspect(synthetic_ply(2)) == (2, 1)


@pytest.mark.parametrize("header,needle", [
    ("ply\nformat binary_little_endian 1.0\nelement vertex 1\nproperty float x\nend_header\n",
     "Missing property"),
    ("ply\nformat binary_little_endian 1.0\nelement vertex 0\nproperty float x\nend_header\n",
     "no vertices"),
    ("ply\nformat binary_big_endian 1.0\nelement vertex 1\nproperty float x\nend_header\n",
     "Unsupported PLY format"),
    ("ply\nformat binary_little_endian 1.0\nelement vertex 1\nproperty float x\nproperty uchar red\nend_header\n",
     "Unsupported property type"),
])
def test_inspect_rejects_like_reference(built_lib, header, needle):
    """ply.rs:251-294 (the loader and the oracle agree on each error)."""
    with pytest.raises(sf.SplatfieldError) as e:
        sf.ply_inspect(header.encode())
    assert needle in str(e.value)
    with pytest.raises(oply.PlyError) as e2:
        oply.parse_ply(header.encode())
    assert needle in str(e2.value)


def test_missing_property_reports_first_missing(built_lib):
    props = "".join(f"property float {p}\n" for p in ["x", "y", "z", "scale_0"])
    with pytest.raises(sf.SplatfieldError) as e:
        sf.ply_inspect(f"ply\nformat binary_little_endian 1.0\nelement vertex 1\n{props}end_header\n".encode())
    assert "Missing property: scale_1" in str(e.value)


def test_truncated_vertex_block_is_reported(built_lib):
    data = synthetic_ply(4)
    with pytest.raises(sf.SplatfieldError) as e:
        sf.ply_inspect(data[:-10])
    assert "failed to read vertex 3 of 4" in str(e.value)


@pytest.mark.parametrize("k", [1, 3, 16])
def test_writer_roundtrips_through_parse(built_lib, k):
    """ply.rs:296-321: written files parse back to the exact planes."""
    n = 3
    attr = np.array([((i * 7 % 23) - 11.0) / 8.0 for i in range(11 * n)], np.float32)
    a = attr.reshape(11, n)
    a[3], a[4], a[5], a[6] = 1.0, 0.0, 0.0, 0.0
    sh = np.array([i * 0.25 - 9.0 for i in range(n * k * 3)], np.float32)
    data = sf.CpuSplats(attr, sh).write_ply()
    got_attr, got_sh = oply.parse_ply(data)
    np.testing.assert_array_equal(got_attr, attr)
    np.testing.assert_array_equal(got_sh, sh)
    assert sf.ply_inspect(data) == (n, k)
