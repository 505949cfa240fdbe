"""Test infrastructure: a numpy restatement of the reference's parse_ply
(src/ply.rs:9-112), the checker for the CUDA PLY loader. Not imported by the
product path."""
from __future__ import annotations

import numpy as np

REQUIRED = ["x", "y", "z", "scale_0", "scale_1", "scale_2", "opacity", "rot_0", "rot_1", "rot_2", "rot_3",
            "f_dc_0", "f_dc_1", "f_dc_2"]


class PlyError(ValueError):
    pass


def parse_ply(data: bytes):
    """(attributes [11 n], sh [3 k n]) as parse_ply returns them (ply.rs:9-112)."""
    pos, n, props = 0, 0, []
    while pos < len(data):  # header lines (ply.rs:13-31)
        e = data.find(b"\n", pos)
        e = len(data) if e < 0 else e
        line = data[pos:e].decode("latin-1").rstrip("\r")
        pos = min(e + 1, len(data))
        t = line.split()
        if t[:1] == ["end_header"]:
            break
        if len(t) >= 2 and t[0] == "format" and t[1] != "binary_little_endian":
            raise PlyError(f"Unsupported PLY format: {t[1]}")
        if len(t) == 3 and t[0] == "element" and t[1] == "vertex":
            n = int(t[2])
        if len(t) == 3 and t[0] == "property":
            if t[1] != "float":
                raise PlyError(f"Unsupported property type {t[1]}: {t[2]}")
            props.append(t[2])
    if n == 0:
        raise PlyError("PLY contains no vertices")
    idx = {}
    for name in REQUIRED:  # first missing name reported (ply.rs:46-53)
        if name not in props:
            raise PlyError(f"Missing property: {name}")
        idx[name] = props.index(name)
    rest = sorted(((int(p[7:]), i) for i, p in enumerate(props)
                   if p.startswith("f_rest_") and p[7:].isdigit()), key=lambda t: t[0])
    stride = len(props)
    m = len(rest) // 3
    rows = np.frombuffer(data, np.float32, count=n * stride, offset=pos).reshape(n, stride)
    attr = np.zeros((11, n), np.float32)
    # glam Quat::from_xyzw(rot_1, rot_2, rot_3, rot_0).normalize(), SSE2 dot
    # order (x2 + z2) + (y2 + w2), q * (1 / sqrt(dot)).
    qx, qy, qz, qw = (rows[:, idx[k]] for k in ("rot_1", "rot_2", "rot_3", "rot_0"))
    d = (qx * qx + qz * qz) + (qy * qy + qw * qw)
    inv = np.float32(1.0) / np.sqrt(d)
    for plane, v in enumerate([rows[:, idx["x"]], rows[:, idx["y"]], rows[:, idx["z"]], qw * inv, qx * inv,
                               qy * inv, qz * inv, rows[:, idx["scale_0"]], rows[:, idx["scale_1"]],
                               rows[:, idx["scale_2"]], rows[:, idx["opacity"]]]):
        attr[plane] = v
    sh = np.zeros((3 * (m + 1), n), np.float32)
    for c in range(3):
        sh[c] = rows[:, idx[f"f_dc_{c}"]]
    for j in range(m):
        for c in range(3):
            sh[(j + 1) * 3 + c] = rows[:, rest[c * m + j][1]]
    return attr.reshape(-1), sh.reshape(-1)
