"""Test infrastructure: a numpy restatement of the reference's parse_sog
(src/sog.rs:97-198), the checker for the SOG loader. Its WebP planes are
decoded with Pillow's own decoder (the reference uses the `image` crate), so
it also checks the loader's WebP decoder. Not imported by the product path."""
from __future__ import annotations

import io
import json
import zipfile

import numpy as np

SQRT_2 = np.float32(1.4142135623730951)


class SogError(ValueError):
    pass


def decode_rgba(zf: zipfile.ZipFile, name: str, min_pixels: int) -> np.ndarray:
    """decode_rgba (sog.rs:44-66): [h, w, 4] uint8."""
    from PIL import Image

    try:
        data = zf.read(name)
    except KeyError:
        raise SogError(f"missing {name}") from None
    img = np.array(Image.open(io.BytesIO(data)).convert("RGBA"))
    h, w = img.shape[:2]
    if w * h < min_pixels:
        raise SogError(f"{name}: {w}x{h} < {min_pixels} pixels")
    return img


def inv_log(v: np.ndarray) -> np.ndarray:
    """sign(v) * expm1(|v|) in f32 (sog.rs:68-70)."""
    v = v.astype(np.float32)
    s = np.where(np.signbit(v), np.float32(-1), np.float32(1))
    return (s * np.expm1(np.abs(v))).astype(np.float32)


def logit(y: np.ndarray) -> np.ndarray:
    """sog.rs:72-76."""
    e = np.clip(y.astype(np.float32), np.float32(1e-6), np.float32(1 - 1e-6))
    return np.log(e / (np.float32(1) - e)).astype(np.float32)


def unpack_quat(px, py, pz, tag) -> np.ndarray:
    """sog.rs:80-93, vectorised: [4, n] (w, x, y, z)."""
    def u(v):
        return ((v.astype(np.float32) / np.float32(255) * np.float32(2) - np.float32(1)) / SQRT_2).astype(np.float32)

    a, b, c = u(px), u(py), u(pz)
    d = np.sqrt(np.maximum(((np.float32(1) - a * a) - b * b) - c * c, np.float32(0))).astype(np.float32)
    out = np.stack([a, b, c, d])
    out[:, tag == 252] = np.stack([d, a, b, c])[:, tag == 252]
    out[:, tag == 253] = np.stack([a, d, b, c])[:, tag == 253]
    out[:, tag == 254] = np.stack([a, b, d, c])[:, tag == 254]
    return out


def palette_offset(label, cw: int, coeffs: int):
    """sog.rs:202-205: (column in pixels, row)."""
    per_row = cw // coeffs
    return label % per_row * coeffs, label // per_row


def codebook(cb, what: str) -> np.ndarray:
    if len(cb) != 256:
        raise SogError(f"{what} codebook: 256 floats expected, got {len(cb)}")
    return np.asarray(cb, np.float32)


def parse_sog(data: bytes):
    """(attributes [11 n], sh [3 k n]) as parse_sog returns them."""
    try:
        zf = zipfile.ZipFile(io.BytesIO(data))
    except zipfile.BadZipFile:
        raise SogError("not a SOG archive") from None
    try:
        meta = json.loads(zf.read("meta.json"))
    except KeyError:
        raise SogError("missing meta.json") from None
    n = int(meta["count"])
    if n == 0:
        raise SogError("SOG contains no splats")
    attr = np.zeros((11, n), np.float32)
    lo = decode_rgba(zf, meta["means"]["files"][0], n).reshape(-1, 4)[:n]
    hi = decode_rgba(zf, meta["means"]["files"][1], n).reshape(-1, 4)[:n]
    mins = np.asarray(meta["means"]["mins"], np.float32)
    spans = np.asarray(meta["means"]["maxs"], np.float32) - mins
    for k in range(3):
        t = (lo[:, k].astype(np.uint32) | (hi[:, k].astype(np.uint32) << 8)).astype(np.float32) / np.float32(65535)
        attr[k] = inv_log(mins[k] + spans[k] * t)
    sl = decode_rgba(zf, meta["scales"]["files"][0], n).reshape(-1, 4)[:n]
    scb = codebook(meta["scales"]["codebook"], "scales")
    for k in range(3):
        attr[7 + k] = scb[sl[:, k]]
    qr = decode_rgba(zf, meta["quats"]["files"][0], n).reshape(-1, 4)[:n]
    bad = qr[:, 3] < 252
    if bad.any():
        raise SogError(f"quats: invalid rotation tag {int(qr[np.argmax(bad), 3])}")
    attr[3:7] = unpack_quat(qr[:, 0], qr[:, 1], qr[:, 2], qr[:, 3])
    shn = meta.get("shN")
    k = 1 if shn is None else {1: 4, 2: 9, 3: 16}.get(shn["bands"])
    if k is None:
        raise SogError(f"shN.bands {shn['bands']} outside 1..=3")
    c0 = decode_rgba(zf, meta["sh0"]["files"][0], n).reshape(-1, 4)[:n]
    sh = np.zeros((k, 3, n), np.float32)
    s0 = codebook(meta["sh0"]["codebook"], "sh0")
    for c in range(3):
        sh[0, c] = s0[c0[:, c]]
    attr[10] = logit(c0[:, 3].astype(np.float32) / np.float32(255))
    if shn is not None:
        coeffs = k - 1
        cent = decode_rgba(zf, shn["files"][0], 1)
        labels_img = decode_rgba(zf, shn["files"][1], n).reshape(-1, 4)[:n]
        cb = codebook(shn["codebook"], "shN")
        cw = cent.shape[1]
        flat = cent.reshape(-1, 4)
        palettes = flat.shape[0] // coeffs
        labels = labels_img[:, 0].astype(np.int64) | (labels_img[:, 1].astype(np.int64) << 8)
        if (labels >= palettes).any():
            lab = int(labels[np.argmax(labels >= palettes)])
            raise SogError(f"shN label {lab} >= palette size {palettes}")
        bx, by = palette_offset(labels, cw, coeffs)
        for j in range(coeffs):
            p = by * cw + bx + j
            for c in range(3):
                sh[j + 1, c] = cb[flat[p, c]]
    return attr.reshape(-1), sh.reshape(-1)
