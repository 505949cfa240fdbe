"""Writes the SOG fixtures of tests/test_sog.py and tests/test_gpu_sog.py.

The reference's own SOG test scenes (bear*.sog) are release downloads and
not in this tree, so these fixtures are synthetic, built here by a small SOG
writer that follows the layout parse_sog reads (src/sog.rs:8-198): meta.json
plus lossless WebP planes (Pillow's encoder) in a zip archive, one pixel per
splat, row-major over a fixed plane width. `make_sog` returns the archive
bytes and the quantised sources it encoded, so a test can compare a decoder
with the values that went in.

Run from the repository root:  python tests/golden/make_sog_fixtures.py
"""
from __future__ import annotations

import io
import json
import math
import os
import zipfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
FIXTURES = {"sog_bands0.sog": (600, 0, 1), "sog_bands1.sog": (777, 1, 2), "sog_bands3.sog": (1000, 3, 3)}


def webp_lossless(pixels: np.ndarray) -> bytes:
    from PIL import Image

    b = io.BytesIO()
    Image.fromarray(np.ascontiguousarray(pixels, np.uint8), "RGBA").save(b, "WEBP", lossless=True, quality=100,
                                                                         method=4, exact=True)
    return b.getvalue()


def plane(values: np.ndarray, width: int) -> np.ndarray:
    """[n, 4] bytes -> a [rows, width, 4] image, padded with zeros."""
    n = values.shape[0]
    rows = (n + width - 1) // width
    img = np.zeros((rows * width, 4), np.uint8)
    img[:n] = values
    return img.reshape(rows, width, 4)


def make_sog(n: int, bands: int, seed: int, width: int = 64, stored: bool = False, meta_edit=None,
             quat_tags=None):
    """A SOG archive of n splats with shN bands (0: none). Returns (bytes,
    sources): the u16 means, codebook indices, packed quaternions, opacity
    bytes, palette and labels that were encoded."""
    rng = np.random.default_rng(seed)
    src = {}
    mins = np.sort(rng.normal(0.0, 1.0, 3)).astype(np.float32) - 1.5
    maxs = mins + rng.uniform(0.5, 3.0, 3).astype(np.float32)
    means16 = rng.integers(0, 65536, (n, 3)).astype(np.uint32)
    src["means16"], src["mins"], src["maxs"] = means16, mins, maxs
    lo = np.zeros((n, 4), np.uint8)
    hi = np.zeros((n, 4), np.uint8)
    lo[:, :3] = means16 & 0xFF
    hi[:, :3] = means16 >> 8
    lo[:, 3] = hi[:, 3] = 255
    scales_cb = np.sort(rng.normal(-4.0, 1.0, 256)).astype(np.float32)
    scale_idx = rng.integers(0, 256, (n, 3)).astype(np.uint8)
    sc = np.zeros((n, 4), np.uint8)
    sc[:, :3] = scale_idx
    sc[:, 3] = 255
    src["scales_cb"], src["scale_idx"] = scales_cb, scale_idx
    # Quaternions: the largest component is dropped and its index is the tag
    # (252 + index, w x y z), the other three stored in order, sign-flipped
    # so the dropped one is non-negative.
    q = rng.normal(size=(n, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    big = np.argmax(np.abs(q), axis=1)
    q *= np.where(q[np.arange(n), big] < 0, -1.0, 1.0)[:, None]
    qs = np.zeros((n, 4), np.uint8)
    for i in range(n):
        rest = [q[i, j] for j in range(4) if j != big[i]]
        qs[i, :3] = np.clip(np.round((np.array(rest) * math.sqrt(2) + 1.0) / 2.0 * 255.0), 0, 255)
    qs[:, 3] = 252 + big
    if quat_tags is not None:
        qs[:, 3] = quat_tags
    src["quats"] = qs
    sh0_cb = np.sort(rng.normal(0.0, 0.6, 256)).astype(np.float32)
    sh0_idx = rng.integers(0, 256, (n, 3)).astype(np.uint8)
    opac = rng.integers(0, 256, n).astype(np.uint8)
    c0 = np.zeros((n, 4), np.uint8)
    c0[:, :3] = sh0_idx
    c0[:, 3] = opac
    src["sh0_cb"], src["sh0_idx"], src["opacity"] = sh0_cb, sh0_idx, opac
    meta = {"version": 2, "count": n,
            "means": {"mins": mins.tolist(), "maxs": maxs.tolist(), "files": ["means_l.webp", "means_u.webp"]},
            "scales": {"codebook": scales_cb.tolist(), "files": ["scales.webp"]},
            "quats": {"files": ["quats.webp"]},
            "sh0": {"codebook": sh0_cb.tolist(), "files": ["sh0.webp"]}}
    files = {"means_l.webp": plane(lo, width), "means_u.webp": plane(hi, width), "scales.webp": plane(sc, width),
             "quats.webp": plane(qs, width), "sh0.webp": plane(c0, width)}
    if bands:
        coeffs = (bands + 1) ** 2 - 1
        palettes = 96
        per_row = 4
        cw = per_row * coeffs
        rows = (palettes + per_row - 1) // per_row
        cent = rng.integers(0, 256, (rows, cw, 4)).astype(np.uint8)
        cent[..., 3] = 255
        labels = rng.integers(0, palettes, n).astype(np.uint32)
        lab = np.zeros((n, 4), np.uint8)
        lab[:, 0] = labels & 0xFF
        lab[:, 1] = labels >> 8
        lab[:, 3] = 255
        shn_cb = np.sort(rng.normal(0.0, 0.2, 256)).astype(np.float32)
        meta["shN"] = {"bands": bands, "codebook": shn_cb.tolist(), "files": ["shN_centroids.webp", "shN_labels.webp"]}
        files["shN_centroids.webp"] = cent
        files["shN_labels.webp"] = plane(lab, width)
        src["centroids"], src["labels"], src["shn_cb"], src["coeffs"] = cent, labels, shn_cb, coeffs
    if meta_edit is not None:
        meta_edit(meta)
    out = io.BytesIO()
    method = zipfile.ZIP_STORED if stored else zipfile.ZIP_DEFLATED
    with zipfile.ZipFile(out, "w", method) as zf:
        zf.writestr("meta.json", json.dumps(meta))
        for name, img in files.items():
            zf.writestr(name, webp_lossless(img))
    return out.getvalue(), src


def expected_planes(src: dict, n: int, bands: int):
    """The planes parse_sog gives for these sources (sog.rs:114-193), in f32."""
    from oracle import sog as O

    attr = np.zeros((11, n), np.float32)
    spans = src["maxs"] - src["mins"]
    for k in range(3):
        t = src["means16"][:, k].astype(np.float32) / np.float32(65535)
        attr[k] = O.inv_log(src["mins"][k] + spans[k] * t)
    for k in range(3):
        attr[7 + k] = src["scales_cb"][src["scale_idx"][:, k]]
    qs = src["quats"]
    attr[3:7] = O.unpack_quat(qs[:, 0], qs[:, 1], qs[:, 2], qs[:, 3])
    attr[10] = O.logit(src["opacity"].astype(np.float32) / np.float32(255))
    k = {0: 1, 1: 4, 2: 9, 3: 16}[bands]
    sh = np.zeros((k, 3, n), np.float32)
    for c in range(3):
        sh[0, c] = src["sh0_cb"][src["sh0_idx"][:, c]]
    if bands:
        coeffs = src["coeffs"]
        cent = src["centroids"]
        cw = cent.shape[1]
        flat = cent.reshape(-1, 4)
        bx, by = O.palette_offset(src["labels"].astype(np.int64), cw, coeffs)
        for j in range(coeffs):
            for c in range(3):
                sh[j + 1, c] = src["shn_cb"][flat[by * cw + bx + j, c]]
    return attr.reshape(-1), sh.reshape(-1)


if __name__ == "__main__":
    import sys

    sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
    for name, (n, bands, seed) in FIXTURES.items():
        data, _ = make_sog(n, bands, seed, stored=(bands == 1))
        with open(os.path.join(HERE, name), "wb") as f:
            f.write(data)
        print(name, len(data), "bytes")
