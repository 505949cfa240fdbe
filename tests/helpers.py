"""Scenes and cameras of the reference's tests, shared by the test modules.

Each helper names the reference fixture it restates.
"""
from __future__ import annotations

import json
import math
import os

import numpy as np

GOLDEN_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def known_answers():
    with open(os.path.join(GOLDEN_DIR, "reference_known_answers.json")) as f:
        return json.load(f)


def opaque(positions) -> np.ndarray:
    """sample_opaque_attributes (src/render.rs:478-494)."""
    pos = np.asarray(positions, np.float32).reshape(-1, 3)
    n = pos.shape[0]
    a = np.zeros((11, n), np.float32)
    a[0:3] = pos.T
    a[3] = 1.0
    a[7:10] = -2.0
    a[10] = 8.0
    return a.reshape(-1)


def zero_sh(n: int, k: int = 1) -> np.ndarray:
    return np.zeros(3 * k * n, np.float32)


def stacked_positions(n=5):
    return [(0.0, 0.0, 1.0 + i * 0.5) for i in range(n)]


def row_positions(n: int, z: float, spacing: float):
    """row_attributes (src/seg/tests.rs:11-15)."""
    return [((i - (n - 1) * 0.5) * spacing, 0.0, z) for i in range(n)]


def overdraw_positions():
    """overdraw_scene (src/seg/tests.rs:78-89)."""
    out = []
    for i in range(40):
        x = float(i % 4) - 1.5
        y = float(i % 3) - 1.0
        out.append((np.float32(x) * np.float32(0.04), np.float32(y) * np.float32(0.04),
                    np.float32(1.0) + np.float32(i) * np.float32(0.5)))
    return out


def left_half_mask(w: int, h: int) -> np.ndarray:
    """left_half_mask (src/seg/tests.rs:67-72)."""
    p = np.arange(w * h)
    return ((p % w) < (w // 2)).astype(np.uint8)


def yawed_rotation():
    """Quat::from_rotation_y(pi/2) in f32 (src/render.rs:679-683)."""
    h = np.float32(math.pi / 2) * np.float32(0.5)
    return (0.0, float(np.sin(h, dtype=np.float32)), 0.0, float(np.cos(h, dtype=np.float32)))


def rgba(px):
    px = int(px)
    return [px & 255, (px >> 8) & 255, (px >> 16) & 255, (px >> 24) & 255]


def sine_attributes(n: int, freq: float, amp: float) -> np.ndarray:
    """The (i * f).sin() * amp attribute fill of test_render_reuses_scratch
    (src/render.rs:715-717) and test_scratch_stops_allocating (:737-739)."""
    i = np.arange(n * 11, dtype=np.float32)
    return (np.sin(i * np.float32(freq)) * np.float32(amp)).astype(np.float32)


def small_scene(n: int, k: int, seed: int):
    """A seeded uniform scene (the small workload's distributions) of n splats."""
    from splatfield_b200 import synth

    return synth.scene_uniform(n, k, seed)


def jitter(i: int):
    """views.rs:99-107: deterministic offset of splat i in [-0.5, 0.5]^3."""
    return np.array([((i * 73) % 17) / 17.0 - 0.5, ((i * 151) % 13) / 13.0 - 0.5,
                     ((i * 201) % 11) / 11.0 - 0.5], np.float32)


PER_CLUSTER = 40
CLUSTER_CENTERS = [((1.2, 0.0, 0.0), 0.30), ((-1.6, 0.6, 0.4), 0.45), ((0.1, -0.4, 1.9), 0.40)]


def cluster_scene():
    """views.rs:113-129: three separated spherical clusters of 40 opaque
    splats; cluster 0 is the segmentation target."""
    pos = []
    for i in range(len(CLUSTER_CENTERS) * PER_CLUSTER):
        c, r = CLUSTER_CENTERS[i // PER_CLUSTER]
        pos.append(np.asarray(c, np.float32) + np.float32(1.4 * r) * jitter(i))
    return opaque(pos), CLUSTER_CENTERS


# ---- GPU frame capture and comparison (used by the -m gpu modules)

def gpu_frame(splats, scratch, cam, w, h, n):
    """Every array of one GPU frame (prepare + RGB finalize with the float
    plane), read back for comparison with the oracle's prepare/rasterize."""
    import splatfield_b200 as sf
    from splatfield_b200 import _lib as L

    isects = splats.prepare_isects(scratch, cam, (w, h))
    bitmap = splats.finalize_rgb(scratch, isects, (w, h), want_float=True).read()
    rgba_f = sf.DeviceView(scratch.rgba_ptr(), np.float32, (h, w, 4)).read()
    V, I = isects.num_visible, isects.num_isects
    tiles = isects.tile_bounds[0] * isects.tile_bounds[1]
    depth_sorted = scratch.get_tuning()["isect_build"] == sf.ISECTS_DEPTH_SORTED
    return dict(
        depth_keys=scratch.read(L.READ_DEPTH_KEYS, n),
        tile_counts=scratch.read(L.READ_TILE_COUNTS, n),
        bbox=scratch.read(L.READ_BBOX, 2 * n),
        projected=scratch.read(L.READ_PROJECTED, 9 * n, np.float32).reshape(n, 9),
        # The binned build keeps no depth order or offsets (they are not on
        # its path); the depth-sorted build is checked on them.
        order=scratch.read(L.READ_ORDER, V) if depth_sorted else None,
        offsets=scratch.read(L.READ_OFFSETS, V) if depth_sorted else None,
        tile_ids=isects.tile_ids().read(),
        gaussian_ids=isects.gaussian_ids().read(),
        tile_start=scratch.read(L.READ_TILE_START, tiles + 1),
        bitmap=bitmap, rgba=rgba_f, num_visible=V, num_isects=I)


def assert_frame_equal(got, want):
    np.testing.assert_array_equal(got["depth_keys"], want["depth_keys"])
    np.testing.assert_array_equal(got["tile_counts"], want["tile_counts"])
    np.testing.assert_array_equal(got["bbox"], want["bbox"])
    np.testing.assert_array_equal(got["projected"].view(np.uint32), want["projected"].view(np.uint32))
    assert got["num_visible"] == want["num_visible"]
    assert got["num_isects"] == want["num_isects"]
    if got["order"] is not None:
        np.testing.assert_array_equal(got["order"], want["order"])
        np.testing.assert_array_equal(got["offsets"], want["offsets"])
    np.testing.assert_array_equal(got["tile_ids"], want["tile_ids"])
    np.testing.assert_array_equal(got["gaussian_ids"], want["gaussian_ids"])
    ranges = want["ranges"]
    np.testing.assert_array_equal(got["tile_start"][:-1], ranges[:, 0])
    np.testing.assert_array_equal(got["tile_start"][1:], ranges[:, 1])
