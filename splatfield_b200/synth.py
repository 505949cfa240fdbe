"""Seeded synthetic scenes, cameras and masks for the benchmark workloads.

The reference benchmarks a real scan (bear.sog, 970,948 SH-3 splats) that is
not available here; these generators produce scenes of the same scale and
value distributions instead. Randomness is splitmix64 (counter-based, one
64-bit word per draw) with Box–Muller normals, so every array is a pure
function of (seed, stream, index) and reproducible on any machine.

Workloads:
  small     100k splats, SH0, uniform means in [-1,1]^3, one 512x512 camera
            at (0,0,-3) with a 60-degree fov.
  frame     1M splats, SH3, means from 8 Gaussian clusters (sigma 0.3,
            centres in [-2,2]^3), 1920x1080, 30 cameras on a radius-4 orbit.
  round     the frame scene + Beta(a, b) with a, b log-uniform in [1, 1024],
            20 cameras uniform on a radius-3.5 sphere at 512x512, one mask of
            1-3 random ellipses (5-30% of pixels) per view.
  adjoint   the frame scene, one camera; the target is the render of a copy
            with means + N(0, 0.01) and opacity logits + N(0, 0.2).
  uneven    3M splats, SH1, clustered; 64 views with sides drawn from
            {256, 384, 512, 768, 1024}; ellipse masks.
"""
from __future__ import annotations

import math

import numpy as np

GOLDEN = np.uint64(0x9E3779B97F4A7C15)
M1 = np.uint64(0xBF58476D1CE4E5B9)
M2 = np.uint64(0x94D049BB133111EB)


def _mix(z: np.ndarray) -> np.ndarray:
    z = (z ^ (z >> np.uint64(30))) * M1
    z = (z ^ (z >> np.uint64(27))) * M2
    return z ^ (z >> np.uint64(31))


class Rng:
    """Counter-based splitmix64 stream: draw k of stream s is mix(seed' + k*golden)."""

    def __init__(self, seed: int, stream: int = 0):
        base = np.uint64((seed * 0x632BE59BD9B4E019 + stream * 0x8CB92BA72F3D8DD7) & 0xFFFFFFFFFFFFFFFF)
        self.base = _mix(np.array([base], np.uint64))[0]
        self.pos = 0

    def u64(self, n: int) -> np.ndarray:
        with np.errstate(over="ignore"):
            k = np.arange(self.pos + 1, self.pos + n + 1, dtype=np.uint64)
            z = self.base + k * GOLDEN
            out = _mix(z)
        self.pos += n
        return out

    def uniform(self, n: int) -> np.ndarray:
        """Doubles in [0, 1)."""
        return (self.u64(n) >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)

    def normal(self, n: int) -> np.ndarray:
        """Box–Muller standard normals."""
        m = (n + 1) // 2
        u1 = 1.0 - self.uniform(m)
        u2 = self.uniform(m)
        r = np.sqrt(-2.0 * np.log(u1))
        z = np.concatenate([r * np.cos(2 * math.pi * u2), r * np.sin(2 * math.pi * u2)])
        return z[:n]

    def integers(self, lo: int, hi: int, n: int) -> np.ndarray:
        return lo + (self.uniform(n) * (hi - lo)).astype(np.int64)


def _assemble(means, log_scales, quats, opacity_logit, sh):
    n = means.shape[0]
    attr = np.empty((11, n), np.float32)
    attr[0:3] = means.T
    attr[3:7] = quats.T
    attr[7:10] = log_scales.T
    attr[10] = opacity_logit
    return attr.reshape(-1), np.ascontiguousarray(sh, np.float32).reshape(-1)


def _common(rng: Rng, n: int, k: int):
    log_scales = -4.0 + 0.5 * rng.normal(3 * n).reshape(n, 3)
    q = rng.normal(4 * n).reshape(n, 4)
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    opacity = 1.5 * rng.normal(n)
    sh = np.empty((k, 3, n), np.float64)
    sh[0] = 0.5 * rng.normal(3 * n).reshape(3, n)
    if k > 1:
        sh[1:] = 0.1 * rng.normal(3 * (k - 1) * n).reshape(k - 1, 3, n)
    return log_scales, q, opacity, sh


def scene_uniform(n: int = 100_000, sh_per_ch: int = 1, seed: int = 0):
    """Means uniform in [-1,1]^3 (the small CPU-runnable workload)."""
    rng = Rng(seed, 1)
    means = rng.uniform(3 * n).reshape(n, 3) * 2.0 - 1.0
    return _assemble(means, *_common(rng, n, sh_per_ch))


def scene_clustered(n: int = 1_000_000, sh_per_ch: int = 16, seed: int = 0, clusters: int = 8,
                    sigma: float = 0.3, extent: float = 2.0):
    """Means from `clusters` isotropic Gaussians, clamped to [-extent, extent]^3."""
    rng = Rng(seed, 2)
    centres = rng.uniform(3 * clusters).reshape(clusters, 3) * (2 * extent) - extent
    which = rng.integers(0, clusters, n)
    means = centres[which] + sigma * rng.normal(3 * n).reshape(n, 3)
    means = np.clip(means, -extent, extent)
    return _assemble(means, *_common(rng, n, sh_per_ch))


def fov_for(w: int, h: int, vertical_deg: float = 60.0):
    """Vertical fov fixed, horizontal from the aspect so that fx == fy."""
    fy = math.radians(vertical_deg)
    fx = 2.0 * math.atan(math.tan(fy / 2.0) * w / h)
    return (fx, fy)


def orbit_cameras(count: int, radius: float, w: int, h: int, make_look_at, vertical_deg=60.0):
    """`count` cameras evenly spaced on the equatorial (y = 0) circle, looking at the origin."""
    fov = fov_for(w, h, vertical_deg)
    cams = []
    for i in range(count):
        t = 2.0 * math.pi * (i + 0.25) / count
        cam = make_look_at((radius * math.cos(t), 0.0, radius * math.sin(t)), (0.0, 0.0, 0.0))
        cam.fov[0], cam.fov[1] = fov
        cams.append(cam)
    return cams


def sphere_cameras(count: int, radius: float, seed: int, make_look_at, fov_deg=60.0):
    """`count` cameras uniform on a sphere, looking at the origin."""
    rng = Rng(seed, 3)
    cams = []
    while len(cams) < count:
        v = rng.normal(3)
        nv = float(np.linalg.norm(v))
        if nv < 1e-6:
            continue
        v = v / nv * radius
        cam = make_look_at(tuple(v), (0.0, 0.0, 0.0))
        f = math.radians(fov_deg)
        cam.fov[0], cam.fov[1] = f, f
        cams.append(cam)
    return cams


def beta_posterior(n: int, seed: int = 0):
    """a, b log-uniform in [1, 1024]."""
    rng = Rng(seed, 4)
    a = np.exp(rng.uniform(n) * math.log(1024.0)).astype(np.float32)
    b = np.exp(rng.uniform(n) * math.log(1024.0)).astype(np.float32)
    return a, b


def ellipse_mask(w: int, h: int, seed: int, stream: int = 5):
    """Union of 1-3 random ellipses covering 5-30% of the pixels (bytes, row-major)."""
    rng = Rng(seed, stream)
    yy, xx = np.mgrid[0:h, 0:w]
    for _ in range(64):
        k = 1 + int(rng.integers(0, 3, 1)[0])
        m = np.zeros((h, w), bool)
        for _e in range(k):
            cx, cy = rng.uniform(2) * (w, h)
            ax, ay = (0.08 + 0.3 * rng.uniform(2)) * (w, h)
            th = rng.uniform(1)[0] * math.pi
            c, s = math.cos(th), math.sin(th)
            dx, dy = xx + 0.5 - cx, yy + 0.5 - cy
            u = (c * dx + s * dy) / ax
            v = (-s * dx + c * dy) / ay
            m |= (u * u + v * v) <= 1.0
        frac = m.mean()
        if 0.05 <= frac <= 0.30:
            return m.astype(np.uint8).reshape(-1)
    return m.astype(np.uint8).reshape(-1)


def perturbed(attributes: np.ndarray, n: int, seed: int = 0):
    """The adjoint workload's target scene: means + N(0, 0.01), opacity logits + N(0, 0.2)."""
    rng = Rng(seed, 6)
    a = attributes.reshape(11, n).astype(np.float64).copy()
    a[0:3] += 0.01 * rng.normal(3 * n).reshape(3, n)
    a[10] += 0.2 * rng.normal(n)
    return a.astype(np.float32).reshape(-1)


UNEVEN_SIDES = (256, 384, 512, 768, 1024)


def uneven_sizes(views: int = 64, seed: int = 0):
    rng = Rng(seed, 7)
    idx = rng.integers(0, len(UNEVEN_SIDES), views)
    return [UNEVEN_SIDES[i] for i in idx]


def opaque_attributes(positions) -> np.ndarray:
    """sample_opaque_attributes (src/render.rs:478-494): identity rotation,
    log-scale -2, opacity logit 8, at the given positions."""
    pos = np.asarray(positions, np.float32).reshape(-1, 3)
    n = pos.shape[0]
    a = np.zeros((11, n), np.float32)
    a[0:3] = pos.T
    a[3] = 1.0
    a[7:10] = -2.0
    a[10] = 8.0
    return a.reshape(-1)


# ---- the workloads' fixed draws (shared by the benchmark and the tests)

ROUND_VIEWS, ROUND_SIDE, ROUND_RADIUS = 20, 512, 3.5


def round_workload(n: int, make_look_at):
    """The segmentation round on an n-splat scene: posterior a, b (seed 1),
    20 cameras on a radius-3.5 sphere (seed 2), one 512x512 ellipse-union
    mask per view (seeds 100 + v, bytes row-major)."""
    a, b = beta_posterior(n, seed=1)
    cams = sphere_cameras(ROUND_VIEWS, ROUND_RADIUS, 2, make_look_at)
    masks = [ellipse_mask(ROUND_SIDE, ROUND_SIDE, seed=100 + v) for v in range(ROUND_VIEWS)]
    return a, b, cams, masks


UNEVEN_SPLATS, UNEVEN_SH, UNEVEN_VIEWS = 3_000_000, 4, 64


def uneven_scene():
    """3M splats, SH degree 1, clustered as the frame scene (seed 7)."""
    return scene_clustered(UNEVEN_SPLATS, UNEVEN_SH, seed=7)


def uneven_workload(make_look_at, views: int = UNEVEN_VIEWS):
    """The uneven round's draws: per view a side from UNEVEN_SIDES, a camera
    on the radius-3.5 sphere (seed 9) and an ellipse mask (seeds 300 + v);
    posterior a, b (seed 5)."""
    rng = np.random.default_rng(11)
    sides = [int(x) for x in rng.choice(UNEVEN_SIDES, UNEVEN_VIEWS)][:views]
    cams = sphere_cameras(UNEVEN_VIEWS, ROUND_RADIUS, 9, make_look_at)[:views]
    masks = [ellipse_mask(s, s, seed=300 + v) for v, s in enumerate(sides)]
    a, b = beta_posterior(UNEVEN_SPLATS, seed=5)
    return sides, cams, masks, a, b

