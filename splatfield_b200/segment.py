"""The active segmentation loop over the CUDA path (B3-Seg Algorithm 1).

Mirrors suous/splatfield's src/seg/active.rs and src/seg/views.rs:

* ``localize`` (views.rs:24-66): weighted centre / radius of the foreground
  set {a > b}, reduced on the GPU (``sf_localize``);
* ``candidates`` (views.rs:73-96): N cameras on a Fibonacci sphere of radius
  1.5 r / tan(fov / 2) around the centre, each looking at it;
* ``Segmenter`` (active.rs:70-240): per round, pick a view (the caller's
  camera first, then the highest-EIG candidate), render it, ask the oracle
  for a mask, lift the mask to per-splat evidence and fold it into the Beta
  posterior. Candidates are scored by one batched ``Round`` (one CUDA graph
  per round) instead of the reference's per-view render + EIG calls;
* ``sphere_oracle`` (views.rs:131-178): the tests' perfect oracle, a pixel is
  foreground iff its camera ray hits one of the spheres.

Errors the reference reports through ``anyhow`` (bad config, a failing
oracle) raise ``ValueError`` / ``RuntimeError`` here.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass

import numpy as np

from . import _lib as L
from .core import (EIG_LUT_F32, Accumulators, BetaState, Camera, Mask, RenderScratch, Round, Splats,
                   focal, look_at, make_camera)

# Camera::BASE_FOV (src/camera.rs:25): the candidate sphere's fov.
CANDIDATE_FOV = 0.8


@dataclass
class ObjectLocalization:
    """views.rs:17-21."""

    center: np.ndarray  # float32[3]
    radius: float


def localize(splats: Splats, state: BetaState, stream=None) -> ObjectLocalization | None:
    """Where the object is per the current posterior, None while nothing is
    foreground (views.rs:24-66)."""
    found = C.c_int()
    center = np.zeros(3, np.float32)
    radius = C.c_float()
    L.check(L.lib().sf_localize(splats.handle, state.handle, _stream(stream), C.byref(found),
                                center.ctypes.data_as(C.c_void_p), C.byref(radius)))
    if not found.value:
        return None
    return ObjectLocalization(center, float(radius.value))


def candidates(loc: ObjectLocalization, count: int) -> list[Camera]:
    """``count`` cameras on a Fibonacci sphere around the object at distance
    1.5 r / tan(fov / 2), each looking at the centre (views.rs:73-96), in f32."""
    f = np.float32
    golden = (f(math.sqrt(5.0)) - f(1.0)) / f(2.0)
    radius = max(f(loc.radius), f(1e-3))  # a one-splat localization has r = 0
    dist = f(1.5) * radius / f(math.tan(f(CANDIDATE_FOV) * f(0.5)))
    center = np.asarray(loc.center, np.float32)
    cams = []
    for k in range(count):
        z = f(1.0) - f(2.0) * (f(k) + f(0.5)) / f(count)
        r = f(math.sqrt(max(f(1.0) - z * z, f(0.0))))
        theta = f(2.0) * f(math.pi) * golden * f(k)
        d = np.array([r * f(math.cos(theta)), r * f(math.sin(theta)), z], np.float32)
        cams.append(look_at(center + dist * d, center))
    return cams


def frame_bounds(bounds) -> Camera:
    """Camera::frame_bounds (src/camera.rs:46-54) applied to Camera::default:
    centred on the bounds, pulled back along -Y by twice the largest extent,
    pitched -90 degrees about X."""
    mn, mx = (np.asarray(b, np.float32) for b in bounds)
    d = np.float32((mx - mn).max() * np.float32(2.0))
    pos = (mn + mx) * np.float32(0.5) - np.array([0, 1, 0], np.float32) * d
    h = np.float32(-math.pi / 2) * np.float32(0.5)
    return make_camera(position=pos, rotation=(float(np.sin(h)), 0.0, 0.0, float(np.cos(h))))


def quat_rotate(q, v):
    """Quat * Vec3 (glam's mul_vec3 form), batched over the last axis of v."""
    b = np.asarray(q[:3], np.float32)
    w = np.float32(q[3])
    b2 = np.float32(b @ b)
    vb = v @ b
    return (v * (w * w - b2) + np.multiply.outer(vb * np.float32(2.0), b)
            + np.cross(b, v) * (w * np.float32(2.0))).astype(np.float32)


def sphere_oracle(spheres):
    """views.rs:131-178: the perfect oracle. A pixel is foreground iff its
    camera ray hits any sphere (c, r); the ray convention is the renderer's
    (screen = focal * cam.xy / cam.z + size / 2)."""
    spheres = [(np.asarray(c, np.float32), np.float32(r)) for c, r in spheres]

    def oracle(_rgb, size, camera):
        w, h = size
        fx, fy = focal(camera, w, h)
        cx, cy = np.float32(w) * np.float32(0.5), np.float32(h) * np.float32(0.5)
        ys, xs = np.mgrid[0:h, 0:w].astype(np.float32)
        cam = np.stack([(xs + np.float32(0.5) - cx) / fx, (ys + np.float32(0.5) - cy) / fy,
                        np.ones_like(xs)], -1)
        cam = cam / np.linalg.norm(cam, axis=-1, keepdims=True).astype(np.float32)
        dirs = quat_rotate(np.array(camera.rotation, np.float32), cam.reshape(-1, 3))
        pos = np.array(camera.position, np.float32)
        hit = np.zeros(w * h, bool)
        for c, r in spheres:
            oc = c - pos
            t = dirs @ oc
            oc2 = np.float32(oc @ oc)
            d2 = np.where(t < 0, oc2, oc2 - t * t)
            hit |= d2 <= r * r
        return hit.astype(np.uint8)

    return oracle


def bitmap_to_rgb(words: np.ndarray, width: int) -> np.ndarray:
    """active.rs:244-259: packed RGBA8 rows [h, row_stride] to tight RGB
    bytes (row padding and alpha dropped)."""
    w = np.ascontiguousarray(words, np.uint32)[:, :width]
    return w.view(np.uint8).reshape(w.shape[0], width, 4)[..., :3].reshape(-1).copy()


@dataclass
class Config:
    """active.rs:30-55: square render resolution, candidates per round,
    rounds."""

    resolution: int = 512
    candidates: int = 20
    iterations: int = 20


@dataclass
class Iteration:
    """active.rs:57-67."""

    camera: Camera
    eig: float
    fg_pixels: int


class Segmenter:
    """The active loop (active.rs:70-240), GPU state sized once for
    (splat count x resolution). ``eig_mode`` selects the f32 LUT (the
    reference's) or the FP64 EIG."""

    def __init__(self, splats: Splats, cfg: Config, camera: Camera, eig_mode: int = EIG_LUT_F32):
        # Validated before any GPU allocation (active.rs:89-97).
        if cfg.iterations < 1:
            raise ValueError("iterations must be >= 1")
        if cfg.resolution < 16:
            raise ValueError("resolution must be >= 16")
        if cfg.candidates < 1:
            raise ValueError("candidates must be >= 1")
        self.splats = splats
        self.cfg = cfg
        self.camera = camera
        self.eig_mode = eig_mode
        n = splats.n
        res = (cfg.resolution, cfg.resolution)
        self.state = BetaState.new_uniform(n, splats.ctx)
        self.scratch = RenderScratch(n, res, splats.ctx)
        self.acc = Accumulators(n, splats.ctx)
        self.round = Round(n, [res] * cfg.candidates, splats.ctx)
        self.bootstrapped = False

    def select_view(self, loc: ObjectLocalization):
        """Score every candidate around ``loc`` (one batched round) and keep
        the first best (active.rs:113-129: strictly greater replaces)."""
        cams = candidates(loc, self.cfg.candidates)
        eigs = self.round.eig(self.splats, self.state, cams, self.eig_mode)
        best, best_eig = cams[0], -math.inf
        for cam, e in zip(cams, eigs):
            if e > best_eig:
                best, best_eig = cam, float(e)
        return best, best_eig

    def step(self, oracle) -> Iteration:
        """One observation round (active.rs:133-181)."""
        res = (self.cfg.resolution, self.cfg.resolution)
        loc = localize(self.splats, self.state)
        if loc is not None:
            camera, eig = self.select_view(loc)
        elif not self.bootstrapped:
            camera, eig = self.camera, 0.0
        else:
            mn, mx = (np.asarray(b, np.float32) for b in self.splats.bounds)
            camera, eig = self.select_view(ObjectLocalization((mn + mx) * np.float32(0.5),
                                                              float((mx - mn).max() * np.float32(0.5))))
        self.bootstrapped = True
        isects = self.splats.prepare_isects(self.scratch, camera, res)
        words = self.splats.finalize_rgb(self.scratch, isects, res).read()
        rgb = bitmap_to_rgb(words, self.cfg.resolution)
        try:
            mask_bytes = oracle(rgb, res, camera)
        except Exception as e:  # the reference's .context("oracle failed")
            raise RuntimeError(f"oracle failed: {e}") from e
        mask = Mask.from_bytes(res, mask_bytes, self.splats.ctx)
        self.splats.accumulate_prepared(self.scratch, isects, res, self.acc, mask)
        self.state.update(self.acc)
        return Iteration(camera, eig, mask.fg_pixels)

    def run_with(self, oracle, on_round=lambda it, state: True) -> list[Iteration]:
        """T rounds with the reference's stop rules (active.rs:204-225):
        ``on_round`` returning False stops after that round; an empty mask
        ends the run while no round has seen foreground yet."""
        any_fg = False
        rounds = []
        for _ in range(self.cfg.iterations):
            it = self.step(oracle)
            any_fg |= it.fg_pixels > 0
            stop = not on_round(it, self.state)
            rounds.append(it)
            if stop or (it.fg_pixels == 0 and not any_fg):
                break
        return rounds

    def posteriors(self):
        return self.state.read()

    def segmentation(self) -> np.ndarray:
        """{i : a_i > b_i} (active.rs:229-232)."""
        a, b = self.posteriors()
        return a > b


def _stream(stream):
    if stream is None:
        return None
    if isinstance(stream, int):
        return C.c_void_p(stream)
    return C.c_void_p(int(getattr(stream, "cuda_stream")))
