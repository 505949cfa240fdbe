"""CPU oracle for the splat render + segmentation-evidence path.

TEST INFRASTRUCTURE ONLY. This package restates the reference
(suous/splatfield v0.2.0, Rust/cubecl) in C++ (``sfo_*.cpp``); the test suite,
``__graft_entry__.smoke()`` and the benchmark's CPU-baseline leg load it, and
only as the checker or the timed CPU baseline. The product path (package
``splatfield_b200``) never imports it.

Parity pins: the known-answer vectors of the reference's own tests
(``tests/golden/reference_known_answers.json``, read from the reference's test
sources as text). The reference itself cannot be built in this environment
(Rust toolchain absent, wgpu is its only runtime), so there is no ``_ref``
build; bit parity with the reference's Metal-driver rounding is unpinned and
the u32 responsibility golden is matched within a stated tolerance.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "liboracle_sf.so")


def build() -> str:
    """Compile the oracle with its Makefile; returns the library path."""
    import subprocess

    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


class Camera(C.Structure):
    """Camera{fov, position, rotation} (src/camera.rs:5-9); rotation x,y,z,w."""

    _fields_ = [("fov", C.c_float * 2), ("position", C.c_float * 3), ("rotation", C.c_float * 4)]


class View(C.Structure):
    """CameraView kernel scalars (src/project.rs:63-74)."""

    _fields_ = [
        ("rot0", C.c_float * 3),
        ("rot1", C.c_float * 3),
        ("rot2", C.c_float * 3),
        ("trans", C.c_float * 3),
        ("focal", C.c_float * 2),
        ("world_pos", C.c_float * 3),
        ("img", C.c_float * 2),
        ("tile_bounds", C.c_float * 2),
    ]


class FrameInfo(C.Structure):
    _fields_ = [
        ("num_visible", C.c_uint32),
        ("num_isects", C.c_uint64),
        ("tiles_x", C.c_uint32),
        ("tiles_y", C.c_uint32),
        ("row_stride", C.c_uint32),
    ]


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = C.CDLL(_LIB_PATH)
        P = C.c_void_p
        u32, u64, f32, f64, i32 = C.c_uint32, C.c_uint64, C.c_float, C.c_double, C.c_int
        sig = {
            "sfo_camera_look_at": (None, [P, P, P]),
            "sfo_view_for_camera": (None, [P, u32, u32, P]),
            "sfo_project": (u32, [P, P, P, u32, u32, P, P, P, P, P]),
            "sfo_depth_order": (u32, [P, u32, P]),
            "sfo_scan_gather": (u64, [P, P, u32, P]),
            "sfo_emit": (None, [P, P, P, u32, u32, P, P]),
            "sfo_sort_pairs": (None, [P, P, u32, u32, P, P]),
            "sfo_tile_ranges": (None, [P, u32, u32, P]),
            "sfo_rasterize": (None, [i32, u32, u32, u32, P, P, P, f32, P, u32, P, P, P, P, P, P, P]),
            "sfo_prepare": (i32, [P, u32, u32, P, P, u32, u32, P, P, P, P, P, P, P, P, u64, P, P]),
            "sfo_fractional_bits": (u32, [u32, u32]),
            "sfo_scale_for": (f32, [u32, u32]),
            "sfo_mask_pack": (u32, [P, u32, u32, P]),
            "sfo_lgamma": (f64, [f64]),
            "sfo_digamma": (f64, [f64]),
            "sfo_beta_entropy": (f64, [f64, f64]),
            "sfo_entropy_table": (None, [P]),
            "sfo_table_entropy": (f32, [f32, f32, P]),
            "sfo_delta_lut": (f32, [f32, f32, u32, f32, P]),
            "sfo_delta_f64": (f64, [f32, f32, u32, f32]),
            "sfo_eig": (f64, [i32, P, P, P, u32, f32, P]),
            "sfo_beta_update": (None, [f32, P, P, P, P, u32]),
            "sfo64_render": (i32, [P, u32, u32, P, P, u32, u32, P]),
            "sfo64_render_backward": (i32, [P, u32, u32, P, P, u32, u32, P, P, P]),
            "sfo64_probe_open": (P, [P, u32, u32, P, P, u32, u32, P]),
            "sfo64_probe_close": (None, [P]),
            "sfo64_probe_bbox": (i32, [P, u32, P]),
            "sfo64_probe_loss": (f64, [P, u32, u32, f64, u32, u32, u32, u32]),
            "sfo_num_threads": (i32, []),
            "sfo_set_num_threads": (None, [i32]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def _p(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def _c(a, dtype):
    return np.ascontiguousarray(a, dtype=dtype)


def camera(fov=(0.8, 0.8), position=(0.0, 0.0, 0.0), rotation=(0.0, 0.0, 0.0, 1.0)) -> Camera:
    c = Camera()
    c.fov[:] = list(fov)
    c.position[:] = list(position)
    c.rotation[:] = list(rotation)
    return c


def look_at(position, target) -> Camera:
    """Camera::look_at (src/camera.rs:57-63)."""
    out = Camera()
    p = _c(position, np.float32)
    t = _c(target, np.float32)
    lib().sfo_camera_look_at(_p(p), _p(t), C.byref(out))
    return out


def view_for_camera(cam: Camera, w: int, h: int) -> View:
    v = View()
    lib().sfo_view_for_camera(C.byref(cam), w, h, C.byref(v))
    return v


def row_stride(w: int) -> int:
    """Bitmap row stride in words: rows padded to 256 bytes (src/render.rs:150)."""
    return ((4 * w + 255) // 256 * 256) // 4


def project(view: View, attributes, sh, n: int, sh_per_ch: int):
    attributes = _c(attributes, np.float32)
    sh = _c(sh, np.float32)
    keys = np.empty(n, np.uint32)
    counts = np.empty(n, np.uint32)
    bbox = np.empty(2 * n, np.uint32)
    proj = np.empty(9 * n, np.float32)
    total = C.c_uint64(0)
    vis = lib().sfo_project(C.byref(view), _p(attributes), _p(sh), n, sh_per_ch, _p(keys),
                            _p(counts), _p(bbox), _p(proj), C.byref(total))
    return dict(visible=int(vis), total=int(total.value), depth_keys=keys, tile_counts=counts,
                bbox=bbox, projected=proj.reshape(n, 9))


def depth_order(keys):
    keys = _c(keys, np.uint32)
    order = np.empty(len(keys), np.uint32)
    v = lib().sfo_depth_order(_p(keys), len(keys), _p(order))
    return order[:v]


def scan_gather(gids, counts):
    gids = _c(gids, np.uint32)
    counts = _c(counts, np.uint32)
    out = np.empty(len(gids), np.uint32)
    total = lib().sfo_scan_gather(_p(gids), _p(counts), len(gids), _p(out))
    return out, int(total)


def sort_pairs(keys, vals, bits):
    keys = _c(keys, np.uint32)
    vals = _c(vals, np.uint32)
    ko = np.empty_like(keys)
    vo = np.empty_like(vals)
    lib().sfo_sort_pairs(_p(keys), _p(vals), len(keys), bits, _p(ko), _p(vo))
    return ko, vo


def prepare(cam: Camera, w: int, h: int, attributes, sh, sh_per_ch: int, capacity: int | None = None):
    """Project, depth-sort, scan, emit, tile-sort and range one frame."""
    attributes = _c(attributes, np.float32)
    sh = _c(sh, np.float32)
    n = attributes.size // 11
    tx, ty = (w + 15) // 16, (h + 15) // 16
    keys = np.empty(n, np.uint32)
    counts = np.empty(n, np.uint32)
    bbox = np.empty(2 * n, np.uint32)
    proj = np.empty(9 * n, np.float32)
    order = np.empty(n, np.uint32)
    offsets = np.empty(n, np.uint32)
    ranges = np.empty(2 * tx * ty, np.uint32)
    info = FrameInfo()
    if capacity is None:
        view = view_for_camera(cam, w, h)
        capacity = project(view, attributes, sh, n, sh_per_ch)["total"]
    tids = np.empty(max(capacity, 1), np.uint32)
    gids = np.empty(max(capacity, 1), np.uint32)
    rc = lib().sfo_prepare(C.byref(cam), w, h, _p(attributes), _p(sh), n, sh_per_ch, _p(keys),
                           _p(counts), _p(bbox), _p(proj), _p(order), _p(offsets), _p(tids),
                           _p(gids), capacity, _p(ranges), C.byref(info))
    if rc != 0:
        raise RuntimeError(f"oracle: {info.num_isects} intersections exceed capacity {capacity}")
    V, I = info.num_visible, int(info.num_isects)
    return dict(depth_keys=keys, tile_counts=counts, bbox=bbox, projected=proj.reshape(n, 9),
                order=order[:V], offsets=offsets[:V], tile_ids=tids[:I], gaussian_ids=gids[:I],
                ranges=ranges.reshape(-1, 2), num_visible=V, num_isects=I, tiles_x=tx,
                tiles_y=ty, row_stride=info.row_stride, w=w, h=h)


def rasterize(prep: dict, mode: int = 0, scale: float = 0.0, mask_bits=None, words_per_row: int = 0,
              want_float: bool = True, want_state: bool = False):
    """rasterize_kernel over a prepared frame; mode 0 RGB, 1 total, 2 evidence."""
    w, h = prep["w"], prep["h"]
    n = prep["projected"].shape[0]
    rs = prep["row_stride"]
    out = {}
    bitmap = np.zeros(h * rs, np.uint32) if mode == 0 else None
    rgba = np.zeros(h * w * 4, np.float32) if (mode == 0 and want_float) else None
    resp = np.zeros(n, np.uint32) if mode == 1 else None
    fg = np.zeros(n, np.uint32) if mode == 2 else None
    bg = np.zeros(n, np.uint32) if mode == 2 else None
    ft = np.zeros(h * w, np.float32) if want_state else None
    nc = np.zeros(h * w, np.uint32) if want_state else None
    mask = _c(mask_bits, np.uint32) if mask_bits is not None else None
    ranges = _c(prep["ranges"], np.uint32)
    gids = _c(prep["gaussian_ids"], np.uint32)
    proj = _c(prep["projected"], np.float32)
    lib().sfo_rasterize(mode, w, h, rs, _p(ranges), _p(gids), _p(proj), scale, _p(mask),
                        words_per_row, _p(bitmap), _p(rgba), _p(resp), _p(fg), _p(bg), _p(ft), _p(nc))
    if bitmap is not None:
        out["bitmap"] = bitmap.reshape(h, rs)
    if rgba is not None:
        out["rgba"] = rgba.reshape(h, w, 4)
    if resp is not None:
        out["resp"] = resp
    if fg is not None:
        out["fg"], out["bg"] = fg, bg
    if want_state:
        out["final_t"] = ft.reshape(h, w)
        out["n_contrib"] = nc.reshape(h, w)
    return out


def render(cam: Camera, w: int, h: int, attributes, sh, sh_per_ch: int, **kw):
    prep = prepare(cam, w, h, attributes, sh, sh_per_ch)
    out = rasterize(prep, 0, **kw)
    out["prep"] = prep
    return out


def fractional_bits(w: int, h: int) -> int:
    return int(lib().sfo_fractional_bits(w, h))


def scale_for(w: int, h: int) -> float:
    return float(lib().sfo_scale_for(w, h))


def mask_pack(mask_bytes, w: int, h: int):
    mb = _c(mask_bytes, np.uint8).reshape(-1)
    wpr = (w + 31) // 32
    bits = np.zeros(wpr * h, np.uint32)
    fg = lib().sfo_mask_pack(_p(mb), w, h, _p(bits))
    return bits, wpr, int(fg)


def responsibility(cam: Camera, w: int, h: int, attributes, sh, sh_per_ch: int, prep=None):
    if prep is None:
        prep = prepare(cam, w, h, attributes, sh, sh_per_ch)
    return rasterize(prep, 1, scale=scale_for(w, h))["resp"]


def evidence(prep: dict, mask_bytes):
    w, h = prep["w"], prep["h"]
    bits, wpr, _ = mask_pack(mask_bytes, w, h)
    out = rasterize(prep, 2, scale=scale_for(w, h), mask_bits=bits, words_per_row=wpr)
    return out["fg"], out["bg"]


def lgamma(x):
    return lib().sfo_lgamma(float(x))


def digamma(x):
    return lib().sfo_digamma(float(x))


def beta_entropy(a, b):
    return lib().sfo_beta_entropy(float(a), float(b))


_TABLE = None


def entropy_table():
    global _TABLE
    if _TABLE is None:
        t = np.empty(445 * 445, np.float32)
        lib().sfo_entropy_table(_p(t))
        _TABLE = t
    return _TABLE


def table_entropy(a, b):
    t = entropy_table()
    return np.array([lib().sfo_table_entropy(float(x), float(y), _p(t)) for x, y in zip(a, b)],
                    np.float32)


def eig(a, b, resp, scale, mode=0):
    a = _c(a, np.float32)
    b = _c(b, np.float32)
    resp = _c(resp, np.uint32)
    t = entropy_table()
    return float(lib().sfo_eig(mode, _p(a), _p(b), _p(resp), len(a), scale, _p(t)))


def beta_update(a, b, fg, bg, scale):
    a = np.array(a, np.float32)
    b = np.array(b, np.float32)
    fg = _c(fg, np.uint32)
    bg = _c(bg, np.uint32)
    lib().sfo_beta_update(scale, _p(fg), _p(bg), _p(a), _p(b), len(a))
    return a, b


def render64(cam: Camera, w: int, h: int, attributes, sh, sh_per_ch: int):
    attributes = _c(attributes, np.float64)
    sh = _c(sh, np.float64)
    n = attributes.size // 11
    out = np.empty(h * w * 4, np.float64)
    lib().sfo64_render(C.byref(cam), w, h, _p(attributes), _p(sh), n, sh_per_ch, _p(out))
    return out.reshape(h, w, 4)


def render64_backward(cam: Camera, w: int, h: int, attributes, sh, sh_per_ch: int, dl_drgba):
    """dL/d(attributes), dL/d(sh) of L = sum(dl_drgba * rgba) (dl_drgba [h, w, 4];
    a [h, w, 3] array is taken as zero gradient on alpha)."""
    attributes = _c(attributes, np.float64)
    sh = _c(sh, np.float64)
    dl = np.asarray(dl_drgba, np.float64)
    if dl.shape[-1] == 3:
        dl = np.concatenate([dl, np.zeros(dl.shape[:-1] + (1,))], axis=-1)
    dl = _c(dl, np.float64)
    n = attributes.size // 11
    d_attr = np.empty(11 * n, np.float64)
    d_sh = np.empty(3 * sh_per_ch * n, np.float64)
    lib().sfo64_render_backward(C.byref(cam), w, h, _p(attributes), _p(sh), n, sh_per_ch, _p(dl),
                                _p(d_attr), _p(d_sh))
    return d_attr, d_sh


class ProbeLoss:
    """FP64 L2 loss of the forward against a target image over a tile region,
    with one parameter of one splat replaced (sfo64_probe_*): central
    differences on scenes too large to render whole per probe. Parameters:
    0..10 the attribute planes, 11 + k*3 + c the SH coefficient (k, c)."""

    def __init__(self, cam: Camera, w: int, h: int, attributes, sh, sh_per_ch: int, target_rgba):
        self.attr = _c(attributes, np.float64)
        self.sh = _c(sh, np.float64)
        self.n = self.attr.size // 11
        self.w, self.h = w, h
        target = _c(target_rgba, np.float64)
        assert target.size == 4 * w * h
        self.handle = lib().sfo64_probe_open(C.byref(cam), w, h, _p(self.attr), _p(self.sh), self.n, sh_per_ch,
                                             _p(target))

    def bbox(self, i: int):
        """(visible, (min_x, min_y, max_x, max_y)) tile box of splat i."""
        out = np.zeros(2, np.uint32)
        vis = lib().sfo64_probe_bbox(self.handle, i, _p(out))
        return bool(vis), (int(out[0] & 0xFFFF), int(out[0] >> 16), int(out[1] & 0xFFFF), int(out[1] >> 16))

    def base_value(self, i: int, param: int) -> float:
        if param < 11:
            return float(self.attr[param * self.n + i])
        return float(self.sh[(param - 11) * self.n + i])

    def loss(self, i: int, param: int, value: float, region) -> float:
        tx0, ty0, tx1, ty1 = region
        return float(lib().sfo64_probe_loss(self.handle, i, param, value, tx0, ty0, tx1, ty1))

    def close(self):
        if getattr(self, "handle", None):
            lib().sfo64_probe_close(self.handle)
            self.handle = None

    def __del__(self):
        self.close()


def num_threads() -> int:
    return int(lib().sfo_num_threads())


def set_num_threads(n: int) -> None:
    lib().sfo_set_num_threads(int(n))
