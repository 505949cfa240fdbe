"""Host-side mirror of the reference's Rust API over the C ABI.

Names follow suous/splatfield v0.2.0: ``CpuSplats.upload`` / ``Splats``
(src/render.rs:25-269), ``RenderScratch`` (:116-198), ``Splats.render_with``
(:371-380), ``prepare_isects`` / ``finalize`` (:274-460), ``Camera``
(src/camera.rs:5-63), ``Accumulators`` / ``Mask`` / ``render_responsibility``
/ ``accumulate_prepared`` (src/seg/mod.rs:52-210), ``BetaState`` /
``map_labels`` (src/seg/beta.rs:215-297), ``RadixScratch`` / ``bits_for``
(crates/sort/src/sort.rs:259-381), ``ScanScratch`` / ``exclusive_scan_gather``
(crates/sort/src/scan.rs:49-255). Errors the reference raises by panicking
(zero splats, undersized scratch) raise ``SplatfieldError`` here.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from . import _lib as L
from ._lib import Camera, Isects, SplatfieldError, View, check, lib

__all__ = [
    "Camera", "View", "Isects", "SplatfieldError", "Context", "default_context", "DeviceBuffer",
    "DeviceView", "camera_default", "look_at", "focal", "view_for_camera", "CpuSplats", "Splats",
    "RenderScratch", "TileIsects", "Accumulators", "Mask", "BetaState", "map_labels", "bits_for",
    "RadixScratch", "ScanScratch", "exclusive_scan_gather", "exclusive_scan_buf", "entropy_table",
    "table_entropy", "fractional_bits", "row_stride_for", "EIG_LUT_F32", "EIG_FP64", "Round",
    "ISECTS_BINNED", "ISECTS_DEPTH_SORTED", "ORDER_IN_RASTER", "ORDER_SORTED", "ORDER_HYBRID", "SCHEDULE_LONGEST", "SCHEDULE_TILES", "ply_inspect", "load_ply", "sog_inspect", "load_sog", "webp_decode",
    "pinned_empty", "ROUND_RESPONSIBILITY", "ROUND_EVIDENCE", "ROUND_ADJOINT",
]

EIG_LUT_F32, EIG_FP64 = L.EIG_LUT_F32, L.EIG_FP64
ISECTS_BINNED, ISECTS_DEPTH_SORTED = L.ISECTS_BINNED, L.ISECTS_DEPTH_SORTED
ORDER_IN_RASTER, ORDER_SORTED, ORDER_HYBRID = L.ORDER_IN_RASTER, L.ORDER_SORTED, L.ORDER_HYBRID
SCHEDULE_TILES, SCHEDULE_LONGEST = L.SCHEDULE_TILES, L.SCHEDULE_LONGEST
ROUND_RESPONSIBILITY, ROUND_EVIDENCE, ROUND_ADJOINT = L.ROUND_RESPONSIBILITY, L.ROUND_EVIDENCE, L.ROUND_ADJOINT
BASE_FOV = 0.8  # Camera::BASE_FOV (src/camera.rs:86)


class _PinnedOwner:
    """Frees one sf_host_alloc block when the last array viewing it goes."""

    def __init__(self, nbytes: int):
        p = C.c_void_p()
        check(lib().sf_host_alloc(max(nbytes, 1), C.byref(p)))
        self.ptr = p

    def __del__(self):
        if self.ptr is not None:
            try:
                lib().sf_host_free(self.ptr)
            except Exception:  # interpreter shutdown
                pass
            self.ptr = None


class _PinnedArray(np.ndarray):
    _pin = None

    def __array_finalize__(self, obj):
        self._pin = getattr(obj, "_pin", None)


def pinned_empty(shape, dtype=np.uint32) -> np.ndarray:
    """An uninitialised array in page-locked host memory (copies to and from
    it run asynchronously); the memory lives as long as the array or any view
    of it."""
    dtype = np.dtype(dtype)
    shape = tuple(int(x) for x in (shape if isinstance(shape, (tuple, list)) else (shape,)))
    nbytes = int(np.prod(shape, dtype=np.int64)) * dtype.itemsize
    owner = _PinnedOwner(nbytes)
    raw = (C.c_uint8 * max(nbytes, 1)).from_address(owner.ptr.value)
    arr = np.frombuffer(raw, np.uint8, nbytes).view(dtype).reshape(shape).view(_PinnedArray)
    arr._pin = owner
    return arr


def _vp(x) -> C.c_void_p:
    if x is None:
        return None
    if isinstance(x, (DeviceBuffer, DeviceView)):
        return C.c_void_p(x.ptr)
    if isinstance(x, int):
        return C.c_void_p(x)
    if isinstance(x, np.ndarray):
        return x.ctypes.data_as(C.c_void_p)
    raise TypeError(type(x))


def _stream(stream) -> C.c_void_p:
    if stream is None:
        return None
    if isinstance(stream, int):
        return C.c_void_p(stream)
    # torch.cuda.Stream and friends
    return C.c_void_p(int(getattr(stream, "cuda_stream")))


class Context:
    """One CUDA device; owns the entropy LUT."""

    def __init__(self, device: int = 0):
        h = C.c_void_p()
        check(lib().sf_ctx_create(device, C.byref(h)))
        self.handle = h
        self.device = device

    def close(self):
        if self.handle:
            lib().sf_ctx_destroy(self.handle)
            self.handle = None


_DEFAULT: Context | None = None


def default_context() -> Context:
    global _DEFAULT
    if _DEFAULT is None:
        _DEFAULT = Context(0)
    return _DEFAULT


class DeviceView:
    """A non-owning view of device memory returned by the library (it aliases
    a handle's storage, like the reference's returned GpuTensors)."""

    def __init__(self, ptr: int, dtype, shape, keepalive=None):
        self.ptr = int(ptr or 0)
        self.dtype = np.dtype(dtype)
        self.shape = tuple(shape)
        self._keep = keepalive

    @property
    def nbytes(self) -> int:
        return int(np.prod(self.shape)) * self.dtype.itemsize

    def read(self, stream=None) -> np.ndarray:
        """Blocking read-back (GpuTensor::read_vec)."""
        out = np.empty(self.shape, self.dtype)
        if out.nbytes:
            check(lib().sf_memcpy_dtoh(_vp(out), C.c_void_p(self.ptr), out.nbytes, _stream(stream)))
        return out


class DeviceBuffer(DeviceView):
    """An owned device allocation."""

    def __init__(self, nbytes_or_array, dtype=np.uint32, ctx: Context | None = None, shape=None):
        self.ctx = ctx or default_context()
        if isinstance(nbytes_or_array, np.ndarray):
            arr = np.ascontiguousarray(nbytes_or_array)
            dtype, shape, nbytes = arr.dtype, arr.shape, arr.nbytes
        else:
            nbytes = int(nbytes_or_array)
            arr = None
            dtype = np.dtype(dtype)
            shape = shape or (nbytes // dtype.itemsize,)
        p = C.c_void_p()
        check(lib().sf_buffer_alloc(self.ctx.handle, max(nbytes, 1), C.byref(p)))
        super().__init__(p.value, dtype, shape)
        if arr is not None and arr.nbytes:
            self.write(arr)

    @classmethod
    def from_array(cls, arr, ctx: Context | None = None) -> "DeviceBuffer":
        return cls(np.ascontiguousarray(arr), ctx=ctx)

    @classmethod
    def empty(cls, count: int, dtype=np.uint32, ctx: Context | None = None) -> "DeviceBuffer":
        dt = np.dtype(dtype)
        return cls(count * dt.itemsize, dt, ctx, shape=(count,))

    def write(self, arr: np.ndarray, stream=None) -> None:
        arr = np.ascontiguousarray(arr)
        check(lib().sf_memcpy_htod(C.c_void_p(self.ptr), _vp(arr), arr.nbytes, _stream(stream)))
        check(lib().sf_stream_sync(_stream(stream)))

    def fill_zero(self, stream=None) -> None:
        check(lib().sf_memset(C.c_void_p(self.ptr), 0, self.nbytes, _stream(stream)))

    def free(self):
        if self.ptr:
            lib().sf_buffer_free(self.ctx.handle, C.c_void_p(self.ptr))
            self.ptr = 0

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


# ------------------------------------------------------------------ camera

def camera_default() -> Camera:
    """Camera::default (src/camera.rs:72-80)."""
    return make_camera()


def make_camera(fov=(BASE_FOV, BASE_FOV), position=(0.0, 0.0, 0.0), rotation=(0.0, 0.0, 0.0, 1.0)) -> Camera:
    c = Camera()
    c.fov[:] = [float(v) for v in fov]
    c.position[:] = [float(v) for v in position]
    c.rotation[:] = [float(v) for v in rotation]
    return c


def quat_from_rotation_y(angle: float):
    h = np.float32(angle) * np.float32(0.5)
    return (0.0, float(np.sin(h, dtype=np.float32)), 0.0, float(np.cos(h, dtype=np.float32)))


def look_at(position, target) -> Camera:
    """Camera::look_at (src/camera.rs:57-63)."""
    out = Camera()
    p = np.ascontiguousarray(position, np.float32)
    t = np.ascontiguousarray(target, np.float32)
    check(lib().sf_camera_look_at(_vp(p), _vp(t), C.byref(out)))
    return out


def focal(cam: Camera, w: int, h: int):
    out = np.empty(2, np.float32)
    check(lib().sf_camera_focal(C.byref(cam), w, h, _vp(out)))
    return out


def view_for_camera(cam: Camera, w: int, h: int) -> View:
    v = View()
    check(lib().sf_view_for_camera(C.byref(cam), w, h, C.byref(v)))
    return v


def row_stride_for(w: int) -> int:
    return ((4 * w + 255) // 256 * 256) // 4


# ------------------------------------------------------------------ splats

def ply_inspect(data: bytes):
    """parse_ply's header checks (src/ply.rs:9-77): (vertex count, SH
    coefficients per channel); raises SplatfieldError with the reference's
    messages."""
    buf = np.frombuffer(data, np.uint8)
    n, k = C.c_uint32(), C.c_uint32()
    check(lib().sf_ply_inspect(_vp(buf) if buf.size else None, buf.size, C.byref(n), C.byref(k)))
    return int(n.value), int(k.value)


def load_ply(source, ctx: Context | None = None) -> "Splats":
    """parse_ply + upload (src/ply.rs:9-112): a path or the file's bytes."""
    ctx = ctx or default_context()
    h = C.c_void_p()
    if isinstance(source, (bytes, bytearray, memoryview)):
        buf = np.frombuffer(bytes(source), np.uint8)
        check(lib().sf_ply_load(ctx.handle, _vp(buf) if buf.size else None, buf.size, C.byref(h)))
    else:
        check(lib().sf_ply_load_file(ctx.handle, str(source).encode(), C.byref(h)))
    return Splats._adopt(h, ctx)


def sog_inspect(data: bytes):
    """parse_sog's meta.json checks (src/sog.rs:97-108, 151-159): (splat
    count, SH coefficients per channel); raises SplatfieldError with the
    reference's messages."""
    buf = np.frombuffer(bytes(data), np.uint8)
    n, k = C.c_uint32(), C.c_uint32()
    check(lib().sf_sog_inspect(_vp(buf) if buf.size else None, buf.size, C.byref(n), C.byref(k)))
    return int(n.value), int(k.value)


def load_sog(source, ctx: Context | None = None) -> "Splats":
    """parse_sog + upload (src/sog.rs:97-198): a path or the archive's bytes."""
    ctx = ctx or default_context()
    h = C.c_void_p()
    if isinstance(source, (bytes, bytearray, memoryview)):
        buf = np.frombuffer(bytes(source), np.uint8)
        check(lib().sf_sog_load(ctx.handle, _vp(buf) if buf.size else None, buf.size, C.byref(h)))
    else:
        check(lib().sf_sog_load_file(ctx.handle, str(source).encode(), C.byref(h)))
    return Splats._adopt(h, ctx)


def webp_decode(data: bytes) -> np.ndarray:
    """The lossless WebP decoder of the SOG loader: RGBA8 pixels [h, w, 4]."""
    buf = np.frombuffer(bytes(data), np.uint8)
    w, h = C.c_uint32(), C.c_uint32()
    check(lib().sf_webp_decode(_vp(buf), buf.size, C.byref(w), C.byref(h), None, 0))
    out = np.zeros((h.value, w.value, 4), np.uint8)
    check(lib().sf_webp_decode(_vp(buf), buf.size, C.byref(w), C.byref(h), _vp(out), out.size))
    return out


class CpuSplats:
    """Host splat payload, field-major (src/render.rs:20-28)."""

    def __init__(self, attributes, sh_coeffs):
        self.attributes = np.ascontiguousarray(attributes, np.float32).reshape(-1)
        self.sh_coeffs = np.ascontiguousarray(sh_coeffs, np.float32).reshape(-1)

    def count(self) -> int:
        return self.attributes.size // 11

    def upload(self, ctx: Context | None = None) -> "Splats":
        return Splats(self.attributes, self.sh_coeffs, ctx)

    def write_ply(self) -> bytes:
        """CpuSplats::write_ply (src/ply.rs:115-180): binary little-endian 3DGS PLY."""
        n = self.count()
        k = self.sh_coeffs.size // max(3 * n, 1) if n else 0
        ln = C.c_size_t()
        check(lib().sf_ply_write(_vp(self.attributes), _vp(self.sh_coeffs), n, k, None, 0, C.byref(ln)))
        out = np.empty(ln.value, np.uint8)
        check(lib().sf_ply_write(_vp(self.attributes), _vp(self.sh_coeffs), n, k, _vp(out), out.size,
                                 C.byref(ln)))
        return out.tobytes()


class Splats:
    """GPU splats (Splats::new, src/render.rs:242-269)."""

    def __init__(self, attributes, sh_coeffs, ctx: Context | None = None):
        self.ctx = ctx or default_context()
        attributes = np.ascontiguousarray(attributes, np.float32).reshape(-1)
        sh_coeffs = np.ascontiguousarray(sh_coeffs, np.float32).reshape(-1)
        n = attributes.size // 11
        k = sh_coeffs.size // max(3 * n, 1) if n else 1
        h = C.c_void_p()
        check(lib().sf_splats_create(self.ctx.handle, _vp(attributes), _vp(sh_coeffs), n, k, C.byref(h)))
        self.handle = h
        self.n = n
        self.sh_per_ch = k
        b = np.empty(6, np.float32)
        check(lib().sf_splats_info(h, None, None, _vp(b), None, None))
        self.bounds = (b[:3].copy(), b[3:].copy())
        self.positions = attributes[: 3 * n].copy()

    @classmethod
    def _adopt(cls, handle, ctx: Context) -> "Splats":
        """Wraps a handle the library created (e.g. by the PLY loader)."""
        self = cls.__new__(cls)
        self.ctx = ctx
        self.handle = handle
        n, k = C.c_uint32(), C.c_uint32()
        b = np.empty(6, np.float32)
        check(lib().sf_splats_info(handle, C.byref(n), C.byref(k), _vp(b), None, None))
        self.n, self.sh_per_ch = int(n.value), int(k.value)
        self.bounds = (b[:3].copy(), b[3:].copy())
        self.positions = self.read_planes()[0][: 3 * self.n].copy()
        return self

    def read_planes(self):
        """Host copies of the device planes: (attributes [11 n], sh [3 k n])."""
        pa, ps = C.c_void_p(), C.c_void_p()
        check(lib().sf_splats_info(self.handle, None, None, None, C.byref(pa), C.byref(ps)))
        attr = DeviceView(pa.value, np.float32, (11 * self.n,), self).read()
        sh = DeviceView(ps.value, np.float32, (3 * self.sh_per_ch * self.n,), self).read()
        return attr, sh

    def close(self):
        if getattr(self, "handle", None):
            lib().sf_splats_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- render paths
    def render_with(self, scratch: "RenderScratch", camera: Camera, img_size, stream=None) -> DeviceView:
        w, h = img_size
        ptr = C.c_void_p()
        rs = C.c_uint32()
        check(lib().sf_render_with(self.handle, scratch.handle, C.byref(camera), w, h, _stream(stream),
                                   C.byref(ptr), C.byref(rs)))
        return DeviceView(ptr.value, np.uint32, (h, rs.value), scratch)

    def render_posterior(self, scratch: "RenderScratch", beta: "BetaState", camera: Camera, img_size,
                         stream=None) -> DeviceView:
        """Posterior-mean heatmap frame (src/seg/paint.rs:22-47)."""
        w, h = img_size
        ptr = C.c_void_p()
        rs = C.c_uint32()
        check(lib().sf_render_posterior(self.handle, scratch.handle, beta.handle if beta else None,
                                        C.byref(camera), w, h, _stream(stream), C.byref(ptr), C.byref(rs)))
        return DeviceView(ptr.value, np.uint32, (h, rs.value), scratch)

    def tint(self, beta: "BetaState", color, stream=None) -> None:
        """DC colour of the foreground splats (src/seg/paint.rs:49-66)."""
        r, g, b = (float(c) for c in color)
        check(lib().sf_splats_tint(self.handle, beta.handle, r, g, b, _stream(stream)))

    def save_colors(self, stream=None) -> "DeviceBuffer":
        """Device snapshot of the DC planes [3, n] (src/seg/paint.rs:68-75)."""
        buf = DeviceBuffer.empty(3 * self.n, np.float32, self.ctx)
        check(lib().sf_splats_save_colors(self.handle, C.c_void_p(buf.ptr), _stream(stream)))
        return buf

    def restore_colors(self, saved: "DeviceView", stream=None) -> None:
        check(lib().sf_splats_restore_colors(self.handle, C.c_void_p(saved.ptr), _stream(stream)))

    def render_float(self, scratch: "RenderScratch", camera: Camera, img_size, stream=None) -> DeviceView:
        w, h = img_size
        ptr = C.c_void_p()
        check(lib().sf_render_float(self.handle, scratch.handle, C.byref(camera), w, h, _stream(stream),
                                    C.byref(ptr)))
        return DeviceView(ptr.value, np.float32, (h, w, 4), scratch)

    def render_forward(self, scratch: "RenderScratch", camera: Camera, img_size, stream=None) -> DeviceView:
        """Float RGBA frame that keeps the per-pixel state render_backward replays."""
        w, h = img_size
        ptr = C.c_void_p()
        check(lib().sf_render_forward(self.handle, scratch.handle, C.byref(camera), w, h, _stream(stream),
                                      C.byref(ptr)))
        return DeviceView(ptr.value, np.float32, (h, w, 4), scratch)

    def render_backward(self, scratch: "RenderScratch", camera: Camera, img_size, dl_drgba,
                        want_proj: bool = False, stream=None):
        """dL/d(attributes) [11, n] and dL/d(sh) [K, 3, n] (field-major) for
        L = sum(dl_drgba * rgba) of the last render_forward; with want_proj also
        the per-splat 2D adjoint [n, 9] (mean2d xy, conic xyz, rgb, opacity)."""
        w, h = img_size
        dl = dl_drgba if isinstance(dl_drgba, DeviceView) else DeviceBuffer.from_array(
            np.ascontiguousarray(dl_drgba, np.float32).reshape(h, w, 4), self.ctx)
        d_attr = DeviceBuffer.empty(11 * self.n, np.float32, self.ctx)
        d_sh = DeviceBuffer.empty(3 * self.sh_per_ch * self.n, np.float32, self.ctx)
        d_proj = DeviceBuffer.empty(9 * self.n, np.float32, self.ctx) if want_proj else None
        check(lib().sf_render_backward(self.handle, scratch.handle, C.byref(camera), w, h, _vp(dl),
                                       _vp(d_attr), _vp(d_sh), _vp(d_proj), _stream(stream)))
        out = (d_attr.read().reshape(11, self.n), d_sh.read().reshape(self.sh_per_ch, 3, self.n))
        if want_proj:
            out = out + (d_proj.read().reshape(self.n, 9),)
        return out

    def render_feature_adjoint(self, scratch: "RenderScratch", camera: Camera, img_size, mask: "Mask | None" = None,
                               stream=None, out=None):
        """Real-valued (fg, bg) responsibilities [n] from the adjoint of a
        per-splat scalar feature (fg weighted by the mask, bg by its
        complement; no mask: all in fg), as device buffers (new ones, or the
        pair `out`)."""
        w, h = img_size
        if out is not None:
            fg, bg = out
        else:
            fg = DeviceBuffer.empty(self.n, np.float32, self.ctx)
            bg = DeviceBuffer.empty(self.n, np.float32, self.ctx)
        check(lib().sf_render_feature_adjoint(self.handle, scratch.handle, C.byref(camera), w, h,
                                              mask.handle if mask is not None else None, _stream(stream),
                                              _vp(fg), _vp(bg)))
        return fg, bg

    def render_backward_into(self, scratch: "RenderScratch", camera: Camera, img_size, dl_drgba,
                             d_attr, d_sh, d_proj=None, stream=None) -> None:
        """render_backward into caller-owned device buffers; enqueues only."""
        w, h = img_size
        check(lib().sf_render_backward(self.handle, scratch.handle, C.byref(camera), w, h, _vp(dl_drgba),
                                       _vp(d_attr), _vp(d_sh), _vp(d_proj), _stream(stream)))

    def render_to_host(self, scratch: "RenderScratch", camera: Camera, img_size, out=None, stream=None):
        w, h = img_size
        if out is None:
            out = np.empty((h, w), np.uint32)
        check(lib().sf_render_to_host(self.handle, scratch.handle, C.byref(camera), w, h, _stream(stream),
                                      _vp(out)))
        return out

    def render_frames(self, scratch: "RenderScratch", cameras, img_size, stream=None) -> DeviceView:
        """``len(cameras)`` frames enqueued back to back with one sync at the
        end; returns the last frame's image (device view, [h][row_stride])."""
        w, h = img_size
        cams = (Camera * len(cameras))(*cameras)
        check(lib().sf_render_frames(self.handle, scratch.handle, cams, len(cameras), w, h, _stream(stream)))
        return DeviceView(scratch.bitmap_ptr(), np.uint32, (h, row_stride_for(w)), scratch)

    def render_frames_to_host(self, scratch: "RenderScratch", cameras, img_size, out=None, stream=None):
        """One RGBA8 image per camera, [count, h, w] words in host memory
        (``out``: pinned memory lets each image's read-back overlap the next
        frame; see ``pinned_empty``)."""
        w, h = img_size
        cams = (Camera * len(cameras))(*cameras)
        if out is None:
            out = np.empty((len(cameras), h, w), np.uint32)
        if out.dtype != np.uint32 or not out.flags.c_contiguous or out.size < len(cameras) * w * h:
            raise ValueError("out must be a C-contiguous uint32 array of count * h * w words")
        check(lib().sf_render_frames_to_host(self.handle, scratch.handle, cams, len(cameras), w, h,
                                             _stream(stream), _vp(out)))
        return out

    def prepare_isects(self, scratch: "RenderScratch", camera: Camera, img_size, stream=None) -> "TileIsects":
        w, h = img_size
        out = Isects()
        check(lib().sf_prepare_isects(self.handle, scratch.handle, C.byref(camera), w, h, _stream(stream),
                                      C.byref(out)))
        return TileIsects(out, scratch)

    def finalize_rgb(self, scratch: "RenderScratch", isects: "TileIsects", img_size, want_float=False,
                     stream=None) -> DeviceView:
        w, h = img_size
        check(lib().sf_finalize_rgb(self.handle, scratch.handle, C.byref(isects.raw), w, h,
                                    1 if want_float else 0, _stream(stream)))
        return DeviceView(scratch.bitmap_ptr(), np.uint32, (h, isects.raw.row_stride), scratch)

    def render_responsibility(self, scratch: "RenderScratch", acc: "Accumulators", camera: Camera, img_size,
                              stream=None) -> None:
        w, h = img_size
        check(lib().sf_render_responsibility(self.handle, scratch.handle, acc.handle, C.byref(camera), w, h,
                                             _stream(stream)))
        acc._sync_scale()

    def accumulate_prepared(self, scratch: "RenderScratch", isects: "TileIsects", img_size,
                            acc: "Accumulators", mask: "Mask | None" = None, stream=None) -> None:
        w, h = img_size
        check(lib().sf_accumulate_prepared(self.handle, scratch.handle, C.byref(isects.raw), w, h,
                                           acc.handle, mask.handle if mask else None, _stream(stream)))
        acc._sync_scale()


class TileIsects:
    def __init__(self, raw: Isects, scratch):
        self.raw = raw
        self._scratch = scratch

    @property
    def num_isects(self) -> int:
        return int(self.raw.num_isects)

    @property
    def num_visible(self) -> int:
        return int(self.raw.num_visible)

    @property
    def tile_bounds(self):
        return (int(self.raw.tile_bounds[0]), int(self.raw.tile_bounds[1]))

    def tile_ids(self) -> DeviceView:
        return DeviceView(self.raw.tile_ids, np.uint32, (self.num_isects,), self._scratch)

    def gaussian_ids(self) -> DeviceView:
        return DeviceView(self.raw.gaussian_ids, np.uint32, (self.num_isects,), self._scratch)


class RenderScratch:
    """Per-frame buffers (RenderScratch::new, src/render.rs:144-167)."""

    def __init__(self, total: int, img_size, ctx: Context | None = None):
        self.ctx = ctx or default_context()
        w, h = img_size
        hd = C.c_void_p()
        check(lib().sf_scratch_create(self.ctx.handle, total, w, h, C.byref(hd)))
        self.handle = hd

    def capacity(self) -> int:
        c = C.c_uint64()
        check(lib().sf_scratch_capacity(self.handle, C.byref(c)))
        return int(c.value)

    def reserve(self, isects: int) -> None:
        """Grow the intersection capacity to at least ``isects`` up front."""
        check(lib().sf_scratch_reserve(self.handle, int(isects)))

    def set_tuning(self, raster_cull: int = 0, isect_build: int = L.ISECTS_BINNED, raster_detail: int = 0,
                   raster_order: int = L.ORDER_SORTED, raster_schedule: int = L.SCHEDULE_LONGEST,
                   raster_split: int = 1, radix_bits: int = 8, frame_pipes: int = 2) -> None:
        """Kernel forms (results are identical across forms): raster_cull 0/1,
        isect_build ISECTS_BINNED (default) or ISECTS_DEPTH_SORTED,
        raster_detail 1 to count the per-pair diagnostics of ``stats``,
        raster_order ORDER_SORTED (default), ORDER_IN_RASTER or ORDER_HYBRID,
        raster_schedule SCHEDULE_LONGEST (default) or SCHEDULE_TILES,
        raster_split 1 (default), 2 or 4 rasterizer CTAs per tile,
        radix_bits 4..8 (default 8) digit width of the depth-sorted build,
        frame_pipes 2 (default) or 1 frame pipes of the camera-path calls."""
        t = L.Tuning()
        t.raster_cull = int(raster_cull)
        t.isect_build = int(isect_build)
        t.raster_detail = int(raster_detail)
        t.raster_order = int(raster_order)
        t.raster_schedule = int(raster_schedule)
        t.raster_split = int(raster_split)
        t.radix_bits = int(radix_bits)
        t.frame_pipes = int(frame_pipes)
        check(lib().sf_scratch_set_tuning(self.handle, C.byref(t)))

    def autotune(self, splats: "Splats", cameras, img_size, stream=None) -> tuple:
        """Pick the raster form by measured time on a camera path (same images
        in every form); returns (tuning, ms per frame)."""
        w, h = img_size
        arr = (Camera * len(cameras))(*cameras)
        t = L.Tuning()
        ms = C.c_double()
        check(lib().sf_scratch_autotune(splats.handle, self.handle, arr, len(cameras), w, h, _stream(stream),
                                        C.byref(t), C.byref(ms)))
        return self.get_tuning(), float(ms.value)

    def get_tuning(self) -> dict:
        t = L.Tuning()
        check(lib().sf_scratch_get_tuning(self.handle, C.byref(t)))
        return {"raster_cull": int(t.raster_cull), "isect_build": int(t.isect_build),
                "raster_detail": int(t.raster_detail), "raster_order": int(t.raster_order),
                "raster_schedule": int(t.raster_schedule), "raster_split": int(t.raster_split) or 1,
                "radix_bits": int(t.radix_bits) or 8, "frame_pipes": int(t.frame_pipes) or 2}

    def read(self, what: int, count: int, dtype=np.uint32, stream=None) -> np.ndarray:
        out = np.empty(count, dtype)
        check(lib().sf_scratch_read(self.handle, what, _vp(out), out.nbytes, _stream(stream)))
        return out

    def stats(self, stream=None) -> dict:
        """Pair statistics of the last rasterization on this scratch."""
        out = np.zeros(4, np.uint64)
        check(lib().sf_scratch_stats(self.handle, _vp(out), _stream(stream)))
        return dict(pairs_visited=int(out[0]), exp_evaluated=int(out[1]), contributing=int(out[2]),
                    pairs_processed=int(out[3]))

    def bitmap_ptr(self) -> int:
        b = C.c_void_p()
        check(lib().sf_scratch_buffers(self.handle, C.byref(b), None, None))
        return b.value

    def rgba_ptr(self) -> int:
        r = C.c_void_p()
        check(lib().sf_scratch_buffers(self.handle, None, C.byref(r), None))
        return r.value

    def close(self):
        if getattr(self, "handle", None):
            lib().sf_scratch_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ------------------------------------------------------------ segmentation

def fractional_bits(w: int, h: int) -> int:
    return int(lib().sf_fractional_bits(w, h))


class Accumulators:
    """u32 fixed-point eps / fg / bg per splat (src/seg/mod.rs:52-85)."""

    def __init__(self, total: int, ctx: Context | None = None):
        self.ctx = ctx or default_context()
        h = C.c_void_p()
        check(lib().sf_accum_create(self.ctx.handle, total, C.byref(h)))
        self.handle = h
        self.total = total
        self.scale = 1.0
        self._ptrs()

    def _ptrs(self):
        s = C.c_float()
        r, f, b = C.c_void_p(), C.c_void_p(), C.c_void_p()
        check(lib().sf_accum_info(self.handle, C.byref(s), C.byref(r), C.byref(f), C.byref(b)))
        self.scale = float(s.value)
        self.bits = DeviceView(r.value, np.uint32, (self.total,), self)
        self.fg = DeviceView(f.value, np.uint32, (self.total,), self)
        self.bg = DeviceView(b.value, np.uint32, (self.total,), self)

    def _sync_scale(self):
        s = C.c_float()
        check(lib().sf_accum_info(self.handle, C.byref(s), None, None, None))
        self.scale = float(s.value)

    def set_scale(self, scale: float) -> None:
        check(lib().sf_accum_set_scale(self.handle, float(scale)))
        self.scale = float(scale)

    def write_bits(self, bits) -> None:
        """Overwrite the total-responsibility words (host array of total u32)."""
        b = np.ascontiguousarray(bits, np.uint32)
        if b.size != self.total:
            raise SplatfieldError(L.SF_ERR_SHAPE, "bits length must equal the accumulator size")
        check(lib().sf_memcpy_htod(C.c_void_p(self.bits.ptr), _vp(b), b.nbytes, None))
        check(lib().sf_stream_sync(None))

    @classmethod
    def from_eps(cls, eps, scale: float, ctx: "Context | None" = None) -> "Accumulators":
        """An accumulator holding trunc(eps * scale) at `scale` (the reference
        tests' eps_acc, src/seg/beta.rs:351-359)."""
        bits = (np.asarray(eps, np.float32) * np.float32(scale)).astype(np.uint32)
        acc = cls(bits.size, ctx)
        acc.write_bits(bits)
        acc.set_scale(scale)
        return acc

    def read_f32(self) -> np.ndarray:
        return self.bits.read().astype(np.float32) / np.float32(self.scale)

    def read_evidence_f32(self):
        s = np.float32(self.scale)
        return self.fg.read().astype(np.float32) / s, self.bg.read().astype(np.float32) / s

    def close(self):
        if getattr(self, "handle", None):
            lib().sf_accum_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Mask:
    """Bit-packed binary mask (src/seg/mod.rs:105-144)."""

    def __init__(self, handle, size, fg_pixels: int):
        self.handle = handle
        self.size = tuple(size)
        self.words_per_row = (size[0] + 31) // 32
        self.fg_pixels = fg_pixels

    @classmethod
    def from_bytes(cls, size, data, ctx: Context | None = None) -> "Mask":
        ctx = ctx or default_context()
        w, h = size
        b = np.ascontiguousarray(data, np.uint8).reshape(-1)
        if b.size != w * h:
            raise SplatfieldError(L.SF_ERR_SHAPE, "mask bytes must be one per pixel")
        hd = C.c_void_p()
        fg = C.c_uint32()
        check(lib().sf_mask_create(ctx.handle, w, h, _vp(b), C.byref(hd), C.byref(fg)))
        return cls(hd, size, int(fg.value))

    @classmethod
    def from_words(cls, size, words, ctx: Context | None = None) -> "Mask":
        ctx = ctx or default_context()
        w, h = size
        wd = np.ascontiguousarray(words, np.uint32).reshape(-1)
        hd = C.c_void_p()
        check(lib().sf_mask_create_packed(ctx.handle, w, h, _vp(wd), C.byref(hd)))
        return cls(hd, size, int(sum(bin(int(x)).count("1") for x in wd)))

    def close(self):
        if getattr(self, "handle", None):
            lib().sf_mask_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class BetaState:
    """Per-splat Beta(a, b) posteriors (src/seg/beta.rs:215-287)."""

    def __init__(self, handle, n: int, ctx: Context):
        self.handle = handle
        self.n = n
        self.ctx = ctx

    @classmethod
    def new_uniform(cls, total: int, ctx: Context | None = None) -> "BetaState":
        ctx = ctx or default_context()
        h = C.c_void_p()
        check(lib().sf_beta_create_uniform(ctx.handle, total, C.byref(h)))
        return cls(h, total, ctx)

    @classmethod
    def from_host(cls, a, b, ctx: Context | None = None) -> "BetaState":
        ctx = ctx or default_context()
        a = np.ascontiguousarray(a, np.float32)
        b = np.ascontiguousarray(b, np.float32)
        h = C.c_void_p()
        check(lib().sf_beta_create(ctx.handle, _vp(a), _vp(b), a.size, C.byref(h)))
        return cls(h, a.size, ctx)

    def eig(self, acc: Accumulators, mode: int = EIG_LUT_F32, stream=None) -> float:
        out = C.c_double()
        check(lib().sf_beta_eig(self.handle, acc.handle, mode, _stream(stream), C.byref(out)))
        return float(out.value)

    def update(self, acc: Accumulators, stream=None) -> None:
        check(lib().sf_beta_update(self.handle, acc.handle, _stream(stream)))

    def eig_real(self, fg, bg=None, mode: int = EIG_LUT_F32, stream=None) -> float:
        """EIG over real-valued responsibilities eps = fg + bg (device arrays)."""
        out = C.c_double()
        check(lib().sf_beta_eig_real(self.handle, _vp(fg), _vp(bg), mode, _stream(stream), C.byref(out)))
        return float(out.value)

    def update_real(self, fg, bg, stream=None) -> None:
        """a += fg, b += bg (device arrays of real-valued responsibilities)."""
        check(lib().sf_beta_update_real(self.handle, _vp(fg), _vp(bg), _stream(stream)))

    def read(self, stream=None):
        a = np.empty(self.n, np.float32)
        b = np.empty(self.n, np.float32)
        check(lib().sf_beta_read(self.handle, _vp(a), _vp(b), _stream(stream)))
        return a, b

    def close(self):
        if getattr(self, "handle", None):
            lib().sf_beta_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def map_labels(a, b) -> np.ndarray:
    """MAP foreground labels a > b (src/seg/beta.rs:294-297)."""
    a = np.ascontiguousarray(a, np.float32)
    b = np.ascontiguousarray(b, np.float32)
    if a.size != b.size:
        raise SplatfieldError(L.SF_ERR_SHAPE, "posterior length mismatch")
    out = np.empty(a.size, np.uint8)
    check(lib().sf_map_labels(_vp(a), _vp(b), a.size, _vp(out)))
    return out.astype(bool)


def entropy_table() -> np.ndarray:
    t = np.empty(445 * 445, np.float32)
    check(lib().sf_entropy_table(_vp(t)))
    return t


def table_entropy(a, b, ctx: Context | None = None) -> np.ndarray:
    """The probe of the LUT lookup the EIG kernel uses (src/seg/beta.rs:336-342)."""
    ctx = ctx or default_context()
    da = DeviceBuffer.from_array(np.asarray(a, np.float32), ctx)
    db = DeviceBuffer.from_array(np.asarray(b, np.float32), ctx)
    out = DeviceBuffer.empty(da.shape[0], np.float32, ctx)
    check(lib().sf_table_entropy(ctx.handle, _vp(da), _vp(db), da.shape[0], _vp(out), None))
    return out.read()


# ------------------------------------------------------------ batched round

class Round:
    """Every candidate view of a segmentation round scored in one CUDA graph
    (the batched Segmenter::select_view, src/seg/active.rs:113-129)."""

    def __init__(self, total: int, sizes, ctx: Context | None = None):
        self.ctx = ctx or default_context()
        sizes = [(int(w), int(h)) for w, h in sizes]
        ws = np.array([s[0] for s in sizes], np.uint32)
        hs = np.array([s[1] for s in sizes], np.uint32)
        hd = C.c_void_p()
        check(lib().sf_round_create(self.ctx.handle, total, len(sizes), _vp(ws), _vp(hs), C.byref(hd)))
        self.handle = hd
        self.total = total
        self.sizes = sizes

    @property
    def views(self) -> int:
        return len(self.sizes)

    def set_tuning(self, lanes: int = 4, raster_cull: int = 0, isect_build: int = L.ISECTS_BINNED,
                   raster_order: int = L.ORDER_SORTED, raster_split: int = 1, radix_bits: int = 8) -> None:
        t = L.RoundTuning()
        t.lanes, t.raster_cull, t.isect_build = int(lanes), int(raster_cull), int(isect_build)
        t.raster_order = int(raster_order)
        t.raster_split = int(raster_split)
        t.radix_bits = int(radix_bits)
        check(lib().sf_round_set_tuning(self.handle, C.byref(t)))

    @staticmethod
    def _tuning_dict(t) -> dict:
        return {"lanes": int(t.lanes), "raster_cull": int(t.raster_cull), "isect_build": int(t.isect_build),
                "raster_order": int(t.raster_order), "raster_split": int(t.raster_split) or 1,
                "radix_bits": int(t.radix_bits) or 8}

    def get_tuning(self) -> dict:
        t = L.RoundTuning()
        check(lib().sf_round_get_tuning(self.handle, C.byref(t)))
        return self._tuning_dict(t)

    @staticmethod
    def _cams(cameras):
        arr = (Camera * len(cameras))()
        for i, c in enumerate(cameras):
            arr[i] = c
        return arr

    def eig(self, splats: Splats, beta: "BetaState | None", cameras, mode: int = EIG_LUT_F32,
            stream=None) -> np.ndarray:
        """Responsibility of every view and (with a posterior) its EIG."""
        if len(cameras) != self.views:
            raise SplatfieldError(L.SF_ERR_SHAPE, "one camera per view")
        out = np.zeros(self.views, np.float64)
        check(lib().sf_round_eig(self.handle, splats.handle, beta.handle if beta else None,
                                 self._cams(cameras), mode, _stream(stream), _vp(out)))
        return out

    def evidence(self, splats: Splats, beta: "BetaState | None", cameras, masks, mode: int = EIG_LUT_F32,
                 stream=None) -> np.ndarray:
        """Masked evidence of every view (fg / bg words, read with
        ``evidence_words``) and, with a posterior, each view's EIG."""
        if len(cameras) != self.views or len(masks) != self.views:
            raise SplatfieldError(L.SF_ERR_SHAPE, "one camera and one mask per view")
        hs = (C.c_void_p * self.views)(*[m.handle for m in masks])
        self._masks = list(masks)  # the graph holds their device words
        out = np.zeros(self.views, np.float64)
        check(lib().sf_round_evidence(self.handle, splats.handle, beta.handle if beta else None,
                                      self._cams(cameras), hs, mode, _stream(stream), _vp(out)))
        return out

    def evidence_adjoint(self, splats: Splats, beta: "BetaState | None", cameras, masks=None,
                         mode: int = EIG_LUT_F32, stream=None) -> np.ndarray:
        """Every view's real-valued (fg, bg) responsibilities from the adjoint
        of a per-splat scalar feature (read with ``adjoint_responsibility``)
        and, with a posterior, each view's EIG over fg + bg."""
        if len(cameras) != self.views or (masks is not None and len(masks) != self.views):
            raise SplatfieldError(L.SF_ERR_SHAPE, "one camera (and mask) per view")
        hs = None
        if masks is not None:
            hs = (C.c_void_p * self.views)(*[m.handle if m is not None else None for m in masks])
            self._masks = list(masks)
        out = np.zeros(self.views, np.float64)
        check(lib().sf_round_evidence_adjoint(self.handle, splats.handle, beta.handle if beta else None,
                                              self._cams(cameras), hs, mode, _stream(stream), _vp(out)))
        return out

    def adjoint_responsibility(self, view: int) -> tuple:
        """(fg, bg) device floats of a view of the last adjoint round."""
        fg, bg = C.c_void_p(), C.c_void_p()
        check(lib().sf_round_adjoint_responsibility(self.handle, view, C.byref(fg), C.byref(bg)))
        return (DeviceView(fg.value, np.float32, (self.total,), self),
                DeviceView(bg.value, np.float32, (self.total,), self))

    def evidence_words(self, view: int) -> tuple:
        """(fg, bg) device words of a view of the last evidence round."""
        fg, bg = C.c_void_p(), C.c_void_p()
        check(lib().sf_round_evidence_words(self.handle, view, C.byref(fg), C.byref(bg)))
        return (DeviceView(fg.value, np.uint32, (self.total,), self),
                DeviceView(bg.value, np.uint32, (self.total,), self))

    def responsibility(self, view: int) -> tuple:
        """(device words, scale, intersections, visible) of a view of the last round."""
        p = C.c_void_p()
        scale = C.c_float()
        nis = C.c_uint64()
        vis = C.c_uint32()
        check(lib().sf_round_responsibility(self.handle, view, C.byref(p), C.byref(scale), C.byref(nis),
                                            C.byref(vis)))
        return DeviceView(p.value, np.uint32, (self.total,), self), float(scale.value), int(nis.value), int(vis.value)

    def autotune(self, splats: Splats, beta: "BetaState | None", cameras, mode: int = EIG_LUT_F32,
                 stream=None, kind: int = L.ROUND_RESPONSIBILITY, masks=None) -> tuple:
        """Pick the round's kernel forms by measured time for rounds of
        `kind` (ROUND_RESPONSIBILITY, ROUND_EVIDENCE with masks, or
        ROUND_ADJOINT); returns (tuning, best ms per round)."""
        t = L.RoundTuning()
        ms = C.c_double()
        hs = None
        if masks is not None:
            hs = (C.c_void_p * self.views)(*[m.handle if m is not None else None for m in masks])
            self._masks = list(masks)
        check(lib().sf_round_autotune_kind(self.handle, splats.handle, beta.handle if beta else None,
                                           self._cams(cameras), hs, int(kind), mode, _stream(stream), C.byref(t),
                                           C.byref(ms)))
        return self._tuning_dict(t), float(ms.value)

    def close(self):
        if getattr(self, "handle", None):
            lib().sf_round_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ------------------------------------------------------------- sort / scan

def bits_for(max_exclusive: int) -> int:
    """bits_for (crates/sort/src/sort.rs:259-261)."""
    return int(lib().sf_bits_for(int(max_exclusive) & 0xFFFFFFFF))


class RadixScratch:
    """Onesweep radix scratch (RadixScratch, crates/sort/src/sort.rs:282-381)."""

    def __init__(self, max_elems: int, ctx: Context | None = None):
        self.ctx = ctx or default_context()
        h = C.c_void_p()
        check(lib().sf_radix_create(self.ctx.handle, max_elems, C.byref(h)))
        self.handle = h
        self.max = max_elems

    def set_digit_bits(self, digit_bits: int) -> None:
        """Digit width of the passes, 4..8 bits (default 8)."""
        check(lib().sf_radix_set_digit_bits(self.handle, int(digit_bits)))

    def argsort(self, keys, vals, n: int, bits: int, write_keys: bool = True, stream=None, sync: bool = True):
        """Sorted (keys, values) views into the scratch. sync=False only
        enqueues the sort (sf_radix_argsort_async); ``status`` then reports a
        timed-out look-back wait of any sort since the last check."""
        ko, vo = C.c_void_p(), C.c_void_p()
        fn = lib().sf_radix_argsort if sync else lib().sf_radix_argsort_async
        check(fn(self.handle, _vp(keys), _vp(vals), n, bits, 1 if write_keys else 0, _stream(stream),
                 C.byref(ko), C.byref(vo)))
        return DeviceView(ko.value, np.uint32, (n,), self), DeviceView(vo.value, np.uint32, (n,), self)

    def status(self, stream=None) -> None:
        """Waits for the stream; raises if a sort since the last check timed out."""
        check(lib().sf_radix_status(self.handle, _stream(stream)))

    def close(self):
        if getattr(self, "handle", None):
            lib().sf_radix_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class ScanScratch:
    """Decoupled look-back scan scratch (ScanScratch, crates/sort/src/scan.rs:49-60)."""

    def __init__(self, max_elems: int, ctx: Context | None = None):
        self.ctx = ctx or default_context()
        h = C.c_void_p()
        check(lib().sf_scan_create(self.ctx.handle, max_elems, C.byref(h)))
        self.handle = h

    def status(self, stream=None) -> None:
        """Waits for the stream; raises if a scan since the last check timed out."""
        check(lib().sf_scan_status(self.handle, _stream(stream)))

    def close(self):
        if getattr(self, "handle", None):
            lib().sf_scan_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def exclusive_scan_gather(gids, counts, offsets, n: int, scratch: ScanScratch, stream=None,
                          sync: bool = True) -> None:
    """offsets[i] = sum_{j<i} counts[gids[j]] (crates/sort/src/scan.rs:219-255).
    sync=False only enqueues the scan (``scratch.status`` checks it later)."""
    fn = lib().sf_exclusive_scan_gather if sync else lib().sf_exclusive_scan_gather_async
    check(fn(scratch.handle, _vp(gids), _vp(counts), _vp(offsets), n, _stream(stream)))


def exclusive_scan_buf(buf, n: int, scratch: ScanScratch, stream=None) -> None:
    check(lib().sf_exclusive_scan(scratch.handle, _vp(buf), n, _stream(stream)))
