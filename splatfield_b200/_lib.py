"""ctypes binding of libsplatfield_b200.so (the C ABI in include/splatfield_cuda.h).

The library is built in-tree by ``splatfield_b200.build``; importing this
module never falls back to anything else: a missing library raises.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libsplatfield_b200.so")

SF_OK, SF_ERR_ARG, SF_ERR_SHAPE, SF_ERR_CAPACITY, SF_ERR_TIMEOUT, SF_ERR_CUDA, SF_ERR_NOMEM = range(7)
ERROR_NAMES = {
    SF_ERR_ARG: "SF_ERR_ARG",
    SF_ERR_SHAPE: "SF_ERR_SHAPE",
    SF_ERR_CAPACITY: "SF_ERR_CAPACITY",
    SF_ERR_TIMEOUT: "SF_ERR_TIMEOUT",
    SF_ERR_CUDA: "SF_ERR_CUDA",
    SF_ERR_NOMEM: "SF_ERR_NOMEM",
}

# sf_scratch_read fields
READ_DEPTH_KEYS, READ_TILE_COUNTS, READ_BBOX, READ_PROJECTED, READ_ORDER, READ_OFFSETS = range(6)
READ_TILE_IDS, READ_GAUSSIAN_IDS, READ_TILE_START, READ_BITMAP, READ_RGBA, READ_FINAL_T, READ_N_CONTRIB = range(6, 13)

EIG_LUT_F32, EIG_FP64 = 0, 1
ROUND_RESPONSIBILITY, ROUND_EVIDENCE, ROUND_ADJOINT = 0, 1, 2
ISECTS_BINNED, ISECTS_DEPTH_SORTED = 0, 1
ORDER_SORTED, ORDER_IN_RASTER, ORDER_HYBRID = 0, 1, 2
SCHEDULE_LONGEST, SCHEDULE_TILES = 0, 1


class SplatfieldError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{ERROR_NAMES.get(code, code)}: {msg}")
        self.code = code


class Camera(C.Structure):
    """Camera{fov, position, rotation} (src/camera.rs:5-9); rotation x, y, z, w."""

    _fields_ = [("fov", C.c_float * 2), ("position", C.c_float * 3), ("rotation", C.c_float * 4)]


class View(C.Structure):
    _fields_ = [
        ("rot0", C.c_float * 3), ("rot1", C.c_float * 3), ("rot2", C.c_float * 3),
        ("trans", C.c_float * 3), ("focal", C.c_float * 2), ("world_pos", C.c_float * 3),
        ("img", C.c_float * 2), ("tile_bounds", C.c_float * 2),
    ]


class Tuning(C.Structure):
    """sf_tuning: kernel forms of a scratch (results are identical across forms)."""

    _fields_ = [("raster_cull", C.c_uint32), ("isect_build", C.c_uint32), ("raster_detail", C.c_uint32),
                ("raster_order", C.c_uint32), ("raster_schedule", C.c_uint32), ("raster_split", C.c_uint32),
                ("radix_bits", C.c_uint32), ("frame_pipes", C.c_uint32)]


class RoundTuning(C.Structure):
    """sf_round_tuning."""

    _fields_ = [("lanes", C.c_uint32), ("raster_cull", C.c_uint32), ("isect_build", C.c_uint32),
                ("raster_order", C.c_uint32), ("raster_split", C.c_uint32), ("radix_bits", C.c_uint32),
                ("reserved", C.c_uint32 * 2)]


class Isects(C.Structure):
    """TileIsects (src/render.rs:463-471)."""

    _fields_ = [
        ("tile_ids", C.c_void_p), ("gaussian_ids", C.c_void_p), ("tile_start", C.c_void_p),
        ("num_isects", C.c_uint32), ("num_visible", C.c_uint32),
        ("tile_bounds", C.c_uint32 * 2), ("row_stride", C.c_uint32),
    ]


_lib = None


_P, _u32, _i32, _sz = C.c_void_p, C.c_uint32, C.c_int, C.c_size_t
_PP = C.POINTER(C.c_void_p)
P, u32, i32, sz, PP = _P, _u32, _i32, _sz, _PP
# name -> (restype, argtypes): every entry point of include/splatfield_cuda.h
SIGNATURES = {
        "sf_last_error": (C.c_char_p, []),
        "sf_abi_version": (i32, []),
        "sf_kernel_launches": (C.c_uint64, []),
        "sf_ctx_create": (i32, [i32, PP]),
        "sf_ctx_destroy": (i32, [P]),
        "sf_buffer_alloc": (i32, [P, sz, PP]),
        "sf_buffer_free": (i32, [P, P]),
        "sf_memcpy_htod": (i32, [P, P, sz, P]),
        "sf_memcpy_dtoh": (i32, [P, P, sz, P]),
        "sf_memset": (i32, [P, i32, sz, P]),
        "sf_stream_sync": (i32, [P]),
        "sf_host_alloc": (i32, [sz, PP]),
        "sf_host_free": (i32, [P]),
        "sf_camera_look_at": (i32, [P, P, P]),
        "sf_camera_focal": (i32, [P, u32, u32, P]),
        "sf_view_for_camera": (i32, [P, u32, u32, P]),
        "sf_splats_create": (i32, [P, P, P, u32, u32, PP]),
        "sf_splats_destroy": (i32, [P]),
        "sf_splats_info": (i32, [P, P, P, P, PP, PP]),
        "sf_scratch_create": (i32, [P, u32, u32, u32, PP]),
        "sf_scratch_destroy": (i32, [P]),
        "sf_scratch_capacity": (i32, [P, P]),
        "sf_scratch_set_tuning": (i32, [P, P]),
        "sf_scratch_get_tuning": (i32, [P, P]),
        "sf_render_with": (i32, [P, P, P, u32, u32, P, PP, P]),
        "sf_render_posterior": (i32, [P, P, P, P, u32, u32, P, PP, P]),
        "sf_splats_tint": (i32, [P, P, C.c_float, C.c_float, C.c_float, P]),
        "sf_splats_save_colors": (i32, [P, P, P]),
        "sf_splats_restore_colors": (i32, [P, P, P]),
        "sf_render_float": (i32, [P, P, P, u32, u32, P, PP]),
        "sf_render_to_host": (i32, [P, P, P, u32, u32, P, P]),
        "sf_render_frames_to_host": (i32, [P, P, P, u32, u32, u32, P, P]),
        "sf_render_frames": (i32, [P, P, P, u32, u32, u32, P]),
        "sf_scratch_reserve": (i32, [P, C.c_uint64]),
        "sf_render_forward": (i32, [P, P, P, u32, u32, P, PP]),
        "sf_render_backward": (i32, [P, P, P, u32, u32, P, P, P, P, P]),
        "sf_prepare_isects": (i32, [P, P, P, u32, u32, P, P]),
        "sf_finalize_rgb": (i32, [P, P, P, u32, u32, i32, P]),
        "sf_scratch_buffers": (i32, [P, PP, PP, P]),
        "sf_scratch_stats": (i32, [P, P, P]),
        "sf_scratch_read": (i32, [P, i32, P, sz, P]),
        "sf_accum_create": (i32, [P, u32, PP]),
        "sf_accum_destroy": (i32, [P]),
        "sf_accum_info": (i32, [P, P, PP, PP, PP]),
        "sf_accum_set_scale": (i32, [P, C.c_float]),
        "sf_mask_create": (i32, [P, u32, u32, P, PP, P]),
        "sf_mask_create_packed": (i32, [P, u32, u32, P, PP]),
        "sf_mask_destroy": (i32, [P]),
        "sf_render_responsibility": (i32, [P, P, P, P, u32, u32, P]),
        "sf_accumulate_prepared": (i32, [P, P, P, u32, u32, P, P, P]),
        "sf_fractional_bits": (u32, [u32, u32]),
        "sf_beta_create_uniform": (i32, [P, u32, PP]),
        "sf_beta_create": (i32, [P, P, P, u32, PP]),
        "sf_beta_destroy": (i32, [P]),
        "sf_beta_read": (i32, [P, P, P, P]),
        "sf_beta_info": (i32, [P, P, PP, PP]),
        "sf_beta_eig": (i32, [P, P, i32, P, P]),
        "sf_beta_eig_async": (i32, [P, P, i32, P, P]),
        "sf_beta_update": (i32, [P, P, P]),
        "sf_localize": (i32, [P, P, P, P, P, P]),
        "sf_map_labels": (i32, [P, P, u32, P]),
        "sf_entropy_table": (i32, [P]),
        "sf_table_entropy": (i32, [P, P, P, u32, P, P]),
        "sf_round_create": (i32, [P, u32, u32, P, P, PP]),
        "sf_round_destroy": (i32, [P]),
        "sf_round_set_tuning": (i32, [P, P]),
        "sf_round_get_tuning": (i32, [P, P]),
        "sf_round_eig": (i32, [P, P, P, P, i32, P, P]),
        "sf_round_responsibility": (i32, [P, u32, PP, P, P, P]),
        "sf_round_evidence": (i32, [P, P, P, P, P, i32, P, P]),
        "sf_round_evidence_words": (i32, [P, u32, PP, PP]),
        "sf_round_autotune": (i32, [P, P, P, P, i32, P, P, P]),
        "sf_ply_inspect": (i32, [P, sz, P, P]),
        "sf_ply_load": (i32, [P, P, sz, PP]),
        "sf_ply_load_file": (i32, [P, C.c_char_p, PP]),
        "sf_ply_write": (i32, [P, P, u32, u32, P, sz, P]),
        "sf_bits_for": (u32, [u32]),
        "sf_radix_create": (i32, [P, u32, PP]),
        "sf_radix_destroy": (i32, [P]),
        "sf_radix_argsort": (i32, [P, P, P, u32, u32, i32, P, PP, PP]),
        "sf_radix_argsort_async": (i32, [P, P, P, u32, u32, i32, P, PP, PP]),
        "sf_radix_status": (i32, [P, P]),
        "sf_radix_set_digit_bits": (i32, [P, u32]),
        "sf_scan_create": (i32, [P, u32, PP]),
        "sf_scan_destroy": (i32, [P]),
        "sf_exclusive_scan_gather": (i32, [P, P, P, P, u32, P]),
        "sf_exclusive_scan_gather_async": (i32, [P, P, P, P, u32, P]),
        "sf_scan_status": (i32, [P, P]),
        "sf_exclusive_scan": (i32, [P, P, u32, P]),
        "sf_exclusive_scan_gather_noalloc": (i32, [P, P, P, u32, P]),
        "sf_debug_lookback": (i32, [u32, i32]),
        "sf_debug_giant_lists": (i32, [u32]),
        "sf_scratch_autotune": (i32, [P, P, P, u32, u32, u32, P, P, P]),
        "sf_sog_inspect": (i32, [P, sz, P, P]),
        "sf_sog_load": (i32, [P, P, sz, PP]),
        "sf_sog_load_file": (i32, [P, C.c_char_p, PP]),
        "sf_webp_decode": (i32, [P, sz, P, P, P, sz]),
        "sf_render_feature_adjoint": (i32, [P, P, P, u32, u32, P, P, P, P]),
        "sf_beta_eig_real": (i32, [P, P, P, i32, P, P]),
        "sf_beta_update_real": (i32, [P, P, P, P]),
        "sf_round_evidence_adjoint": (i32, [P, P, P, P, P, i32, P, P]),
        "sf_round_adjoint_responsibility": (i32, [P, u32, PP, PP]),
        "sf_round_autotune_kind": (i32, [P, P, P, P, P, i32, i32, P, P, P]),
}
del P, u32, i32, sz, PP


def _declare(L):
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args


def lib():
    """The loaded library; raises if it was not built (no fallback path)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"{LIB_PATH} is missing: build it with `python -m splatfield_b200.build` "
                "(the CUDA path has no fallback)")
        L = C.CDLL(LIB_PATH)
        _declare(L)
        _lib = L
    return _lib


def check(rc: int) -> None:
    if rc != SF_OK:
        msg = lib().sf_last_error()
        raise SplatfieldError(rc, msg.decode() if msg else "")
