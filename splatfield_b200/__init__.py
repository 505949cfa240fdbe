"""B200 (sm_100a) splat render + segmentation-evidence path.

A drop-in for the GPU path of suous/splatfield: projection, onesweep depth and
tile sorts, decoupled-look-back scans, the tile rasterizer (RGBA8, float,
responsibility and mask-evidence modes), the Beta-Bernoulli EIG (f32 LUT and
FP64) and the Beta update, all as hand-written CUDA behind the C ABI in
include/splatfield_cuda.h. This package is the Python host side over that
ABI (ctypes); it has no CPU fallback.
"""
from .core import *  # noqa: F401,F403
from .core import make_camera, quat_from_rotation_y  # noqa: F401
from . import segment  # noqa: F401

__version__ = "0.1.0"
