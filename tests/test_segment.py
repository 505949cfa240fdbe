"""Host logic of the active loop (src/seg/views.rs, src/seg/active.rs): the
candidate sphere, the bitmap unpack, the sphere oracle, config validation.
No GPU."""
import math

import numpy as np
import pytest

import splatfield_b200 as sf
from splatfield_b200 import segment as seg


def rotate(cam, v):
    return seg.quat_rotate(np.array(cam.rotation, np.float32), np.asarray(v, np.float32)[None, :])[0]


def test_candidates_on_sphere_looking_at_center(built_lib):
    """views.rs:276-309."""
    loc = seg.ObjectLocalization(np.array([1.0, 2.0, 3.0], np.float32), 0.5)
    want = 1.5 * 0.5 / math.tan(seg.CANDIDATE_FOV * 0.5)
    cams = seg.candidates(loc, 20)
    assert len(cams) == 20
    zs = []
    for k, cam in enumerate(cams):
        off = np.array(cam.position, np.float32) - loc.center
        assert abs(np.linalg.norm(off) - want) < 1e-4, k
        fwd = rotate(cam, [0, 0, 1])
        fwd = fwd / np.linalg.norm(fwd)
        assert fwd @ (-off / np.linalg.norm(off)) > 1 - 1e-4, k
        zs.append((off / np.linalg.norm(off))[2])
    assert all(a > b for a, b in zip(zs, zs[1:])), "fibonacci z must decrease"


def test_candidates_clamp_degenerate_radius(built_lib):
    """views.rs:206-232 (the candidate half): r = 0 is lifted to 1e-3."""
    loc = seg.ObjectLocalization(np.array([2.0, -1.0, 0.5], np.float32), 0.0)
    want = 1.5 * 1e-3 / math.tan(seg.CANDIDATE_FOV * 0.5)
    for cam in seg.candidates(loc, 5):
        off = np.array(cam.position, np.float32) - loc.center
        assert abs(np.linalg.norm(off) - want) < 1e-6
        assert np.all(np.isfinite(cam.position)) and np.all(np.isfinite(rotate(cam, [0, 0, 1])))


def test_bitmap_to_rgb_handles_row_padding():
    """active.rs:266-292."""
    words = np.array([[0x04030201, 0x08070605, 0x0C0B0A09, 0xDEADBEEF, 0xDEADBEEF],
                      [0x14131211, 0x18171615, 0x1C1B1A19, 0xDEADBEEF, 0xDEADBEEF]], np.uint32)
    want = [b for b in list(range(1, 13)) + list(range(17, 29)) if b % 4 != 0]
    assert seg.bitmap_to_rgb(words, 3).tolist() == want


def test_sphere_oracle_marks_ray_hits(built_lib):
    cam = sf.look_at((0.0, 0.0, -3.0), (0.0, 0.0, 0.0))
    mask = seg.sphere_oracle([((0.0, 0.0, 0.0), 0.5)])(None, (64, 48), cam).reshape(48, 64)
    assert mask[24, 32] == 1 and mask[0, 0] == 0 and mask[47, 63] == 0
    # A sphere behind the camera is never hit; one around it always is.
    assert seg.sphere_oracle([((0.0, 0.0, -6.0), 0.5)])(None, (16, 16), cam).sum() == 0
    assert seg.sphere_oracle([((0.0, 0.0, -3.0), 1.0)])(None, (16, 16), cam).all()


def test_empty_sphere_set_is_blind(built_lib):
    cam = sf.look_at((0.0, 0.0, -3.0), (0.0, 0.0, 0.0))
    assert seg.sphere_oracle([])(None, (32, 32), cam).sum() == 0


def test_frame_bounds_pulls_back_along_minus_y(built_lib):
    cam = seg.frame_bounds(((-1.0, -2.0, 0.0), (3.0, 2.0, 1.0)))
    np.testing.assert_allclose(cam.position, [1.0, -8.0, 0.5])
    fwd = rotate(cam, [0, 0, 1])
    np.testing.assert_allclose(fwd, [0.0, 1.0, 0.0], atol=1e-6)


@pytest.mark.parametrize("cfg", [seg.Config(256, 0, 2), seg.Config(8, 12, 2), seg.Config(256, 12, 0)])
def test_segmenter_rejects_invalid_config(cfg):
    """active.rs:318-351: validated before any GPU allocation."""
    with pytest.raises(ValueError):
        seg.Segmenter(None, cfg, sf.camera_default())
