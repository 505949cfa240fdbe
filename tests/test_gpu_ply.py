"""The CUDA PLY loader (device transpose of the stored rows) against the
oracle's parse_ply restatement, bit for bit, and a render of a loaded scene
against the same scene uploaded from planes (GPU)."""
import numpy as np
import pytest

import splatfield_b200 as sf
from oracle import ply as oply
from splatfield_b200 import synth

from test_ply import synthetic_ply

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("extra", [[], ["f_rest_0", "f_rest_2", "f_rest_1"],
                                   [f"f_rest_{j}" for j in (5, 0, 8, 1, 7, 2, 6, 3, 4)],
                                   [f"f_rest_{j}" for j in range(44, -1, -1)] + ["nx", "ny", "nz"]])
def test_loader_planes_match_oracle_parse(ctx, extra):
    data = synthetic_ply(37, extra)
    want_attr, want_sh = oply.parse_ply(data)
    splats = sf.load_ply(data)
    attr, sh = splats.read_planes()
    np.testing.assert_array_equal(attr.view(np.uint32), want_attr.view(np.uint32))
    np.testing.assert_array_equal(sh.view(np.uint32), want_sh.view(np.uint32))
    pos = want_attr.reshape(11, -1)[:3]
    np.testing.assert_array_equal(splats.bounds[0], pos.min(1))
    np.testing.assert_array_equal(splats.bounds[1], pos.max(1))


def test_loaded_scene_renders_like_uploaded_planes(ctx, tmp_path):
    attr, sh = synth.scene_uniform(20000, 16, 21)
    # Stored rotations are unit quaternions (write_ply's contract).
    a = attr.reshape(11, -1)
    q = a[3:7] / np.linalg.norm(a[3:7], axis=0)
    a[3:7] = q
    path = tmp_path / "scene.ply"
    path.write_bytes(sf.CpuSplats(attr, sh).write_ply())
    loaded = sf.load_ply(path)
    want_attr, want_sh = oply.parse_ply(path.read_bytes())
    got_attr, got_sh = loaded.read_planes()
    np.testing.assert_array_equal(got_attr.view(np.uint32), want_attr.view(np.uint32))
    direct = sf.Splats(want_attr, want_sh)
    cam = sf.look_at((0.0, 0.0, -3.0), (0.0, 0.0, 0.0))
    img_a = loaded.render_with(sf.RenderScratch(20000, (160, 120)), cam, (160, 120)).read()
    img_b = direct.render_with(sf.RenderScratch(20000, (160, 120)), cam, (160, 120)).read()
    np.testing.assert_array_equal(img_a, img_b)


def test_two_coefficient_scene_renders_dc_only(ctx, oracle_mod):
    """3 f_rest (1 per channel): the reference's `chs >= 4` test leaves them
    unread; the loaded scene renders like the oracle on the same planes."""
    n = 2000
    attr, sh1 = synth.scene_uniform(n, 1, 23)
    extra = np.random.default_rng(0).normal(0, 0.3, (3, n)).astype(np.float32)
    sh = np.concatenate([sh1.reshape(3, n), extra]).reshape(-1)
    splats = sf.Splats(attr, sh)
    assert splats.sh_per_ch == 2
    cam = sf.look_at((0.0, 0.0, -3.0), (0.0, 0.0, 0.0))
    got = splats.render_with(sf.RenderScratch(n, (96, 96)), cam, (96, 96)).read()
    cam_o = oracle_mod.look_at((0.0, 0.0, -3.0), (0.0, 0.0, 0.0))
    prep = oracle_mod.prepare(cam_o, 96, 96, attr, sh, 2)
    np.testing.assert_array_equal(got, oracle_mod.rasterize(prep, 0)["bitmap"])
