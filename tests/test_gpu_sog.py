"""SOG scenes on the GPU: the planes the loader's device kernel writes
against the oracle's parse_sog (src/sog.rs:97-198) — bit for bit except the
two transcendental planes (means through expm1, opacity through ln), within
2 ulp — and a frame rendered from a loaded scene against the oracle's
render of the same planes."""
import os
import sys

import numpy as np
import pytest

import splatfield_b200 as sf

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
import make_sog_fixtures as M  # noqa: E402


def ulps(a, b):
    a = a.astype(np.float32).view(np.int32).astype(np.int64)
    b = b.astype(np.float32).view(np.int32).astype(np.int64)
    a = np.where(a < 0, -(a & 0x7FFFFFFF), a)
    b = np.where(b < 0, -(b & 0x7FFFFFFF), b)
    return np.abs(a - b)


@pytest.mark.parametrize("name", sorted(M.FIXTURES))
def test_loaded_planes_match_oracle(ctx, name):
    from oracle import sog as O

    path = os.path.join(HERE, "golden", name)
    data = open(path, "rb").read()
    n, bands, _ = M.FIXTURES[name]
    k = {0: 1, 1: 4, 3: 16}[bands]
    want_attr, want_sh = O.parse_sog(data)
    for splats in (sf.load_sog(data), sf.load_sog(path)):
        assert splats.n == n and splats.sh_per_ch == k
        attr, sh = splats.read_planes()
        attr, want = attr.reshape(11, n), want_attr.reshape(11, n)
        assert ulps(attr[0:3], want[0:3]).max() <= 2
        np.testing.assert_array_equal(attr[3:10].view(np.uint32), want[3:10].view(np.uint32))
        assert ulps(attr[10], want[10]).max() <= 2
        np.testing.assert_array_equal(sh.view(np.uint32), want_sh.view(np.uint32))


def test_loaded_scene_renders_as_the_oracle(ctx, oracle_mod):
    data = open(os.path.join(HERE, "golden", "sog_bands3.sog"), "rb").read()
    splats = sf.load_sog(data)
    attr, sh = splats.read_planes()
    w, h = 160, 120
    # Looking at the loaded scene's centre from outside its extent.
    means = attr.reshape(11, -1)[0:3].astype(np.float64)
    centre = means.mean(axis=1)
    extent = float(np.abs(means - centre[:, None]).max())
    pos = tuple(float(c) for c in centre + np.array([0.3, 0.2, -2.0 * extent - 1.0]))
    target = tuple(float(c) for c in centre)
    cam = sf.look_at(pos, target)
    got = splats.render_with(sf.RenderScratch(splats.n, (w, h)), cam, (w, h)).read()
    prep = oracle_mod.prepare(oracle_mod.look_at(pos, target), w, h, attr, sh, 16)
    np.testing.assert_array_equal(got, oracle_mod.rasterize(prep, 0)["bitmap"])
    assert prep["num_isects"] > 0
