"""Paint ops over the shared scene (src/seg/paint.rs) and their reference
tests (src/seg/tests.rs:313-470): the posterior heatmap (also bit-exact
against the oracle with the projected colours replaced by m), the
foreground tint, and the DC snapshot / restore (GPU)."""
import numpy as np
import pytest

import splatfield_b200 as sf
from splatfield_b200 import segment as seg
from splatfield_b200 import synth

from helpers import opaque, row_positions, zero_sh

pytestmark = pytest.mark.gpu

SH_C0 = 0.2820948


def to_dc(color):
    return [(c - 0.5) / SH_C0 for c in color]


def test_render_posterior_ignores_size_mismatch(ctx):
    splats = sf.Splats(opaque(row_positions(2, 2.0, 1.0)), zero_sh(2))
    scratch = sf.RenderScratch(2, (64, 64))
    stale = sf.BetaState.from_host(np.array([2, 1, 3], np.float32), np.array([1, 3, 1], np.float32))
    a = splats.render_posterior(scratch, stale, sf.camera_default(), (64, 64)).read()
    b = splats.render_with(scratch, sf.camera_default(), (64, 64)).read()
    np.testing.assert_array_equal(a, b)


def test_posterior_heatmap_is_grayscale(ctx):
    splats = sf.Splats(opaque(row_positions(2, 2.0, 1.0)), zero_sh(2))
    scratch = sf.RenderScratch(2, (64, 64))
    beta = sf.BetaState.from_host(np.array([3, 1], np.float32), np.array([1, 3], np.float32))
    words = splats.render_posterior(scratch, beta, sf.camera_default(), (64, 64)).read()
    rgb = seg.bitmap_to_rgb(words, 64).reshape(64, 64, 3)
    assert np.all(rgb[..., 0] == rgb[..., 1]) and np.all(rgb[..., 1] == rgb[..., 2])
    assert rgb[:, :32, 0].max() > rgb[:, 32:, 0].max()


def test_posterior_heatmap_bit_exact_vs_oracle(ctx, oracle_mod):
    O = oracle_mod
    n, w, h = 30000, 200, 150
    attr, sh = synth.scene_uniform(n, 4, 41)
    a, b = synth.beta_posterior(n, seed=41)
    splats = sf.Splats(attr, sh)
    beta = sf.BetaState.from_host(a, b)
    cam = sf.look_at((0.0, 0.0, -3.0), (0.0, 0.0, 0.0))
    got = splats.render_posterior(sf.RenderScratch(n, (w, h)), beta, cam, (w, h)).read()
    prep = O.prepare(O.look_at((0.0, 0.0, -3.0), (0.0, 0.0, 0.0)), w, h, attr, sh, 4)
    m = (a / (a + b)).astype(np.float32)
    prep["projected"][:, 5] = m
    prep["projected"][:, 6] = m
    prep["projected"][:, 7] = m
    np.testing.assert_array_equal(got, O.rasterize(prep, 0)["bitmap"])


def center_rgb(splats, scratch):
    words = splats.render_with(scratch, sf.camera_default(), (64, 64)).read()
    rgb = seg.bitmap_to_rgb(words, 64)
    p = (32 * 64 + 32) * 3
    return [int(v) for v in rgb[p:p + 3]]


def test_tint_is_visible_in_next_render(ctx):
    splats = sf.Splats(opaque([(0.0, 0.0, 5.0)]), zero_sh(1))
    scratch = sf.RenderScratch(1, (64, 64))
    before = center_rgb(splats, scratch)
    beta = sf.BetaState.from_host(np.array([2.0], np.float32), np.array([1.0], np.float32))
    splats.tint(beta, to_dc([0.937, 0.267, 0.267]))
    after = center_rgb(splats, scratch)
    assert after[0] > before[0] + 40 and after[1] < before[1] - 10 and after[2] < before[2] - 10


def test_save_colors_roundtrips_dc_of_high_degree_sh(ctx):
    n, k = 3, 2
    attr = opaque([(0.0, 0.0, 2.0 + i) for i in range(n)])
    planes = 3 * k
    sh = np.array([1.0 + c * n + i for c in range(planes) for i in range(n)], np.float32)
    splats = sf.Splats(attr, sh)
    early = splats.save_colors()
    np.testing.assert_array_equal(early.read(), sh[:3 * n])
    splats.tint(sf.BetaState.from_host(np.array([2, 1, 3], np.float32), np.array([1, 3, 1], np.float32)),
                [1.0, 0.0, 0.0])
    saved = splats.save_colors()
    splats.tint(sf.BetaState.from_host(np.full(3, 2, np.float32), np.ones(3, np.float32)), [9.0, 9.0, 9.0])
    splats.restore_colors(saved)
    _, all_sh = splats.read_planes()
    for i in (0, 2):
        assert all_sh[i] == 1.0 and all_sh[n + i] == 0.0 and all_sh[2 * n + i] == 0.0
    for c in range(3):
        assert all_sh[c * n + 1] == sh[c * n + 1]
    np.testing.assert_array_equal(all_sh[3 * n:], sh[3 * n:])
    np.testing.assert_array_equal(early.read(), sh[:3 * n])
