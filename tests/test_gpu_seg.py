"""Responsibility, mask evidence, EIG and the Beta update on the GPU vs the
oracle and the reference's seg/beta tests (src/seg/tests.rs, src/seg/beta.rs)."""
import math

import numpy as np
import pytest

import splatfield_b200 as sf
from helpers import (known_answers, left_half_mask, opaque, overdraw_positions, row_positions,
                     stacked_positions, zero_sh)

pytestmark = pytest.mark.gpu

KA = known_answers()


def responsibility(attr, n, w, h, cam=None):
    splats = sf.Splats(attr, zero_sh(n))
    scratch = sf.RenderScratch(n, (w, h))
    acc = sf.Accumulators(n)
    splats.render_responsibility(scratch, acc, cam or sf.camera_default(), (w, h))
    return splats, scratch, acc


def test_eps_words_match_oracle_and_reference_golden(ctx, oracle_mod):
    """src/seg/tests.rs:185-203: bit-exact vs the oracle; the Metal golden
    within the oracle's stated tolerance."""
    _, _, acc = responsibility(opaque(overdraw_positions()), 40, 70, 70)
    got = acc.bits.read()
    want = oracle_mod.responsibility(oracle_mod.camera(), 70, 70, opaque(overdraw_positions()),
                                     zero_sh(40), 1)
    np.testing.assert_array_equal(got, want)
    golden = np.array(KA["eps_golden_overdraw"]["words"], np.int64)
    assert np.all(np.abs(got.astype(np.int64) - golden) <= 4 + 5e-7 * golden)
    assert acc.scale == 2.0 ** 19


def test_responsibility_is_bit_deterministic_across_renders(ctx):
    """src/seg/tests.rs:157-179."""
    splats, scratch, acc = responsibility(opaque(overdraw_positions()), 40, 70, 70)
    ref = acc.bits.read()
    assert np.any(ref > 0)
    for _ in range(7):
        splats.render_responsibility(scratch, acc, sf.camera_default(), (70, 70))
        np.testing.assert_array_equal(acc.bits.read(), ref)


def test_responsibility_conserves_pixel_weights(ctx):
    """src/seg/tests.rs:115-126."""
    attr = opaque(stacked_positions())
    splats = sf.Splats(attr, zero_sh(5))
    scratch = sf.RenderScratch(5, (64, 64))
    bm = splats.render_with(scratch, sf.camera_default(), (64, 64)).read()
    alpha_sum = float(((bm[:, :64] >> 24) & 255).sum()) / 255.0
    acc = sf.Accumulators(5)
    splats.render_responsibility(scratch, acc, sf.camera_default(), (64, 64))
    assert abs(alpha_sum - float(acc.read_f32().sum())) < 64 * 64 * 3 / 255.0


def test_responsibility_orders_depth_and_culls(ctx):
    """src/seg/tests.rs:130-150."""
    pos = [(0.0, 0.0, -3.0 if i == 5 else 1.0 + i * 0.5) for i in range(6)]
    _, _, acc = responsibility(opaque(pos), 6, 64, 64)
    eps = acc.read_f32()
    for k in range(4):
        assert eps[k] > eps[k + 1]
    assert eps[5] == 0.0


def split_scene():
    """split_scene (src/seg/tests.rs:95-110)."""
    size = (64, 64)
    splats = sf.Splats(opaque(row_positions(2, 2.0, 1.0)), zero_sh(2))
    scratch = sf.RenderScratch(2, size)
    acc = sf.Accumulators(2)
    splats.render_responsibility(scratch, acc, sf.camera_default(), size)
    mask = sf.Mask.from_bytes(size, left_half_mask(*size))
    isects = splats.prepare_isects(scratch, sf.camera_default(), size)
    splats.accumulate_prepared(scratch, isects, size, acc, mask)
    return splats, scratch, acc


def test_evidence_splits_responsibility_exactly(ctx):
    """src/seg/tests.rs:208-227."""
    _, _, acc = split_scene()
    total, fg, bg = acc.bits.read(), acc.fg.read(), acc.bg.read()
    assert total[0] > 0 and total[1] > 0
    np.testing.assert_array_equal(fg + bg, total)
    assert bg[0] == 0 and fg[1] == 0
    assert fg[0] > 0.5 * total[0] and bg[1] > 0.5 * total[1]


def test_evidence_reuse_matches_prepared(ctx):
    """src/seg/tests.rs:233-266: evidence over the RGB render's own
    intersections equals a fresh prepare bit for bit."""
    size = (64, 64)
    splats = sf.Splats(opaque(row_positions(4, 2.0, 0.7)), zero_sh(4))
    scratch = sf.RenderScratch(4, size)
    mask = sf.Mask.from_bytes(size, left_half_mask(*size))
    fresh = sf.Accumulators(4)
    isects = splats.prepare_isects(scratch, sf.camera_default(), size)
    splats.accumulate_prepared(scratch, isects, size, fresh, mask)
    assert np.any(fresh.fg.read() > 0)
    isects = splats.prepare_isects(scratch, sf.camera_default(), size)
    splats.finalize_rgb(scratch, isects, size)
    reused = sf.Accumulators(4)
    splats.accumulate_prepared(scratch, isects, size, reused, mask)
    np.testing.assert_array_equal(fresh.fg.read(), reused.fg.read())
    np.testing.assert_array_equal(fresh.bg.read(), reused.bg.read())


def test_scale_tracks_resolution_change(ctx):
    """src/seg/tests.rs:271-291."""
    splats = sf.Splats(opaque(row_positions(2, 2.0, 1.0)), zero_sh(2))
    scratch = sf.RenderScratch(2, (64, 64))
    reused = sf.Accumulators(2)
    splats.render_responsibility(scratch, reused, sf.camera_default(), (64, 64))
    splats.render_responsibility(scratch, reused, sf.camera_default(), (32, 32))
    fresh = sf.Accumulators(2)
    splats.render_responsibility(scratch, fresh, sf.camera_default(), (32, 32))
    np.testing.assert_array_equal(reused.bits.read(), fresh.bits.read())


def test_beta_update_uses_evidence(ctx):
    """src/seg/tests.rs:296-310."""
    _, _, ev = split_scene()
    state = sf.BetaState.new_uniform(2)
    state.update(ev)
    a, b = state.read()
    assert a[0] > b[0] and b[1] > a[1]
    fg, bg = ev.read_evidence_f32()
    assert abs(a[0] - (1 + fg[0])) < 1e-5
    assert abs(b[1] - (1 + bg[1])) < 1e-5


@pytest.mark.parametrize("cull", [0, 1])
@pytest.mark.parametrize("n,k,w,h,seed", [(30000, 4, 256, 256, 5), (8000, 1, 70, 50, 6)])
def test_seeded_responsibility_and_evidence_bit_exact(ctx, oracle_mod, n, k, w, h, seed, cull):
    from splatfield_b200 import synth

    attr, sh = synth.scene_uniform(n, k, seed)
    cam = sf.look_at((0.3, 0.2, -3.0), (0.0, 0.0, 0.0))
    cam_o = oracle_mod.look_at((0.3, 0.2, -3.0), (0.0, 0.0, 0.0))
    mask = synth.ellipse_mask(w, h, seed)
    splats = sf.Splats(attr, sh)
    scratch = sf.RenderScratch(n, (w, h))
    scratch.set_tuning(raster_cull=cull)
    acc = sf.Accumulators(n)
    isects = splats.prepare_isects(scratch, cam, (w, h))
    splats.accumulate_prepared(scratch, isects, (w, h), acc, None)
    splats.accumulate_prepared(scratch, isects, (w, h), acc, sf.Mask.from_bytes((w, h), mask))
    prep = oracle_mod.prepare(cam_o, w, h, attr, sh, k)
    want = oracle_mod.rasterize(prep, 1, scale=oracle_mod.scale_for(w, h))["resp"]
    fg, bg = oracle_mod.evidence(prep, mask)
    np.testing.assert_array_equal(acc.bits.read(), want)
    np.testing.assert_array_equal(acc.fg.read(), fg)
    np.testing.assert_array_equal(acc.bg.read(), bg)
    np.testing.assert_array_equal(acc.fg.read() + acc.bg.read(), acc.bits.read())
    # Beta update, bit-exact.
    a0, b0 = synth.beta_posterior(n, seed)
    state = sf.BetaState.from_host(a0, b0)
    state.update(acc)
    a1, b1 = state.read()
    wa, wb = oracle_mod.beta_update(a0, b0, fg, bg, oracle_mod.scale_for(w, h))
    np.testing.assert_array_equal(a1.view(np.uint32), wa.view(np.uint32))
    np.testing.assert_array_equal(b1.view(np.uint32), wb.view(np.uint32))


def test_table_entropy_probe_bit_equal_to_oracle(ctx, oracle_mod):
    rng = np.random.default_rng(7)
    a = np.exp(rng.random(5000, dtype=np.float32) * np.float32(7.5)).astype(np.float32)
    b = np.exp(rng.random(5000, dtype=np.float32) * np.float32(7.5)).astype(np.float32)
    a[:5] = [5e5, 1e7, 1.0, 1.0, 1024.0]
    b[:5] = [5e5, 1e7, 1024.0, 1e6, 1.0]
    got = sf.table_entropy(a, b)
    want = oracle_mod.table_entropy(a, b)
    np.testing.assert_array_equal(got.view(np.uint32), want.view(np.uint32))


def test_eig_lut_and_fp64_vs_oracle(ctx, oracle_mod):
    """EIG for a rendered responsibility map: the LUT path's per-splat deltas
    are bit-equal to the oracle's (sums agree to f64 rounding); the FP64 path
    is within 1e-6 nats of the oracle's f64 formulas."""
    from splatfield_b200 import synth

    n, w, h = 40000, 256, 256
    attr, sh = synth.scene_clustered(n, 1, 8)
    cam = sf.look_at((0.0, 0.5, -3.5), (0.0, 0.0, 0.0))
    splats = sf.Splats(attr, sh)
    scratch = sf.RenderScratch(n, (w, h))
    acc = sf.Accumulators(n)
    splats.render_responsibility(scratch, acc, cam, (w, h))
    a, b = synth.beta_posterior(n, 8)
    state = sf.BetaState.from_host(a, b)
    resp = acc.bits.read()
    lut = state.eig(acc, sf.EIG_LUT_F32)
    f64 = state.eig(acc, sf.EIG_FP64)
    want_lut = oracle_mod.eig(a, b, resp, acc.scale, 0)
    want_f64 = oracle_mod.eig(a, b, resp, acc.scale, 1)
    assert abs(lut - want_lut) <= 1e-9 * max(1.0, abs(want_lut))
    assert abs(f64 - want_f64) <= 1e-6
    assert lut > 0 and f64 > 0


def test_eig_matches_reference_mirror(ctx, oracle_mod):
    """src/seg/beta.rs:500-542 on the GPU: EIG vs the f64 mirror within 5e-3
    relative; twice the visibility gains more."""
    n = 1000
    rng = np.random.default_rng(6)
    a = (1 + rng.random(n, dtype=np.float32) * 20).astype(np.float32)
    b = (1 + rng.random(n, dtype=np.float32) * 20).astype(np.float32)
    eps = np.where(np.arange(n) % 2 == 0, rng.random(n, dtype=np.float32) * 0.5, 0).astype(np.float32)
    state = sf.BetaState.from_host(a, b)
    acc = sf.Accumulators.from_eps(eps, 4096.0)
    acc2 = sf.Accumulators.from_eps(eps * 2, 4096.0)

    def delta_ref(x, y, e):
        k = 1.0 + e / (x + y)
        return oracle_mod.beta_entropy(x, y) - oracle_mod.beta_entropy(x * k, y * k)

    want = sum(delta_ref(float(x), float(y), float(e)) for x, y, e in zip(a, b, eps))
    for mode in (sf.EIG_LUT_F32, sf.EIG_FP64):
        eig = state.eig(acc, mode)
        assert abs(eig - want) < 5e-3 * max(abs(want), 1.0)
        assert state.eig(acc2, mode) > eig > 0


def test_eig_reference_properties(ctx, oracle_mod):
    """src/seg/beta.rs:500-611 through the GPU EIG (both modes)."""
    for mode in (sf.EIG_LUT_F32, sf.EIG_FP64):
        # monotone and diminishing
        ka = KA["eig_monotone"]
        acc = sf.Accumulators.from_eps([ka["eps"]], ka["scale"])
        d = [sf.BetaState.from_host([a], [b]).eig(acc, mode) for a, b in ka["states"]]
        assert all(x >= 0 for x in d) and d[0] > d[1] > d[2]
        # ranking survives dominant splats
        kd = KA["eig_ranking_dominant"]
        st = sf.BetaState.from_host(kd["a"], kd["b"])
        acc_a = sf.Accumulators.from_eps(kd["view_a_eps"], kd["scale"])
        acc_b = sf.Accumulators.from_eps(kd["view_b_eps"], kd["scale"])
        ea, eb = st.eig(acc_a, mode), st.eig(acc_b, mode)
        want = oracle_mod.beta_entropy(1, 1) - oracle_mod.beta_entropy(1.25, 1.25)
        assert ea < kd["view_a_max"] and abs(eb - want) < kd["view_b_tolerance"] and eb > ea
        # zero for invisible
        acc0 = sf.Accumulators.from_eps(np.zeros(512), 4096.0)
        assert abs(sf.BetaState.new_uniform(512).eig(acc0, mode)) < 1e-4
