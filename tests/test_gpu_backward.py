"""The CUDA adjoint (raster replay from final T + projection chain rule) vs
the oracle's FP64 adjoint of the same forward and FP64 central differences,
and the adjoint's colour gradient vs the u32 evidence lift (GPU).

Tolerances: the GPU forward is FP32 and replays transmittance by division,
the oracle is FP64 with exact per-pixel contributor lists; a pair sitting on
a threshold (alpha = 1/255, T < 1/255) may be decided differently, so the
checks are on relative L2 error per parameter group and on the fraction of
elements within 1e-3 relative (+ an absolute floor)."""
import numpy as np
import pytest

import splatfield_b200 as sf

pytestmark = pytest.mark.gpu

GROUPS = {"means": slice(0, 3), "quats": slice(3, 7), "log_scales": slice(7, 10), "opacity": slice(10, 11)}


def scene(n, k, seed):
    rng = np.random.default_rng(seed)
    a = np.zeros((11, n))
    a[0:2] = rng.uniform(-0.7, 0.7, (2, n))
    a[2] = rng.uniform(-0.4, 0.6, n)
    q = rng.normal(size=(4, n))
    a[3:7] = q / np.linalg.norm(q, axis=0)
    a[7:10] = rng.normal(-2.6, 0.35, (3, n))
    a[10] = rng.normal(0.0, 1.2, n)
    sh = rng.normal(0, 0.3, (k, 3, n))
    return a.astype(np.float32).reshape(-1), sh.astype(np.float32).reshape(-1)


def gpu_grad(attr, sh, k, w, h, dl, cam_pos=(0.2, -0.1, -2.6), want_proj=False):
    n = attr.size // 11
    splats = sf.Splats(attr, sh)
    scratch = sf.RenderScratch(n, (w, h))
    cam = sf.look_at(cam_pos, (0.0, 0.0, 0.0))
    img = splats.render_forward(scratch, cam, (w, h)).read()
    out = splats.render_backward(scratch, cam, (w, h), dl, want_proj=want_proj)
    return (img,) + out


def rel_l2(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-12))


@pytest.mark.parametrize("n,k,w,h,seed", [(400, 1, 64, 64, 1), (1500, 4, 96, 80, 2), (2500, 16, 128, 112, 3)])
def test_gradient_vs_fp64_adjoint(ctx, oracle_mod, n, k, w, h, seed):
    attr, sh = scene(n, k, seed)
    rng = np.random.default_rng(seed + 10)
    dl = rng.normal(size=(h, w, 4)).astype(np.float32)
    img, d_attr, d_sh = gpu_grad(attr, sh, k, w, h, dl)
    cam_o = oracle_mod.look_at((0.2, -0.1, -2.6), (0.0, 0.0, 0.0))
    ref_attr, ref_sh = oracle_mod.render64_backward(cam_o, w, h, attr.astype(np.float64),
                                                    sh.astype(np.float64), k, dl.astype(np.float64))
    ref_attr = ref_attr.reshape(11, n)
    ref_sh = ref_sh.reshape(k, 3, n)
    ref_img = oracle_mod.render64(cam_o, w, h, attr.astype(np.float64), sh.astype(np.float64), k)
    assert np.mean(np.abs(img - ref_img) < 2e-4) > 0.999
    for name, sl in GROUPS.items():
        g, r = d_attr[sl], ref_attr[sl]
        assert rel_l2(g, r) < 5e-3, (name, rel_l2(g, r))
        close = np.abs(g - r) <= 1e-3 * np.abs(r) + 1e-4 * np.abs(r).max()
        assert close.mean() > 0.98, (name, close.mean())
    assert rel_l2(d_sh, ref_sh) < 5e-3
    assert np.abs(ref_attr).max() > 1e-3


def test_gradient_vs_fp64_central_differences(ctx, oracle_mod):
    """256 random parameters: GPU gradient vs FP64 central differences of the
    oracle's FP64 forward (h = 1e-4, stepping down where a side jumps)."""
    n, k, w, h = 300, 4, 64, 56
    attr, sh = scene(n, k, 7)
    rng = np.random.default_rng(17)
    dl = rng.normal(size=(h, w, 4)).astype(np.float32)
    _, d_attr, d_sh = gpu_grad(attr, sh, k, w, h, dl)
    cam_o = oracle_mod.look_at((0.2, -0.1, -2.6), (0.0, 0.0, 0.0))
    a64, s64 = attr.astype(np.float64), sh.astype(np.float64)

    def loss(av, sv):
        return float(np.sum(oracle_mod.render64(cam_o, w, h, av, sv, k) * dl))

    grads = np.concatenate([d_attr.reshape(-1), d_sh.reshape(-1)])
    picks = rng.choice(grads.size, 256, replace=False)
    ok = checked = 0
    for p in picks:
        on_sh = p >= a64.size
        base = s64 if on_sh else a64
        idx = p - a64.size if on_sh else p
        fd = None
        for step in (1e-4, 1e-5, 1e-6):
            plus, minus = base.copy(), base.copy()
            plus[idx] += step
            minus[idx] -= step
            lp = loss(a64, plus) if on_sh else loss(plus, s64)
            lm = loss(a64, minus) if on_sh else loss(minus, s64)
            l0 = loss(a64, s64)
            if abs((lp - l0) - (l0 - lm)) <= 1e-3 * max(abs(lp - l0), abs(l0 - lm)) + 1e-7:
                fd = (lp - lm) / (2 * step)
                break
        if fd is None:
            continue
        checked += 1
        if abs(grads[p] - fd) <= 2e-3 * abs(fd) + 1e-4:
            ok += 1
    assert checked >= 230
    assert ok >= 0.97 * checked, (ok, checked)


def test_adjoint_responsibilities_match_u32_evidence(ctx, oracle_mod):
    """With dL/d(rgba) = (mask, 1 - mask, 1, 0) the colour adjoint is the
    real-valued fg / bg / total responsibility; the u32 lift truncates each
    pixel's share, so scale*adjoint - words lies in [0, pixels touched]."""
    from splatfield_b200 import synth

    n, w, h = 20000, 256, 256
    attr, sh = synth.scene_uniform(n, 1, 31)
    mask = synth.ellipse_mask(w, h, 31).reshape(h, w).astype(np.float32)
    dl = np.stack([mask, 1.0 - mask, np.ones_like(mask), np.zeros_like(mask)], axis=-1)
    cam = sf.look_at((0.2, -0.1, -2.6), (0.0, 0.0, 0.0))
    splats = sf.Splats(attr, sh)
    scratch = sf.RenderScratch(n, (w, h))
    splats.render_forward(scratch, cam, (w, h))
    _, _, proj = splats.render_backward(scratch, cam, (w, h), dl, want_proj=True)
    acc = sf.Accumulators(n)
    isects = splats.prepare_isects(scratch, cam, (w, h))
    splats.accumulate_prepared(scratch, isects, (w, h), acc, None)
    splats.accumulate_prepared(scratch, isects, (w, h), acc, sf.Mask.from_bytes((w, h), mask.astype(np.uint8)))
    scale = acc.scale
    words = {"fg": acc.fg.read(), "bg": acc.bg.read(), "total": acc.bits.read()}
    # A splat covers at most 256 pixels per tile of its bbox.
    pixels = 256.0 * scratch.read(sf._lib.READ_TILE_COUNTS, n).astype(np.float64)
    for col, name in ((5, "fg"), (6, "bg"), (7, "total")):
        real = proj[:, col].astype(np.float64) * scale
        diff = real - words[name].astype(np.float64)
        # truncation makes every word <= its real value; f32 sums drift by ~1e-6
        assert np.all(diff >= -1e-5 * real - 1.0), name
        # at most one LSB per pixel the splat touched
        assert np.all(diff <= 1e-5 * real + pixels + 1.0), name
        assert np.corrcoef(real, words[name])[0, 1] > 0.999999


def test_backward_needs_matching_forward(ctx):
    attr, sh = scene(50, 1, 3)
    splats = sf.Splats(attr, sh)
    scratch = sf.RenderScratch(50, (32, 32))
    cam = sf.look_at((0.2, -0.1, -2.6), (0.0, 0.0, 0.0))
    dl = np.zeros((32, 32, 4), np.float32)
    with pytest.raises(sf.SplatfieldError):
        splats.render_backward(scratch, cam, (32, 32), dl)
    splats.render_forward(scratch, cam, (32, 32))
    other = sf.look_at((0.3, -0.1, -2.6), (0.0, 0.0, 0.0))
    with pytest.raises(sf.SplatfieldError):
        splats.render_backward(scratch, other, (32, 32), dl)
    splats.render_backward(scratch, cam, (32, 32), dl)
    splats.render_with(scratch, cam, (32, 32))
    with pytest.raises(sf.SplatfieldError):
        splats.render_backward(scratch, cam, (32, 32), dl)


def _lift_bounds(real_scaled, words, pixels):
    """The u32 lift truncates each pixel's share: scale * real - words lies in
    [0, pixels touched] (f32 sums drift by ~1e-5 relative)."""
    diff = real_scaled - words.astype(np.float64)
    assert np.all(diff >= -1e-5 * real_scaled - 1.0)
    assert np.all(diff <= 1e-5 * real_scaled + pixels + 1.0)


def test_feature_adjoint_matches_u32_lift_colour_adjoint_and_fp64(ctx, oracle_mod):
    """sf_render_feature_adjoint: the real-valued fg / bg responsibilities
    (i) bound the u32 evidence words of the same frame as the truncation
    allows, (ii) equal the colour adjoint of sf_render_backward with
    dL/d(rgba) = (mask, 1 - mask, ., 0), and (iii) match the oracle's FP64
    adjoint (the SH-DC gradient over the constant C0)."""
    from splatfield_b200 import synth

    n, w, h = 20000, 256, 192
    attr, sh = synth.scene_uniform(n, 1, 41)
    mask_b = synth.ellipse_mask(w, h, 41)
    mask = mask_b.reshape(h, w).astype(np.float32)
    pos = (0.2, -0.1, -2.6)
    cam = sf.look_at(pos, (0.0, 0.0, 0.0))
    splats = sf.Splats(attr, sh)
    scratch = sf.RenderScratch(n, (w, h))
    m = sf.Mask.from_bytes((w, h), mask_b)
    fg_d, bg_d = splats.render_feature_adjoint(scratch, cam, (w, h), m)
    fg, bg = fg_d.read().astype(np.float64), bg_d.read().astype(np.float64)
    acc = sf.Accumulators(n)
    isects = splats.prepare_isects(scratch, cam, (w, h))
    splats.accumulate_prepared(scratch, isects, (w, h), acc, m)
    pixels = 256.0 * scratch.read(sf._lib.READ_TILE_COUNTS, n).astype(np.float64)
    _lift_bounds(fg * acc.scale, acc.fg.read(), pixels)
    _lift_bounds(bg * acc.scale, acc.bg.read(), pixels)
    assert fg.sum() > 1.0 and bg.sum() > 1.0
    # The RGB adjoint's colour entries for the same weights.
    splats.render_forward(scratch, cam, (w, h))
    dl = np.stack([mask, 1.0 - mask, np.zeros_like(mask), np.zeros_like(mask)], axis=-1)
    _, _, proj = splats.render_backward(scratch, cam, (w, h), dl, want_proj=True)
    np.testing.assert_allclose(fg, proj[:, 5], rtol=1e-4, atol=1e-5)
    np.testing.assert_allclose(bg, proj[:, 6], rtol=1e-4, atol=1e-5)
    # FP64 oracle: d L / d sh_dc[c] = C0 * (colour adjoint of channel c).
    cam_o = oracle_mod.look_at(pos, (0.0, 0.0, 0.0))
    _, d_sh = oracle_mod.render64_backward(cam_o, w, h, attr.astype(np.float64), sh.astype(np.float64), 1,
                                           dl.astype(np.float64))
    d_sh = d_sh.reshape(1, 3, n)
    c0 = 0.2820948
    for got, want in ((fg, d_sh[0, 0] / c0), (bg, d_sh[0, 1] / c0)):
        err = np.linalg.norm(got - want) / np.linalg.norm(want)
        assert err < 5e-3, err


def test_round_adjoint_matches_plain_and_feeds_eig_and_update(ctx, oracle_mod):
    """sf_round_evidence_adjoint over uneven views equals the plain per-view
    feature adjoint (float sums: within 1e-5 relative), its EIG equals
    sf_beta_eig_real of those responsibilities to the same precision, and
    the FP64 EIG is within 1e-6 nats of the oracle's f64 formulas over the
    same real eps; the real-valued Beta update adds fg / bg exactly."""
    from splatfield_b200 import synth

    n = 30000
    attr, sh = synth.scene_clustered(n, 4, seed=5, clusters=4, sigma=0.25, extent=1.0)
    a, b = synth.beta_posterior(n, seed=5)
    splats = sf.Splats(attr, sh)
    beta = sf.BetaState.from_host(a, b)
    sizes = [(96, 96), (160, 128), (64, 48), (200, 200)]
    cams = synth.sphere_cameras(len(sizes), 3.0, 7, sf.look_at)
    masks = [sf.Mask.from_bytes(s, synth.ellipse_mask(s[0], s[1], 50 + v)) for v, s in enumerate(sizes)]
    rnd = sf.Round(n, sizes)
    for lanes, cull in ((1, 0), (3, 1)):
        rnd.set_tuning(lanes=lanes, raster_cull=cull)
        eig = rnd.evidence_adjoint(splats, beta, cams, masks, sf.EIG_FP64)
        for v, s in enumerate(sizes):
            scratch = sf.RenderScratch(n, s)
            fg_p, bg_p = splats.render_feature_adjoint(scratch, cams[v], s, masks[v])
            fg_r, bg_r = rnd.adjoint_responsibility(v)
            np.testing.assert_allclose(fg_r.read(), fg_p.read(), rtol=1e-5, atol=1e-6)
            np.testing.assert_allclose(bg_r.read(), bg_p.read(), rtol=1e-5, atol=1e-6)
            e_plain = beta.eig_real(fg_r, bg_r, sf.EIG_FP64)
            assert abs(eig[v] - e_plain) <= 1e-9 * max(1.0, abs(e_plain))
            eps = fg_r.read().astype(np.float64) + bg_r.read().astype(np.float64)
            want = 0.0
            for ai, bi, e in zip(a, b, eps):
                if e > 0:
                    k = 1.0 + e / (float(ai) + float(bi))
                    d = oracle_mod.beta_entropy(float(ai), float(bi)) - oracle_mod.beta_entropy(float(ai) * k,
                                                                                              float(bi) * k)
                    want += max(d, 0.0)
            assert abs(eig[v] - want) <= 1e-6, (v, eig[v], want)
    fg_r, bg_r = rnd.adjoint_responsibility(3)
    beta.update_real(fg_r, bg_r)
    a2, b2 = beta.read()
    np.testing.assert_array_equal(a2, (a + fg_r.read()).astype(np.float32))
    np.testing.assert_array_equal(b2, (b + bg_r.read()).astype(np.float32))
    with pytest.raises(sf.SplatfieldError):
        rnd.evidence_words(0)
