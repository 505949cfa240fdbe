"""The batched round (one CUDA graph over all candidate views) vs the plain
per-view path (sf_render_responsibility + sf_beta_eig per view, the
reference's Segmenter::select_view loop, src/seg/active.rs:113-129): the
responsibility words must be bit-identical per view and the EIG identical
(same kernels, same fixed-order reductions) (GPU)."""
import numpy as np
import pytest

import splatfield_b200 as sf
from splatfield_b200 import synth

pytestmark = pytest.mark.gpu


def plain(splats, beta, cams, sizes, mode):
    out = []
    for cam, (w, h) in zip(cams, sizes):
        scratch = sf.RenderScratch(splats.n, (w, h))
        acc = sf.Accumulators(splats.n)
        splats.render_responsibility(scratch, acc, cam, (w, h))
        out.append((acc.bits.read(), acc.scale, beta.eig(acc, mode) if beta else None))
    return out


def cams_on_sphere(k, radius, seed):
    return synth.sphere_cameras(k, radius, seed, sf.look_at)


@pytest.mark.parametrize("lanes,cull,build,order,split", [
    (1, 0, sf.ISECTS_BINNED, sf.ORDER_IN_RASTER, 1), (3, 0, sf.ISECTS_DEPTH_SORTED, sf.ORDER_IN_RASTER, 2),
    (4, 1, sf.ISECTS_BINNED, sf.ORDER_SORTED, 4), (2, 1, sf.ISECTS_DEPTH_SORTED, sf.ORDER_SORTED, 1),
    (2, 1, sf.ISECTS_BINNED, sf.ORDER_IN_RASTER, 4), (3, 0, sf.ISECTS_BINNED, sf.ORDER_HYBRID, 2)])
def test_round_matches_plain_per_view(ctx, lanes, cull, build, order, split):
    n = 30000
    attr, sh = synth.scene_clustered(n, 4, seed=3, clusters=4, sigma=0.25, extent=1.0)
    a, b = synth.beta_posterior(n, seed=3)
    splats = sf.Splats(attr, sh)
    beta = sf.BetaState.from_host(a, b)
    sizes = [(64, 48), (128, 128), (96, 160), (70, 70), (33, 17)]
    cams = cams_on_sphere(len(sizes), 3.0, 5)
    rnd = sf.Round(n, sizes)
    rnd.set_tuning(lanes=lanes, raster_cull=cull, isect_build=build, raster_order=order, raster_split=split)
    for mode in (sf.EIG_LUT_F32, sf.EIG_FP64):
        eig = rnd.eig(splats, beta, cams, mode)
        want = plain(splats, beta, cams, sizes, mode)
        for v, (words, scale, e) in enumerate(want):
            got, gscale, _, _ = rnd.responsibility(v)
            np.testing.assert_array_equal(got.read(), words)
            assert gscale == scale
            assert eig[v] == e, (v, eig[v], e)


def test_round_graph_replays_with_new_cameras(ctx):
    n = 20000
    attr, sh = synth.scene_uniform(n, 1, 8)
    a, b = synth.beta_posterior(n, seed=8)
    splats = sf.Splats(attr, sh)
    beta = sf.BetaState.from_host(a, b)
    sizes = [(96, 96)] * 4
    rnd = sf.Round(n, sizes)
    for seed in (1, 2, 3):
        cams = cams_on_sphere(4, 3.0, seed)
        eig = rnd.eig(splats, beta, cams, sf.EIG_LUT_F32)
        want = plain(splats, beta, cams, sizes, sf.EIG_LUT_F32)
        for v in range(4):
            np.testing.assert_array_equal(rnd.responsibility(v)[0].read(), want[v][0])
            assert eig[v] == want[v][2]


@pytest.mark.parametrize("build,order", [(sf.ISECTS_BINNED, sf.ORDER_IN_RASTER),
                                         (sf.ISECTS_BINNED, sf.ORDER_HYBRID),
                                         (sf.ISECTS_BINNED, sf.ORDER_SORTED),
                                         (sf.ISECTS_DEPTH_SORTED, sf.ORDER_SORTED)])
def test_round_capacity_grows_and_reruns(ctx, build, order):
    """Large splats push the intersections past the first-round capacity
    (min(tiles * n, 2^22)); the round grows and re-runs, results unchanged."""
    n = 60000
    attr, sh = synth.scene_uniform(n, 1, 11)
    attr = attr.reshape(11, n)
    attr[7:10] += 2.5
    attr = attr.reshape(-1)
    splats = sf.Splats(attr, sh)
    sizes = [(512, 512), (256, 256)]
    cams = [sf.look_at((0.0, 0.0, -3.0), (0, 0, 0)), sf.look_at((0.5, 0.3, -3.0), (0, 0, 0))]
    rnd = sf.Round(n, sizes)
    rnd.set_tuning(isect_build=build, raster_order=order)
    rnd.eig(splats, None, cams)
    _, _, nis, _ = rnd.responsibility(0)
    assert nis > (1 << 22)
    want = plain(splats, None, cams, sizes, 0)
    for v in range(2):
        np.testing.assert_array_equal(rnd.responsibility(v)[0].read(), want[v][0])


def test_round_autotune_keeps_results(ctx):
    n = 20000
    attr, sh = synth.scene_uniform(n, 1, 12)
    a, b = synth.beta_posterior(n, seed=12)
    splats = sf.Splats(attr, sh)
    beta = sf.BetaState.from_host(a, b)
    sizes = [(128, 128)] * 6
    cams = cams_on_sphere(6, 3.0, 4)
    rnd = sf.Round(n, sizes)
    before = rnd.eig(splats, beta, cams, sf.EIG_FP64)
    tuning, ms = rnd.autotune(splats, beta, cams, sf.EIG_FP64)
    assert tuning["lanes"] in (1, 2, 4, 8) and tuning["raster_cull"] in (0, 1) and ms > 0
    assert rnd.get_tuning() == tuning
    after = rnd.eig(splats, beta, cams, sf.EIG_FP64)
    np.testing.assert_array_equal(before, after)


def test_round_rejects_mismatched_inputs(ctx):
    attr, sh = synth.scene_uniform(100, 1, 1)
    splats = sf.Splats(attr, sh)
    rnd = sf.Round(200, [(32, 32)])
    with pytest.raises(sf.SplatfieldError):
        rnd.eig(splats, None, [sf.camera_default()])
    with pytest.raises(sf.SplatfieldError):
        sf.Round(100, [])


@pytest.mark.parametrize("lanes", [1, 3])
def test_round_evidence_matches_plain_masked_accumulate(ctx, lanes):
    """Evidence round vs per-view prepare + masked accumulate: fg / bg words
    bit-identical, EIG over fg + bg equal to the plain EIG of the same view's
    total responsibility."""
    n = 30000
    attr, sh = synth.scene_clustered(n, 4, seed=21, clusters=4, sigma=0.25, extent=1.0)
    a, b = synth.beta_posterior(n, seed=21)
    splats = sf.Splats(attr, sh)
    beta = sf.BetaState.from_host(a, b)
    sizes = [(64, 48), (128, 128), (96, 160), (33, 17)]
    cams = cams_on_sphere(len(sizes), 3.0, 9)
    masks = [sf.Mask.from_bytes((w, h), synth.ellipse_mask(w, h, seed=40 + i)) for i, (w, h) in enumerate(sizes)]
    rnd = sf.Round(n, sizes)
    rnd.set_tuning(lanes=lanes)
    for mode in (sf.EIG_LUT_F32, sf.EIG_FP64):
        eig = rnd.evidence(splats, beta, cams, masks, mode)
        want = plain(splats, beta, cams, sizes, mode)
        for v, ((w, h), cam, m) in enumerate(zip(sizes, cams, masks)):
            scratch = sf.RenderScratch(n, (w, h))
            acc = sf.Accumulators(n)
            isects = splats.prepare_isects(scratch, cam, (w, h))
            splats.accumulate_prepared(scratch, isects, (w, h), acc, m)
            fg, bg = rnd.evidence_words(v)
            np.testing.assert_array_equal(fg.read(), acc.fg.read())
            np.testing.assert_array_equal(bg.read(), acc.bg.read())
            np.testing.assert_array_equal(fg.read() + bg.read(), want[v][0])
            assert eig[v] == want[v][2], (v, eig[v], want[v][2])
    # A responsibility round after an evidence round rebuilds its graph.
    eig = rnd.eig(splats, beta, cams, sf.EIG_LUT_F32)
    want = plain(splats, beta, cams, sizes, sf.EIG_LUT_F32)
    for v in range(len(sizes)):
        np.testing.assert_array_equal(rnd.responsibility(v)[0].read(), want[v][0])
    with pytest.raises(sf.SplatfieldError):
        rnd.evidence_words(0)
    with pytest.raises(sf.SplatfieldError):
        rnd.evidence(splats, beta, cams, masks[::-1], sf.EIG_LUT_F32)


@pytest.mark.parametrize("kind", [sf.ROUND_RESPONSIBILITY, sf.ROUND_EVIDENCE, sf.ROUND_ADJOINT])
def test_autotune_each_round_kind_keeps_results(ctx, kind):
    """The coordinate search over lanes, build, order, culling and CTAs per
    tile returns a valid tuning for each round kind, caches it, and the
    tuned round's results equal the untuned round's (words bit for bit;
    adjoint floats within 1e-5 relative)."""
    n = 20000
    attr, sh = synth.scene_clustered(n, 1, seed=9, clusters=3, sigma=0.3, extent=1.0)
    a, b = synth.beta_posterior(n, seed=9)
    splats = sf.Splats(attr, sh)
    beta = sf.BetaState.from_host(a, b)
    sizes = [(96, 96), (128, 64), (80, 80)]
    cams = cams_on_sphere(len(sizes), 3.0, 21)
    masks = [sf.Mask.from_bytes(s, synth.ellipse_mask(s[0], s[1], 70 + v)) for v, s in enumerate(sizes)]
    rnd = sf.Round(n, sizes)

    def run():
        if kind == sf.ROUND_EVIDENCE:
            e = rnd.evidence(splats, beta, cams, masks, sf.EIG_FP64)
            return e, [np.concatenate([x.read() for x in rnd.evidence_words(v)]) for v in range(len(sizes))]
        if kind == sf.ROUND_ADJOINT:
            e = rnd.evidence_adjoint(splats, beta, cams, masks, sf.EIG_FP64)
            return e, [np.concatenate([x.read() for x in rnd.adjoint_responsibility(v)]) for v in range(len(sizes))]
        e = rnd.eig(splats, beta, cams, sf.EIG_FP64)
        return e, [rnd.responsibility(v)[0].read() for v in range(len(sizes))]

    e0, w0 = run()
    tuning, ms = rnd.autotune(splats, beta, cams, sf.EIG_FP64, kind=kind, masks=masks)
    assert ms > 0 and tuning["lanes"] in (1, 2, 4, 8) and tuning["raster_split"] in (1, 2, 4)
    if kind == sf.ROUND_ADJOINT:
        assert tuning["raster_order"] == sf.ORDER_SORTED
    assert rnd.get_tuning() == tuning
    e1, w1 = run()
    for x, y in zip(w0, w1):
        if kind == sf.ROUND_ADJOINT:
            np.testing.assert_allclose(y, x, rtol=1e-5, atol=1e-6)
        else:
            np.testing.assert_array_equal(y, x)
    if kind == sf.ROUND_ADJOINT:
        np.testing.assert_allclose(e1, e0, rtol=1e-6)
    else:
        np.testing.assert_array_equal(e1, e0)
