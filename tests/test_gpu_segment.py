"""The active loop on the GPU: localize (src/seg/views.rs:200-274 tests) and
the Segmenter (src/seg/active.rs:295-497 tests) on the three-cluster scene
with the perfect sphere oracle."""
import math

import numpy as np
import pytest

import splatfield_b200 as sf
from splatfield_b200 import segment as seg

from helpers import PER_CLUSTER, cluster_scene, jitter, opaque, zero_sh

pytestmark = pytest.mark.gpu


def splats_at(pos):
    return sf.Splats(opaque(pos), zero_sh(len(pos)))


def test_localize_matches_hand_computed_moments(ctx):
    pos = np.array([[0, 0, 0], [1, 0, 0], [0, 2, 0], [50, -50, 50], [-40, 10, 5]], np.float32)
    splats = splats_at(pos)
    a = np.array([3, 3, 3, 1, 1], np.float32)
    b = np.array([1, 1, 1, 3, 3], np.float32)
    loc = seg.localize(splats, sf.BetaState.from_host(a, b))
    m, w = np.float32(0.75), np.float32(2.25)
    want_c = (pos[0] + pos[1] + pos[2]) * (m / w)
    assert np.linalg.norm(loc.center - want_c) < 1e-6
    want_r = sum(np.linalg.norm(p - want_c) for p in pos[:3]) * (m / w)
    assert abs(loc.radius - want_r) < 1e-6


def test_localize_none_without_fg(ctx):
    pos = [np.ones(3) + 0.1 * jitter(i) for i in range(10)] + [-np.ones(3) + 0.1 * jitter(i) for i in range(10, 20)]
    splats = splats_at(pos)
    assert seg.localize(splats, sf.BetaState.new_uniform(20)) is None


def test_localize_single_fg_splat_clamps_radius(ctx):
    pos = [(2.0, -1.0, 0.5)] + [(-1.0, -1.0, -1.0)] * 7
    splats = splats_at(pos)
    a = np.array([3] + [1] * 7, np.float32)
    b = np.array([1] + [3] * 7, np.float32)
    loc = seg.localize(splats, sf.BetaState.from_host(a, b))
    assert np.isfinite(loc.radius) and loc.radius < 1e-3
    want = 1.5 * max(loc.radius, 1e-3) / math.tan(seg.CANDIDATE_FOV * 0.5)
    for cam in seg.candidates(loc, 5):
        off = np.array(cam.position, np.float32) - loc.center
        assert abs(np.linalg.norm(off) - want) < 1e-6


def harness(iterations, camera=None, candidates=12):
    attr, centers = cluster_scene()
    splats = sf.Splats(attr, zero_sh(3 * PER_CLUSTER))
    if camera is None:
        camera = seg.frame_bounds(splats.bounds)
    cfg = seg.Config(resolution=256, candidates=candidates, iterations=iterations)
    return seg.Segmenter(splats, cfg, camera), centers


def target(centers):
    c, r = centers[0]
    return seg.sphere_oracle([(c, r)])


def test_active_loop_segments_target_cluster(ctx):
    segmenter, centers = harness(6)
    rounds = segmenter.run_with(target(centers))
    assert len(rounds) == 6
    for r in rounds[1:]:
        assert r.eig > 0.0
    labels = segmenter.segmentation()
    n = 3 * PER_CLUSTER
    correct = int(sum(bool(l) == (i < PER_CLUSTER) for i, l in enumerate(labels)))
    assert correct >= n * 90 // 100, (correct, n)
    a, b = segmenter.posteriors()
    means = a / (a + b)
    assert means[:PER_CLUSTER].mean() > 0.7
    assert means[PER_CLUSTER:].max() < 0.5


def test_run_with_stops_when_on_round_returns_false(ctx):
    segmenter, centers = harness(6)
    seen = [0]

    def on_round(_it, _state):
        seen[0] += 1
        return seen[0] < 3

    rounds = segmenter.run_with(target(centers), on_round)
    assert len(rounds) == 3
    a, b = segmenter.posteriors()
    assert np.any((np.abs(a - 1) > 1e-3) | (np.abs(b - 1) > 1e-3))


def test_selected_views_face_the_object(ctx):
    segmenter, centers = harness(3)
    rounds = segmenter.run_with(target(centers))
    c = np.asarray(centers[0][0], np.float32)
    for r in rounds[1:]:
        to_obj = c - np.array(r.camera.position, np.float32)
        fwd = seg.quat_rotate(np.array(r.camera.rotation, np.float32), np.array([[0, 0, 1]], np.float32))[0]
        assert fwd @ to_obj > 0.0


def test_initial_camera_is_honored(ctx):
    _, centers = cluster_scene()
    c = np.asarray(centers[0][0], np.float32)
    cam = sf.look_at(c - np.array([0, 0, 3], np.float32), c)
    segmenter, centers = harness(6, camera=cam)
    rounds = segmenter.run_with(target(centers))
    assert list(rounds[0].camera.position) == list(cam.position)
    assert list(rounds[0].camera.rotation) == list(cam.rotation)
    assert len(rounds) == 6


def test_blind_oracle_stops_after_one_round(ctx):
    segmenter, _ = harness(6)
    rounds = segmenter.run_with(seg.sphere_oracle([]))
    assert len(rounds) == 1 and rounds[0].fg_pixels == 0


def test_unproductive_view_is_not_replayed(ctx):
    def sliver(_rgb, size, _camera):
        m = np.zeros(size[0] * size[1], np.uint8)
        m[0] = 1
        return m

    segmenter, _ = harness(3)
    rounds = segmenter.run_with(sliver)
    assert len(rounds) == 3
    assert rounds[0].fg_pixels == 1
    assert list(rounds[1].camera.position) != list(rounds[0].camera.position)
    assert rounds[1].eig > 0.0


def test_batched_scoring_equals_plain_per_view_scoring(ctx):
    """The round's EIG per candidate equals the plain per-view path
    (render_responsibility + BetaState.eig), so the selected view is the
    reference loop's."""
    segmenter, centers = harness(2)
    segmenter.run_with(target(centers))
    loc = seg.localize(segmenter.splats, segmenter.state)
    cams = seg.candidates(loc, 12)
    batched = segmenter.round.eig(segmenter.splats, segmenter.state, cams, sf.EIG_LUT_F32)
    scratch = sf.RenderScratch(segmenter.splats.n, (256, 256))
    acc = sf.Accumulators(segmenter.splats.n)
    for cam, e in zip(cams, batched):
        segmenter.splats.render_responsibility(scratch, acc, cam, (256, 256))
        assert segmenter.state.eig(acc, sf.EIG_LUT_F32) == e


def test_eig_after_masked_accumulate_equals_responsibility_eig(ctx):
    """sf_beta_eig over an accumulator whose last fill was a masked split
    reads fg + bg, which equals the unmasked ε word for word
    (src/seg/tests.rs:208-227), so its EIG equals the responsibility EIG."""
    from splatfield_b200 import synth

    n, w, h = 20000, 128, 96
    attr, sh = synth.scene_uniform(n, 1, 5)
    splats = sf.Splats(attr, sh)
    scratch = sf.RenderScratch(n, (w, h))
    cam = sf.look_at((0.0, 0.0, -3.0), (0.0, 0.0, 0.0))
    a, b = synth.beta_posterior(n, seed=2)
    beta = sf.BetaState.from_host(a, b)
    acc = sf.Accumulators(n)
    splats.render_responsibility(scratch, acc, cam, (w, h))
    want = {m: beta.eig(acc, m) for m in (sf.EIG_LUT_F32, sf.EIG_FP64)}
    mask = sf.Mask.from_bytes((w, h), synth.ellipse_mask(w, h, seed=4))
    isects = splats.prepare_isects(scratch, cam, (w, h))
    splats.accumulate_prepared(scratch, isects, (w, h), acc, mask)
    assert acc.fg.read().sum() > 0 and acc.bg.read().sum() > 0
    for m, v in want.items():
        assert beta.eig(acc, m) == v
