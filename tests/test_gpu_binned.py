"""The binned intersection build (per-tile counts, place, per-tile shared-memory
sort) against the oracle's reference-order build (depth argsort, scan, emit,
stable tile sort; src/render.rs:318-352): sorted splat ids, tile ids and tile
starts bit-identical, across every per-tile sort size class, with exact depth
ties, and for tile lists too long for the shared-memory sort (GPU)."""
import numpy as np
import pytest

import splatfield_b200 as sf
from splatfield_b200 import _lib as L
from splatfield_b200 import synth

from helpers import opaque, zero_sh

pytestmark = pytest.mark.gpu


def build_both(oracle_mod, attr, sh, k, w, h, cam_pos=(0.0, 0.0, -3.0)):
    O = oracle_mod
    cam_o = O.look_at(cam_pos, (0.0, 0.0, 0.0))
    cam_o.fov[0], cam_o.fov[1] = synth.fov_for(w, h)
    cam = sf.look_at(cam_pos, (0.0, 0.0, 0.0))
    cam.fov[0], cam.fov[1] = synth.fov_for(w, h)
    want = O.prepare(cam_o, w, h, attr, sh, k)
    n = attr.size // 11
    splats = sf.Splats(attr, sh)
    scratch = sf.RenderScratch(n, (w, h))
    scratch.set_tuning(isect_build=sf.ISECTS_BINNED)
    isects = splats.prepare_isects(scratch, cam, (w, h))
    tiles = isects.tile_bounds[0] * isects.tile_bounds[1]
    got = dict(gaussian_ids=isects.gaussian_ids().read(), tile_ids=isects.tile_ids().read(),
               tile_start=scratch.read(L.READ_TILE_START, tiles + 1), num_isects=isects.num_isects)
    img = splats.finalize_rgb(scratch, isects, (w, h)).read()
    want_img = O.rasterize(want, 0)["bitmap"]
    return got, want, img, want_img


def check(got, want, img, want_img):
    assert got["num_isects"] == want["num_isects"]
    np.testing.assert_array_equal(got["gaussian_ids"], want["gaussian_ids"])
    np.testing.assert_array_equal(got["tile_ids"], want["tile_ids"])
    np.testing.assert_array_equal(got["tile_start"][:-1], want["ranges"][:, 0])
    np.testing.assert_array_equal(got["tile_start"][1:], want["ranges"][:, 1])
    np.testing.assert_array_equal(img, want_img)


def test_binned_covers_every_sort_class(ctx, oracle_mod):
    """A dense cluster: tile lists from a handful to ~9k entries, so the
    warp sort (up to 64 entries) and the 512-, 2048-, 4096-, 6144- and
    12288-entry sorts all run."""
    n, w, h = 40000, 256, 256
    attr, sh = synth.scene_clustered(n, 4, seed=31, clusters=1, sigma=0.25, extent=1.0)
    got, want, img, want_img = build_both(oracle_mod, attr, sh, 4, w, h)
    lens = np.diff(got["tile_start"])
    assert lens.max() > 6144 and lens.max() <= 12288, lens.max()
    for lo, hi in [(0, 64), (64, 512), (512, 2048), (2048, 4096), (4096, 6144)]:
        assert ((lens > lo) & (lens <= hi)).any(), (lo, hi)
    check(got, want, img, want_img)


def test_binned_orders_exact_depth_ties_by_id(ctx, oracle_mod):
    """Depths quantised to a few values: most tiles hold runs of equal depth
    keys (buckets past the bucket sort's limit, so the per-tile radix sort
    with its id passes runs), ordered by splat id as the reference's stable
    depth sort does."""
    n, w, h = 20000, 192, 160
    attr, sh = synth.scene_uniform(n, 1, 32)
    a = attr.reshape(11, n)
    a[2] = np.round(a[2] * 4.0) / 4.0
    got, want, img, want_img = build_both(oracle_mod, a.reshape(-1), sh, 1, w, h)
    check(got, want, img, want_img)


@pytest.fixture
def giant_lists():
    """Sets how many of a frame's longest lists the segmented sort takes
    (for scratches created afterwards); restores the default after."""
    def set_(k):
        assert L.lib().sf_debug_giant_lists(k) == 0

    yield set_
    set_(4096)


@pytest.mark.parametrize("segmented", [4096, 1, 0])
@pytest.mark.parametrize("n", [20000, 40000, 150000])
@pytest.mark.parametrize("quantised", [False, True])
def test_binned_sorts_lists_beyond_shared_memory(ctx, oracle_mod, giant_lists, quantised, n, segmented):
    """n splats over one spot: the centre tiles' lists exceed the largest
    register-held sort class (12288 entries). Up to 24576 entries one CTA
    sorts each list in shared memory. Longer lists are by default cut into
    key-contiguous segments sorted on separate CTAs (segments of up to 6144
    entries in registers, longer ones, from bunched keys, by the shared- or
    global-memory form); `segmented` 1 cuts only the first such list and
    sorts the others on one CTA each in global memory, 0 sorts all of them
    that way. With depths quantised to 5 values the buckets overflow and the
    radix sort with its id passes runs, in every form."""
    giant_lists(segmented)
    rng = np.random.default_rng(33)
    z = rng.uniform(0, 1, n)
    if quantised:
        z = np.round(z * 4.0) / 4.0
    pos = np.stack([rng.normal(0, 0.002, n), rng.normal(0, 0.002, n), 1.0 + z], 1)
    attr = opaque(pos)
    got, want, img, want_img = build_both(oracle_mod, attr, zero_sh(n), 1, 64, 64)
    lens = np.diff(got["tile_start"])
    assert lens.max() > (24576 if n > 24576 else 12288)
    if n > 24576:
        assert (lens > 24576).sum() > 1
    check(got, want, img, want_img)


def test_segmented_sort_in_frame_graph_and_round(ctx, oracle_mod):
    """Lists of up to ~100k entries through the frame graph (device-side
    counts, sort classes on side streams) and the batched round: the same
    image as the oracle, and round responsibility words equal to the plain
    per-view path's. The first frame batch and the first round are captured
    before any list length is known (one-CTA sorts); the second ones include
    the segmented sort, chosen from the lists the first ones saw."""
    rng = np.random.default_rng(35)
    n, w, h = 150000, 96, 80
    pos = np.stack([rng.normal(0, 0.01, n), rng.normal(0, 0.01, n), 1.0 + rng.uniform(0, 1, n)], 1)
    attr, sh = opaque(pos), zero_sh(n)
    splats = sf.Splats(attr, sh)
    cam = sf.look_at((0.0, 0.0, -3.0), (0.0, 0.0, 0.0))
    cam.fov[0], cam.fov[1] = synth.fov_for(w, h)
    scratch = sf.RenderScratch(n, (w, h))
    cam_o = oracle_mod.look_at((0.0, 0.0, -3.0), (0.0, 0.0, 0.0))
    cam_o.fov[0], cam_o.fov[1] = synth.fov_for(w, h)
    want = oracle_mod.prepare(cam_o, w, h, attr, sh, 1)
    assert np.diff(want["ranges"], axis=1).max() > 50000
    want_img = oracle_mod.rasterize(want, 0)["bitmap"]
    for _ in range(2):
        got = splats.render_frames(scratch, [cam, cam], (w, h)).read()
        np.testing.assert_array_equal(got, want_img)
    rnd = sf.Round(n, [(w, h)] * 3)
    cams = [cam, sf.look_at((0.2, 0.1, -3.0), (0.0, 0.0, 0.0)), sf.look_at((-0.1, 0.2, -3.0), (0.0, 0.0, 0.0))]
    for c in cams:
        c.fov[0], c.fov[1] = synth.fov_for(w, h)
    rnd.set_tuning(lanes=2)
    plain = []
    for c in cams:
        acc = sf.Accumulators(n)
        splats.render_responsibility(scratch, acc, c, (w, h))
        plain.append((acc.bits.read(), acc.scale))
    for _ in range(2):
        rnd.eig(splats, None, cams)
        for v in range(len(cams)):
            words, scale, _, _ = rnd.responsibility(v)
            np.testing.assert_array_equal(words.read(), plain[v][0])
            assert scale == plain[v][1]


def scene_for(kind):
    if kind == "clustered":
        n, w, h = 40000, 256, 256
        attr, sh = synth.scene_clustered(n, 4, seed=31, clusters=1, sigma=0.25, extent=1.0)
        return attr, sh, 4, w, h
    if kind == "ties":
        n, w, h = 20000, 192, 160
        attr, sh = synth.scene_uniform(n, 1, 32)
        a = attr.reshape(11, n)
        a[2] = np.round(a[2] * 4.0) / 4.0
        return a.reshape(-1), sh, 1, w, h
    rng = np.random.default_rng(33)
    n = 20000
    z = rng.uniform(0, 1, n)
    if kind == "one_spot_ties":
        z = np.round(z * 4.0) / 4.0
    pos = np.stack([rng.normal(0, 0.002, n), rng.normal(0, 0.002, n), 1.0 + z], 1)
    return opaque(pos), zero_sh(n), 1, 64, 64


@pytest.mark.parametrize("order", [sf.ORDER_IN_RASTER, sf.ORDER_HYBRID])
@pytest.mark.parametrize("cull", [0, 1])
@pytest.mark.parametrize("kind", ["clustered", "ties", "one_spot", "one_spot_ties"])
def test_in_raster_order_matches_sorted_lists(ctx, oracle_mod, kind, cull, order):
    """The rasterizer's own slab ordering of the unsorted placed pairs gives
    the same image, float plane and responsibility / evidence words as the
    sorted lists, and the oracle's image (tiles up to 20,000 entries, with
    and without equal depths)."""
    attr, sh, k, w, h = scene_for(kind)
    n = attr.size // 11
    splats = sf.Splats(attr, sh)
    cam = sf.look_at((0.0, 0.0, -3.0), (0.0, 0.0, 0.0))
    cam.fov[0], cam.fov[1] = synth.fov_for(w, h)
    lazy, sorted_ = sf.RenderScratch(n, (w, h)), sf.RenderScratch(n, (w, h))
    lazy.set_tuning(raster_cull=cull, raster_order=order)
    sorted_.set_tuning(raster_cull=cull, raster_order=sf.ORDER_SORTED)
    img_l = splats.render_with(lazy, cam, (w, h)).read()
    img_s = splats.render_with(sorted_, cam, (w, h)).read()
    np.testing.assert_array_equal(img_l, img_s)
    cam_o = oracle_mod.look_at((0.0, 0.0, -3.0), (0.0, 0.0, 0.0))
    cam_o.fov[0], cam_o.fov[1] = synth.fov_for(w, h)
    want = oracle_mod.rasterize(oracle_mod.prepare(cam_o, w, h, attr, sh, k), 0)["bitmap"]
    np.testing.assert_array_equal(img_l, want)
    f_l = splats.render_float(lazy, cam, (w, h)).read()
    f_s = splats.render_float(sorted_, cam, (w, h)).read()
    np.testing.assert_array_equal(f_l.view(np.uint32), f_s.view(np.uint32))
    acc_l, acc_s = sf.Accumulators(n), sf.Accumulators(n)
    splats.render_responsibility(lazy, acc_l, cam, (w, h))
    splats.render_responsibility(sorted_, acc_s, cam, (w, h))
    np.testing.assert_array_equal(acc_l.bits.read(), acc_s.bits.read())
    # Stats count the same walked entries either way.
    assert lazy.stats()["pairs_visited"] == sorted_.stats()["pairs_visited"]



@pytest.mark.parametrize("kind", ["clustered", "one_spot", "ties"])
def test_raster_schedules_match_oracle(ctx, oracle_mod, kind):
    """The rasterizer's block schedules (longest lists first, the default;
    tile order) give the same frame as each other and the oracle, with the
    same walked-pair count, through sf_render_with and sf_render_frames."""
    attr, sh, k, w, h = scene_for(kind)
    n = attr.size // 11
    splats = sf.Splats(attr, sh)
    cam = sf.look_at((0.0, 0.0, -3.0), (0.0, 0.0, 0.0))
    cam.fov[0], cam.fov[1] = synth.fov_for(w, h)
    longest, tiles = sf.RenderScratch(n, (w, h)), sf.RenderScratch(n, (w, h))
    assert longest.get_tuning()["raster_schedule"] == sf.SCHEDULE_LONGEST
    tiles.set_tuning(raster_schedule=sf.SCHEDULE_TILES)
    got = splats.render_with(longest, cam, (w, h)).read()
    np.testing.assert_array_equal(got, splats.render_with(tiles, cam, (w, h)).read())
    assert longest.stats()["pairs_visited"] == tiles.stats()["pairs_visited"]
    cam_o = oracle_mod.look_at((0.0, 0.0, -3.0), (0.0, 0.0, 0.0))
    cam_o.fov[0], cam_o.fov[1] = synth.fov_for(w, h)
    np.testing.assert_array_equal(got, oracle_mod.rasterize(oracle_mod.prepare(cam_o, w, h, attr, sh, k), 0)["bitmap"])
    np.testing.assert_array_equal(splats.render_frames(longest, [cam, cam], (w, h)).read(), got)
