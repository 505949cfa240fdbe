"""CUDA render path vs the CPU oracle, through the C ABI (GPU).

Bit-exact: per-splat depth keys, tile counts, bboxes and projected rows;
depth order; gather-scan offsets; sorted tile ids and splat ids; tile starts;
the RGBA8 bitmap and the float RGBA plane. Plus the reference's own render
tests (known answers and determinism properties)."""
import numpy as np
import pytest

import splatfield_b200 as sf
from splatfield_b200 import _lib as L
from helpers import (assert_frame_equal, gpu_frame, known_answers, opaque, rgba, sine_attributes,
                     stacked_positions, yawed_rotation, zero_sh)

pytestmark = pytest.mark.gpu

KA = known_answers()


BUILDS = [sf.ISECTS_BINNED, sf.ISECTS_DEPTH_SORTED]


@pytest.mark.parametrize("radix_bits", [6, 8])
def test_depth_sorted_build_at_other_digit_widths(ctx, oracle_mod, radix_bits):
    """The depth-sorted build's sorts at 6- and 8-bit digits: the same
    depth order, offsets, tile lists and image as the oracle."""
    from splatfield_b200 import synth

    O = oracle_mod
    n, k, w, h = 30000, 4, 200, 150
    attr, sh = synth.scene_uniform(n, k, 5)
    cam_o = O.look_at((0.1, 0.0, -3.0), (0.0, 0.0, 0.0))
    cam = sf.look_at((0.1, 0.0, -3.0), (0.0, 0.0, 0.0))
    want = O.prepare(cam_o, w, h, attr, sh, k)
    splats = sf.Splats(attr, sh)
    scratch = sf.RenderScratch(n, (w, h))
    scratch.set_tuning(isect_build=sf.ISECTS_DEPTH_SORTED, radix_bits=radix_bits)
    got = gpu_frame(splats, scratch, cam, w, h, n)
    assert_frame_equal(got, want)
    np.testing.assert_array_equal(got["bitmap"], O.rasterize(want, 0)["bitmap"])


@pytest.mark.parametrize("build", BUILDS)
@pytest.mark.parametrize("cull", [0, 1])
@pytest.mark.parametrize("n,k,w,h,seed", [
    (2000, 1, 128, 128, 1),
    (20000, 4, 256, 192, 2),
    (50000, 16, 320, 240, 3),
    (30000, 9, 70, 70, 4),
])
def test_frame_bit_exact_vs_oracle(ctx, oracle_mod, n, k, w, h, seed, cull, build):
    O = oracle_mod
    from splatfield_b200 import synth

    attr, sh = synth.scene_uniform(n, k, seed)
    cam_o = O.look_at((0.0, 0.0, -3.0), (0.0, 0.0, 0.0))
    cam_o.fov[0], cam_o.fov[1] = synth.fov_for(w, h)
    cam = sf.look_at((0.0, 0.0, -3.0), (0.0, 0.0, 0.0))
    cam.fov[0], cam.fov[1] = synth.fov_for(w, h)
    want = O.prepare(cam_o, w, h, attr, sh, k)
    wr = O.rasterize(want, 0)
    splats = sf.Splats(attr, sh)
    scratch = sf.RenderScratch(n, (w, h))
    scratch.set_tuning(raster_cull=cull, isect_build=build)
    got = gpu_frame(splats, scratch, cam, w, h, n)
    assert_frame_equal(got, want)
    np.testing.assert_array_equal(got["bitmap"], wr["bitmap"])
    np.testing.assert_array_equal(got["rgba"].view(np.uint32), wr["rgba"].view(np.uint32))


@pytest.mark.parametrize("build", BUILDS)
def test_full_size_frame_bit_exact_vs_oracle(ctx, oracle_mod, build):
    """The bench workload itself: 1M SH3 splats in 8 clusters, 1920x1080, one
    orbit camera. Every intermediate array and the image, bit for bit."""
    O = oracle_mod
    from splatfield_b200 import synth

    n, k, w, h = 1_000_000, 16, 1920, 1080
    attr, sh = synth.scene_clustered(n, k, seed=0)
    cam_o = synth.orbit_cameras(30, 4.0, w, h, O.look_at)[7]
    cam = synth.orbit_cameras(30, 4.0, w, h, sf.look_at)[7]
    want = O.prepare(cam_o, w, h, attr, sh, k)
    wr = O.rasterize(want, 0)
    splats = sf.Splats(attr, sh)
    scratch = sf.RenderScratch(n, (w, h))
    scratch.set_tuning(isect_build=build)
    got = gpu_frame(splats, scratch, cam, w, h, n)
    assert got["num_isects"] > (1 << 22)
    assert_frame_equal(got, want)
    np.testing.assert_array_equal(got["bitmap"], wr["bitmap"])
    np.testing.assert_array_equal(got["rgba"].view(np.uint32), wr["rgba"].view(np.uint32))


def test_project_counts_tiles_and_packs_bbox(ctx):
    """src/project.rs:399-446 through the GPU path."""
    ka = KA["project_one_splat"]
    splats = sf.Splats(np.array(ka["attributes"], np.float32), np.array(ka["sh"], np.float32))
    scratch = sf.RenderScratch(1, (64, 64))
    isects = splats.prepare_isects(scratch, sf.camera_default(), (64, 64))
    assert isects.num_visible == ka["visible"]
    assert isects.num_isects == ka["isects"]
    assert list(scratch.read(L.READ_TILE_COUNTS, 1)) == ka["tile_counts"]
    assert list(scratch.read(L.READ_BBOX, 2)) == ka["bbox"]


@pytest.mark.parametrize("case", ["stacked", "yawed"])
def test_render_golden_center(ctx, case):
    """src/render.rs:671-710."""
    ka = KA["render_golden_center"]
    if case == "stacked":
        attr, cam = opaque(stacked_positions()), sf.camera_default()
    else:
        attr = opaque([(0.0, 0.0, 0.0)] * 5)
        cam = sf.make_camera(position=(-2.0, 0.0, 0.0), rotation=yawed_rotation())
    splats = sf.Splats(attr, zero_sh(5))
    scratch = sf.RenderScratch(5, (32, 32))
    bm = splats.render_with(scratch, cam, (32, 32)).read()
    r, g, b, a = rgba(bm[16, 16])
    assert a >= ka["min_center_alpha"]
    assert rgba(bm[0, 0])[3] == 0
    for got, want in zip((r, g, b), ka["center_rgb"]):
        assert abs(got - want) <= 1


def test_render_reuses_scratch(ctx):
    """src/render.rs:712-732: re-render through the same scratch is bit-identical."""
    attr = sine_attributes(50, 0.13, 0.5)
    splats = sf.Splats(attr, np.full(150, 0.1, np.float32))
    cam = sf.make_camera(position=(0.0, -1.0, 0.0))
    scratch = sf.RenderScratch(50, (64, 64))
    b = splats.render_with(scratch, cam, (64, 64)).read()
    c = splats.render_with(scratch, cam, (64, 64)).read()
    np.testing.assert_array_equal(b, c)


def test_render_ties_deterministic(ctx):
    """src/render.rs:790-812: 200 identical splats at one depth."""
    n = 200
    splats = sf.Splats(opaque([(0.0, 0.0, 1.0)] * n), zero_sh(n))
    cam = sf.camera_default()
    scratch = sf.RenderScratch(n, (64, 64))
    a = splats.render_with(scratch, cam, (64, 64)).read()
    b = splats.render_with(scratch, cam, (64, 64)).read()
    fresh = sf.RenderScratch(n, (64, 64))
    c = splats.render_with(fresh, cam, (64, 64)).read()
    np.testing.assert_array_equal(a, b)
    np.testing.assert_array_equal(a, c)


def test_delete_then_undo_restores_render_bitwise(ctx):
    """src/render.rs:626-647 (gather = plane-wise selection on the host)."""
    attr = opaque([(i - 1.0, 0.0, 5.0) for i in range(3)])

    def gather(keep):
        a = attr.reshape(11, 3)[:, keep]
        return np.ascontiguousarray(a).reshape(-1)

    def render(keep):
        s = sf.Splats(gather(keep), zero_sh(len(keep)))
        scratch = sf.RenderScratch(len(keep), (32, 32))
        return s.render_with(scratch, sf.camera_default(), (32, 32)).read()

    before = render([0, 1, 2])
    assert not np.array_equal(render([1, 2]), before)
    np.testing.assert_array_equal(render([0, 1, 2]), before)


def test_scratch_stops_allocating_after_first_frame(ctx):
    """src/render.rs:734-763: steady-state frames keep the same capacity."""
    attr = sine_attributes(100, 0.07, 0.4)
    splats = sf.Splats(attr, zero_sh(100))
    cam = sf.make_camera(position=(0.0, -1.2, 0.0))
    scratch = sf.RenderScratch(100, (64, 64))
    splats.render_with(scratch, cam, (64, 64))
    cap = scratch.capacity()
    for _ in range(5):
        splats.render_with(scratch, cam, (64, 64))
        assert scratch.capacity() == cap


def test_scratch_reserve_grows_once_and_keeps_frames_exact(ctx, oracle_mod):
    """sf_scratch_reserve sizes the capacity up front (next power of two, never
    shrinking); frames under it neither grow it nor change."""
    attr = sine_attributes(300, 0.07, 0.4)
    splats = sf.Splats(attr, zero_sh(300))
    cam = sf.make_camera(position=(0.0, -1.2, 0.0))
    scratch = sf.RenderScratch(300, (96, 64))
    scratch.reserve(3_000_000)
    assert scratch.capacity() == 1 << 22
    scratch.reserve(1000)
    assert scratch.capacity() == 1 << 22
    img = splats.render_with(scratch, cam, (96, 64)).read()
    assert scratch.capacity() == 1 << 22
    cam_o = oracle_mod.camera(position=(0.0, -1.2, 0.0))
    np.testing.assert_array_equal(img, oracle_mod.render(cam_o, 96, 64, attr, zero_sh(300), 1)["bitmap"])
    with pytest.raises(sf.SplatfieldError):
        scratch.reserve(1 << 31)


def test_capacity_grows_instead_of_truncating(ctx, oracle_mod):
    """The reference truncates past capacity and grows next frame
    (src/raster.rs:38-46, src/render.rs:171-197); here the first frame is
    already complete: capacity grows to the exact scan total before emission."""
    from splatfield_b200 import synth

    n, w, h = 60000, 512, 512
    attr, sh = synth.scene_uniform(n, 1, 11)
    attr = attr.reshape(11, n)
    attr[7:10] += 2.5  # large splats: many tiles each
    attr = attr.reshape(-1)
    cam = sf.look_at((0.0, 0.0, -3.0), (0.0, 0.0, 0.0))
    splats = sf.Splats(attr, sh)
    scratch = sf.RenderScratch(n, (w, h))
    isects = splats.prepare_isects(scratch, cam, (w, h))
    assert isects.num_isects > (1 << 22)
    assert scratch.capacity() >= isects.num_isects
    cam_o = oracle_mod.look_at((0.0, 0.0, -3.0), (0.0, 0.0, 0.0))
    want = oracle_mod.prepare(cam_o, w, h, attr, sh, 1)
    assert want["num_isects"] == isects.num_isects
    np.testing.assert_array_equal(isects.gaussian_ids().read(), want["gaussian_ids"])


def test_shape_change_rebuilds_scratch(ctx):
    """A scratch built for one size renders another size correctly
    (src/render.rs:171-183 rebuilds in place)."""
    attr = opaque(stacked_positions())
    splats = sf.Splats(attr, zero_sh(5))
    scratch = sf.RenderScratch(5, (64, 64))
    splats.render_with(scratch, sf.camera_default(), (64, 64))
    small = splats.render_with(scratch, sf.camera_default(), (32, 32)).read()
    fresh = splats.render_with(sf.RenderScratch(5, (32, 32)), sf.camera_default(), (32, 32)).read()
    np.testing.assert_array_equal(small[:, :32], fresh[:, :32])


def test_empty_view_renders_transparent(ctx):
    """Every splat behind the camera: zero visible, zero intersections."""
    splats = sf.Splats(opaque([(0.0, 0.0, -5.0)] * 10), zero_sh(10))
    scratch = sf.RenderScratch(10, (48, 40))
    isects = splats.prepare_isects(scratch, sf.camera_default(), (48, 40))
    assert isects.num_visible == 0 and isects.num_isects == 0
    bm = splats.finalize_rgb(scratch, isects, (48, 40)).read()
    assert np.all(bm[:, :48] == 0)


def test_zero_splats_rejected(ctx):
    with pytest.raises(sf.SplatfieldError):
        sf.Splats(np.zeros(0, np.float32), np.zeros(0, np.float32))


def test_render_to_host_matches_device_bitmap(ctx):
    from splatfield_b200 import synth

    attr, sh = synth.scene_uniform(5000, 4, 9)
    cam = sf.look_at((0.0, 0.0, -3.0), (0.0, 0.0, 0.0))
    splats = sf.Splats(attr, sh)
    scratch = sf.RenderScratch(5000, (100, 60))
    dev = splats.render_with(scratch, cam, (100, 60)).read()
    host = splats.render_to_host(scratch, cam, (100, 60))
    np.testing.assert_array_equal(host, dev[:, :100])


def test_float_image_vs_fp64_oracle(ctx, oracle_mod):
    """The FP32 float plane against the FP64 twin of the same forward: max
    abs error per channel, reported; pixels whose alpha sequence crossed a
    threshold differently in f64 are excluded by comparing at the median."""
    from splatfield_b200 import synth

    n, w, h = 20000, 128, 128
    attr, sh = synth.scene_uniform(n, 4, 21)
    cam = sf.look_at((0.0, 0.0, -3.0), (0.0, 0.0, 0.0))
    cam_o = oracle_mod.look_at((0.0, 0.0, -3.0), (0.0, 0.0, 0.0))
    splats = sf.Splats(attr, sh)
    scratch = sf.RenderScratch(n, (w, h))
    got = splats.render_float(scratch, cam, (w, h)).read()
    ref = oracle_mod.render64(cam_o, w, h, attr.astype(np.float64), sh.astype(np.float64), 4)
    err = np.abs(got.astype(np.float64) - ref)
    assert np.median(err) < 1e-6
    assert np.mean(err < 2e-4) > 0.99


@pytest.mark.parametrize("cull", [0, 1])
def test_raster_detail_counters_change_nothing(ctx, cull):
    """The counting form gives the same image; only it fills the per-pair
    diagnostics, and both forms count the same visited pairs."""
    from splatfield_b200 import synth

    attr, sh = synth.scene_uniform(20000, 4, 13)
    cam = sf.look_at((0.0, 0.0, -3.0), (0.0, 0.0, 0.0))
    splats = sf.Splats(attr, sh)
    scratch = sf.RenderScratch(20000, (200, 150))
    scratch.set_tuning(raster_cull=cull)
    a = splats.render_with(scratch, cam, (200, 150)).read()
    plain = scratch.stats()
    scratch.set_tuning(raster_cull=cull, raster_detail=1)
    b = splats.render_with(scratch, cam, (200, 150)).read()
    detail = scratch.stats()
    np.testing.assert_array_equal(a, b)
    assert plain["pairs_visited"] == detail["pairs_visited"] > 0
    assert plain["exp_evaluated"] == 0 and detail["exp_evaluated"] >= detail["contributing"] > 0
    assert detail["pairs_processed"] <= detail["pairs_visited"]


@pytest.mark.parametrize("order", [sf.ORDER_SORTED, sf.ORDER_HYBRID, sf.ORDER_IN_RASTER])
def test_frame_graph_grows_capacity_and_matches_oracle(ctx, oracle_mod, order):
    """sf_render_with / sf_render_to_host run the binned frame as one graph
    with device-side capacity guards: a first frame past the initial
    capacity grows it, re-runs, and still equals the oracle; later frames of
    other cameras replay the graph."""
    from splatfield_b200 import synth

    n, w, h = 60000, 512, 512
    attr, sh = synth.scene_uniform(n, 1, 11)
    attr = attr.reshape(11, n)
    attr[7:10] += 2.5
    attr = attr.reshape(-1)
    splats = sf.Splats(attr, sh)
    scratch = sf.RenderScratch(n, (w, h))
    scratch.set_tuning(raster_order=order)
    for pos in [(0.0, 0.0, -3.0), (0.4, 0.2, -3.2), (0.0, 0.0, -3.0)]:
        cam = sf.look_at(pos, (0.0, 0.0, 0.0))
        got = splats.render_with(scratch, cam, (w, h)).read()
        host = splats.render_to_host(scratch, cam, (w, h))
        prep = oracle_mod.prepare(oracle_mod.look_at(pos, (0.0, 0.0, 0.0)), w, h, attr, sh, 1)
        want = oracle_mod.rasterize(prep, 0)["bitmap"]
        np.testing.assert_array_equal(got, want)
        np.testing.assert_array_equal(host, want[:, :w])
    assert scratch.capacity() > (1 << 22)


def test_frames_to_host_equal_single_frames_and_oracle(ctx, oracle_mod):
    """sf_render_frames_to_host: a camera path in one call (read-backs from
    two staging images overlapping the next frames) gives, frame for frame,
    the images of sf_render_to_host and of the oracle. The first batch starts
    below the capacity its frames need, so the frames past it are rendered
    again after the growth; a second batch into the same pinned buffer
    replays the graph."""
    from splatfield_b200 import synth

    n, w, h = 60000, 320, 240
    attr, sh = synth.scene_uniform(n, 1, 11)
    attr = attr.reshape(11, n)
    attr[7:10] += 2.5
    attr = attr.reshape(-1)
    splats = sf.Splats(attr, sh)
    scratch = sf.RenderScratch(n, (w, h))
    poses = [(0.0, 0.0, -3.0), (0.4, 0.2, -3.2), (-0.5, 0.1, -2.6), (0.0, 0.6, -3.5), (0.2, -0.3, -2.9)]
    cams = [sf.look_at(p, (0.0, 0.0, 0.0)) for p in poses]
    out = sf.pinned_empty((len(cams), h, w), np.uint32)
    splats.render_frames_to_host(scratch, cams, (w, h), out=out)
    assert scratch.capacity() > (1 << 22)
    for i, p in enumerate(poses):
        prep = oracle_mod.prepare(oracle_mod.look_at(p, (0.0, 0.0, 0.0)), w, h, attr, sh, 1)
        want = oracle_mod.rasterize(prep, 0)["bitmap"][:, :w]
        np.testing.assert_array_equal(out[i], want)
    again = sf.pinned_empty((len(cams), h, w), np.uint32)
    splats.render_frames_to_host(scratch, cams[::-1], (w, h), out=again)
    for i in range(len(cams)):
        np.testing.assert_array_equal(again[i], out[len(cams) - 1 - i])
        np.testing.assert_array_equal(splats.render_to_host(scratch, cams[i], (w, h)), out[i])
    # Pageable output memory works too (the copies then do not overlap).
    plain = splats.render_frames_to_host(scratch, cams[:2], (w, h))
    np.testing.assert_array_equal(plain, out[:2])


def test_render_frames_equals_render_with_and_counts_replays(ctx, oracle_mod):
    """sf_render_frames (frames enqueued back to back, one sync) leaves the
    last frame's image, equal to sf_render_with's and the oracle's; each
    graph replay is counted in sf_kernel_launches."""
    from splatfield_b200 import _lib, synth

    n, w, h = 30000, 256, 192
    attr, sh = synth.scene_uniform(n, 1, 21)
    splats = sf.Splats(attr, sh)
    scratch = sf.RenderScratch(n, (w, h))
    poses = [(0.0, 0.0, -3.0), (0.3, 0.1, -2.8), (-0.2, 0.4, -3.3)]
    cams = [sf.look_at(p, (0.0, 0.0, 0.0)) for p in poses]
    splats.render_frames(scratch, cams, (w, h))  # captures the graph
    k0 = _lib.lib().sf_kernel_launches()
    last = splats.render_frames(scratch, cams, (w, h)).read()
    per_frame = (_lib.lib().sf_kernel_launches() - k0) / len(cams)
    assert per_frame >= 8 and per_frame == int(per_frame)
    np.testing.assert_array_equal(last, splats.render_with(scratch, cams[-1], (w, h)).read())
    prep = oracle_mod.prepare(oracle_mod.look_at(poses[-1], (0.0, 0.0, 0.0)), w, h, attr, sh, 1)
    np.testing.assert_array_equal(last, oracle_mod.rasterize(prep, 0)["bitmap"])


@pytest.mark.parametrize("count", [2, 3, 6])
def test_two_frame_pipes_equal_one_pipe_and_oracle(ctx, oracle_mod, count):
    """frame_pipes 2 (frames alternating between the scratch and its internal
    second pipe, on two streams) and frame_pipes 1 give the same images frame
    for frame, through sf_render_frames_to_host and sf_render_frames, for odd
    and even path lengths. The first path starts below the capacity its
    frames need, on both pipes, so frames of either pipe are rendered again
    after the growth; the scratch is left holding the last frame."""
    from splatfield_b200 import synth

    n, w, h = 50000, 288, 200
    attr, sh = synth.scene_uniform(n, 1, 31)
    attr = attr.reshape(11, n)
    attr[7:10] += 3.0  # about 5M intersections per frame, past the first capacity (2^22)
    attr = attr.reshape(-1)
    splats = sf.Splats(attr, sh)
    poses = [(0.0, 0.0, -3.0), (0.4, 0.2, -3.2), (-0.5, 0.1, -2.6), (0.0, 0.6, -3.5), (0.2, -0.3, -2.9),
             (-0.3, -0.4, -3.1)][:count]
    cams = [sf.look_at(p, (0.0, 0.0, 0.0)) for p in poses]
    two = sf.RenderScratch(n, (w, h))
    assert two.get_tuning()["frame_pipes"] == 2
    got = sf.pinned_empty((count, h, w), np.uint32)
    splats.render_frames_to_host(two, cams, (w, h), out=got)
    assert two.capacity() > (1 << 22)
    for i, p in enumerate(poses):
        prep = oracle_mod.prepare(oracle_mod.look_at(p, (0.0, 0.0, 0.0)), w, h, attr, sh, 1)
        np.testing.assert_array_equal(got[i], oracle_mod.rasterize(prep, 0)["bitmap"][:, :w])
    one = sf.RenderScratch(n, (w, h))
    one.set_tuning(frame_pipes=1)
    want = sf.pinned_empty((count, h, w), np.uint32)
    splats.render_frames_to_host(one, cams[::-1], (w, h), out=want)
    again = sf.pinned_empty((count, h, w), np.uint32)
    splats.render_frames_to_host(two, cams[::-1], (w, h), out=again)
    np.testing.assert_array_equal(again, want)
    np.testing.assert_array_equal(again[::-1], got)
    last = splats.render_frames(two, cams, (w, h)).read()
    np.testing.assert_array_equal(last, splats.render_frames(one, cams, (w, h)).read())
    np.testing.assert_array_equal(last[:, :w], got[-1])
    two.reserve(1 << 24)
    splats.render_frames_to_host(two, cams, (w, h), out=again)
    np.testing.assert_array_equal(again, got)


@pytest.mark.parametrize("split", [2, 4])
@pytest.mark.parametrize("cull", [0, 1])
@pytest.mark.parametrize("order", [sf.ORDER_SORTED, sf.ORDER_HYBRID, sf.ORDER_IN_RASTER])
def test_split_tiles_give_the_same_frame_and_words(ctx, oracle_mod, split, cull, order):
    """raster_split 2 / 4 (a tile's pixels over 2 or 4 CTAs, each walking the
    whole list): RGBA8, responsibility and evidence words equal the oracle's
    bit for bit, for sorted, hybrid and in-raster list order."""
    from splatfield_b200 import synth

    O = oracle_mod
    n, w, h = 40000, 200, 136
    attr, sh = synth.scene_uniform(n, 4, 17)
    attr = attr.reshape(11, n)
    attr[7:10] += 1.0  # larger splats: long, partly unsaturated lists
    attr = attr.reshape(-1)
    pos = (0.1, -0.2, -2.8)
    cam, cam_o = sf.look_at(pos, (0.0, 0.0, 0.0)), O.look_at(pos, (0.0, 0.0, 0.0))
    splats = sf.Splats(attr, sh)
    scratch = sf.RenderScratch(n, (w, h))
    scratch.set_tuning(raster_cull=cull, raster_order=order, raster_split=split)
    assert scratch.get_tuning()["raster_split"] == split
    prep = O.prepare(cam_o, w, h, attr, sh, 4)
    got = splats.render_with(scratch, cam, (w, h)).read()
    np.testing.assert_array_equal(got, O.rasterize(prep, 0)["bitmap"])
    acc = sf.Accumulators(n)
    splats.render_responsibility(scratch, acc, cam, (w, h))
    np.testing.assert_array_equal(acc.bits.read(), O.rasterize(prep, 1, scale=O.scale_for(w, h))["resp"])
    mask = synth.ellipse_mask(w, h, 23)
    isects = splats.prepare_isects(scratch, cam, (w, h))
    splats.accumulate_prepared(scratch, isects, (w, h), acc, sf.Mask.from_bytes((w, h), mask))
    fg, bg = O.evidence(prep, mask)
    np.testing.assert_array_equal(acc.fg.read(), fg)
    np.testing.assert_array_equal(acc.bg.read(), bg)


def test_split_rejects_other_values(ctx):
    scratch = sf.RenderScratch(10, (32, 32))
    with pytest.raises(sf.SplatfieldError):
        scratch.set_tuning(raster_split=3)


def test_frame_autotune_picks_a_form_with_the_same_images(ctx, oracle_mod):
    """sf_scratch_autotune times the raster forms on a camera path and keeps
    the fastest; every form gives the oracle's images."""
    from splatfield_b200 import synth

    n, w, h = 30000, 240, 160
    attr, sh = synth.scene_clustered(n, 4, seed=12, clusters=3, sigma=0.3, extent=1.0)
    splats = sf.Splats(attr, sh)
    scratch = sf.RenderScratch(n, (w, h))
    cams = synth.orbit_cameras(4, 3.0, w, h, sf.look_at)
    tuning, ms = scratch.autotune(splats, cams, (w, h))
    assert ms > 0
    assert tuning["raster_cull"] in (0, 1) and tuning["raster_split"] in (1, 2, 4)
    assert tuning["raster_order"] in (sf.ORDER_SORTED, sf.ORDER_HYBRID, sf.ORDER_IN_RASTER)
    assert scratch.get_tuning() == tuning
    cams_o = synth.orbit_cameras(4, 3.0, w, h, oracle_mod.look_at)
    for cam, cam_o in zip(cams, cams_o):
        got = splats.render_with(scratch, cam, (w, h)).read()
        prep = oracle_mod.prepare(cam_o, w, h, attr, sh, 4)
        np.testing.assert_array_equal(got, oracle_mod.rasterize(prep, 0)["bitmap"])
