"""The CPU oracle against the reference's own known answers and test
properties (CPU only). These pin the oracle before any GPU result is compared
with it."""
import math

import numpy as np
import pytest

from helpers import (known_answers, left_half_mask, opaque, overdraw_positions, rgba,
                     row_positions, stacked_positions, yawed_rotation, zero_sh)

KA = known_answers()


def test_project_counts_tiles_and_packs_bbox(oracle_mod):
    """src/project.rs:399-446."""
    O = oracle_mod
    ka = KA["project_one_splat"]
    v = O.view_for_camera(O.camera(), *ka["size"])
    r = O.project(v, np.array(ka["attributes"], np.float32), np.array(ka["sh"], np.float32), 1, 1)
    assert r["visible"] == ka["visible"]
    assert r["total"] == ka["isects"]
    assert list(r["tile_counts"]) == ka["tile_counts"]
    assert list(r["bbox"]) == ka["bbox"]


@pytest.mark.parametrize("case", ["stacked", "yawed"])
def test_render_golden_center(oracle_mod, case):
    """src/render.rs:671-710: center 127 +- 1 LSB, alpha >= 254, corner transparent."""
    O = oracle_mod
    ka = KA["render_golden_center"]
    if case == "stacked":
        attr, cam = opaque(stacked_positions()), O.camera()
    else:
        attr = opaque([(0.0, 0.0, 0.0)] * 5)
        cam = O.camera(position=(-2.0, 0.0, 0.0), rotation=yawed_rotation())
    out = O.render(cam, 32, 32, attr, zero_sh(5), 1)
    bm = out["bitmap"]
    r, g, b, a = rgba(bm[16, 16])
    assert a >= ka["min_center_alpha"]
    assert rgba(bm[0, 0])[3] == ka["corner_alpha"]
    for got, want in zip((r, g, b), ka["center_rgb"]):
        assert abs(got - want) <= ka["rgb_tolerance_lsb"]


def test_eps_words_match_reference_golden(oracle_mod):
    """src/seg/tests.rs:185-203. The golden words come from Metal's exp/ln;
    this oracle's own exp/log reproduce them to a few LSB (worst: 148 in
    4.1e8 on the front splat, 3.6e-7 relative)."""
    O = oracle_mod
    ka = KA["eps_golden_overdraw"]
    resp = O.responsibility(O.camera(), 70, 70, opaque(overdraw_positions()), zero_sh(40), 1)
    want = np.array(ka["words"], np.int64)
    got = resp.astype(np.int64)
    tol = 4 + 5e-7 * want
    assert np.all(np.abs(got - want) <= tol), list(zip(got, want))
    # Splats past the last visible one collect nothing, exactly.
    assert np.all(got[want == 0] == 0)


def test_responsibility_conserves_pixel_weights(oracle_mod):
    """src/seg/tests.rs:115-126."""
    O = oracle_mod
    attr = opaque(stacked_positions())
    out = O.render(O.camera(), 64, 64, attr, zero_sh(5), 1)
    alpha_sum = float(((out["bitmap"][:, :64] >> 24) & 255).sum()) / 255.0
    resp = O.rasterize(out["prep"], 1, scale=O.scale_for(64, 64))["resp"]
    eps_sum = float(resp.sum()) / O.scale_for(64, 64)
    assert abs(alpha_sum - eps_sum) < 64 * 64 * 3 / 255.0


def test_responsibility_orders_depth_and_culls(oracle_mod):
    """src/seg/tests.rs:130-150."""
    O = oracle_mod
    pos = [(0.0, 0.0, -3.0 if i == 5 else 1.0 + i * 0.5) for i in range(6)]
    resp = O.responsibility(O.camera(), 64, 64, opaque(pos), zero_sh(6), 1)
    for k in range(4):
        assert resp[k] > resp[k + 1]
    assert resp[5] == 0


def test_evidence_splits_responsibility_exactly(oracle_mod):
    """src/seg/tests.rs:208-227."""
    O = oracle_mod
    attr = opaque(row_positions(2, 2.0, 1.0))
    prep = O.prepare(O.camera(), 64, 64, attr, zero_sh(2), 1)
    total = O.rasterize(prep, 1, scale=O.scale_for(64, 64))["resp"]
    fg, bg = O.evidence(prep, left_half_mask(64, 64))
    assert total[0] > 0 and total[1] > 0
    np.testing.assert_array_equal(fg + bg, total)
    assert bg[0] == 0 and fg[1] == 0
    assert fg[0] > 0.5 * total[0] and bg[1] > 0.5 * total[1]


def test_beta_update_uses_evidence(oracle_mod):
    """src/seg/tests.rs:296-310."""
    O = oracle_mod
    attr = opaque(row_positions(2, 2.0, 1.0))
    prep = O.prepare(O.camera(), 64, 64, attr, zero_sh(2), 1)
    fg, bg = O.evidence(prep, left_half_mask(64, 64))
    s = O.scale_for(64, 64)
    a, b = O.beta_update(np.ones(2), np.ones(2), fg, bg, s)
    assert a[0] > b[0] and b[1] > a[1]
    assert abs(a[0] - (1 + fg[0] / s)) < 1e-5
    assert abs(b[1] - (1 + bg[1] / s)) < 1e-5


def test_fractional_bits_and_scale(oracle_mod):
    """src/seg/mod.rs:31-34, 178."""
    O = oracle_mod
    assert O.scale_for(512, 512) == 2.0 ** 14
    assert O.scale_for(1920, 1080) == 2.0 ** 11
    assert O.scale_for(256, 256) == 2.0 ** 16
    assert O.scale_for(384, 384) == 2.0 ** 14
    assert O.scale_for(768, 768) == 2.0 ** 12
    assert O.scale_for(1024, 1024) == 2.0 ** 12
    assert O.scale_for(70, 70) == 2.0 ** 19
    assert O.fractional_bits(65536, 65536) == 0


def test_mask_pack_is_lsb_first(oracle_mod):
    O = oracle_mod
    w, h = 70, 3
    m = np.zeros((h, w), np.uint8)
    m[0, 0] = m[1, 33] = m[2, 69] = 1
    bits, wpr, fg = O.mask_pack(m, w, h)
    assert wpr == 3 and fg == 3
    assert bits[0] == 1 and bits[wpr + 1] == 2 and bits[2 * wpr + 2] == 1 << 5


def test_table_grid_geometry_matches_b_max():
    """src/seg/beta.rs:381-396."""
    ka = KA["entropy"]
    want = math.log(1024.0) / (ka["grid_pts"] - 1)
    step = float(np.float32(ka["ln_step"]))
    assert abs(step - want) < 2e-9
    amax = math.exp(float(np.float32(ka["grid_pts"] - 1) * np.float32(ka["ln_step"])))
    assert abs(amax - 1024.0) < 0.5


def _a_max():
    return float(np.float32(math.exp(float(np.float32(444) * np.float32(0.015611423)))))


def test_entropy_table_band_vs_f64(oracle_mod):
    """src/seg/beta.rs:402-431: LUT within 1e-3 nats of f64 everywhere."""
    O = oracle_mod
    ka = KA["entropy"]
    rng = np.random.default_rng(7)
    u_max = np.float32(444) * np.float32(0.015611423)
    a = list(np.exp(rng.random(2048, dtype=np.float32) * u_max).astype(np.float32))
    b = list(np.exp(rng.random(2048, dtype=np.float32) * u_max).astype(np.float32))
    edge = ka["edge_values"] + [_a_max()]
    for x in edge:
        for y in edge:
            a.append(np.float32(x))
            b.append(np.float32(y))
    got = O.table_entropy(a, b)
    ref = np.array([np.float32(O.beta_entropy(float(x), float(y))) for x, y in zip(a, b)])
    worst = float(np.max(np.abs(got - ref)))
    assert worst < ka["int_band"], worst


def test_beta_entropy_matches_reference(oracle_mod):
    """src/seg/beta.rs:433-456."""
    O = oracle_mod
    cases = KA["entropy"]["cases"]
    got = O.table_entropy([c[0] for c in cases], [c[1] for c in cases])
    for (a, b), h in zip(cases, got):
        assert abs(h - np.float32(O.beta_entropy(a, b))) < 1e-3
    assert abs(got[0]) < 1e-6
    assert abs(O.beta_entropy(1.0, 1.0)) < 1e-12


def test_beta_entropy_clamps_beyond_table(oracle_mod):
    """src/seg/beta.rs:458-494."""
    O = oracle_mod
    am = _a_max()
    got = O.table_entropy([5e5, 1e7, am, 1.0, 1.0], [5e5, 1e7, am, am, 1e6])
    assert got[0] == got[1]
    corner = np.float32(O.beta_entropy(am, am))
    edge = np.float32(O.beta_entropy(1.0, am))
    for k in (0, 2):
        assert abs(got[k] - corner) < 1e-5
    for k in (3, 4):
        assert abs(got[k] - edge) < 1e-5


def _eps_bits(eps, scale):
    return (np.asarray(eps, np.float32) * np.float32(scale)).astype(np.uint32)


def test_eig_matches_reference_and_orders(oracle_mod):
    """src/seg/beta.rs:500-542."""
    O = oracle_mod
    n = 1000
    rng = np.random.default_rng(6)
    a = (1 + rng.random(n, dtype=np.float32) * 20).astype(np.float32)
    b = (1 + rng.random(n, dtype=np.float32) * 20).astype(np.float32)
    eps = np.where(np.arange(n) % 2 == 0, rng.random(n, dtype=np.float32) * 0.5, 0).astype(np.float32)
    scale = 4096.0
    bits = _eps_bits(eps, scale)
    eig = O.eig(a, b, bits, scale, 0)

    def delta_ref(x, y, e):
        k = 1.0 + e / (x + y)
        return O.beta_entropy(x, y) - O.beta_entropy(x * k, y * k)

    want = sum(delta_ref(float(x), float(y), float(e)) for x, y, e in zip(a, b, eps))
    assert abs(eig - want) < 5e-3 * max(abs(want), 1.0)
    eig2 = O.eig(a, b, _eps_bits(eps * 2, scale), scale, 0)
    assert eig2 > eig > 0
    # The f64 path against the same mirror, at the quantised eps.
    want_q = sum(delta_ref(float(x), float(y), float(q) / scale) for x, y, q in zip(a, b, bits))
    assert abs(O.eig(a, b, bits, scale, 1) - want_q) < 1e-9


def test_eig_monotone_and_diminishing(oracle_mod):
    """src/seg/beta.rs:547-566."""
    O = oracle_mod
    ka = KA["eig_monotone"]
    bits = _eps_bits([ka["eps"]], ka["scale"])
    d = [O.eig([a], [b], bits, ka["scale"], 0) for a, b in ka["states"]]
    assert all(x >= 0 for x in d)
    assert d[0] > d[1] > d[2]


def test_eig_zero_for_invisible(oracle_mod):
    """src/seg/beta.rs:570-580."""
    O = oracle_mod
    assert abs(O.eig(np.ones(512), np.ones(512), np.zeros(512), 4096.0, 0)) < 1e-4


def test_eig_ranking_survives_dominant_splats(oracle_mod):
    """src/seg/beta.rs:586-611."""
    O = oracle_mod
    ka = KA["eig_ranking_dominant"]
    s = ka["scale"]
    ea = O.eig(ka["a"], ka["b"], _eps_bits(ka["view_a_eps"], s), s, 0)
    eb = O.eig(ka["a"], ka["b"], _eps_bits(ka["view_b_eps"], s), s, 0)
    want = O.beta_entropy(1, 1) - O.beta_entropy(1.25, 1.25)
    assert ea < ka["view_a_max"]
    assert abs(eb - want) < ka["view_b_tolerance"]
    assert eb > ea


@pytest.mark.parametrize("n", KA["scan_sizes"]["gather_n"])
def test_scan_gather_matches_cpu(oracle_mod, n):
    """crates/sort/src/scan.rs:283-311."""
    O = oracle_mod
    rng = np.random.default_rng(5)
    counts = rng.integers(0, 20, n).astype(np.uint32)
    gids = rng.permutation(n).astype(np.uint32)
    offsets, total = O.scan_gather(gids, counts)
    want = np.concatenate([[0], np.cumsum(counts[gids].astype(np.uint64))[:-1]]).astype(np.uint32)
    np.testing.assert_array_equal(offsets, want)
    assert total == int(counts.sum())


def test_depth_order_is_stable_by_key_then_id(oracle_mod):
    O = oracle_mod
    rng = np.random.default_rng(3)
    keys = rng.integers(0, 50, 20000).astype(np.uint32)
    keys[rng.random(20000) < 0.1] = 0xFFFFFFFF
    order = O.depth_order(keys)
    vis = np.nonzero(keys != 0xFFFFFFFF)[0]
    want = vis[np.argsort(keys[vis], kind="stable")]
    np.testing.assert_array_equal(order, want)


def test_bits_for():
    """crates/sort/src/sort.rs:420-431 (the oracle's and the library's rule)."""
    for v, want in KA["bits_for"]["cases"]:
        m = max(v - 1, 0)
        assert (0 if m == 0 else m.bit_length()) == want


def test_map_labels_rule():
    ka = KA["map_labels"]
    assert [a > b for a, b in zip(ka["a"], ka["b"])] == ka["labels"]


def test_look_at_plus_z_is_identity(oracle_mod):
    """Camera::look_at's minimal arc from +Z to +Z is the identity (src/seg/active.rs:447-449)."""
    O = oracle_mod
    cam = O.look_at((1.2, 0.0, -3.0), (1.2, 0.0, 0.0))
    assert list(cam.rotation) == [0.0, 0.0, 0.0, 1.0]
    assert abs(cam.fov[0] - 0.8) < 1e-7


def test_oracle_tile_ranges_lower_bound(oracle_mod):
    """src/render.rs:824-850: ranges are lower_bound pairs."""
    import ctypes as C

    O = oracle_mod
    ids = np.array([0, 0, 1, 2, 2, 2, 5, 5], np.uint32)
    ranges = np.empty(16, np.uint32)
    O.lib().sfo_tile_ranges(ids.ctypes.data_as(C.c_void_p), 8, 8, ranges.ctypes.data_as(C.c_void_p))
    for t in range(8):
        assert ranges[2 * t] == np.searchsorted(ids, t, "left")
        assert ranges[2 * t + 1] == np.searchsorted(ids, t + 1, "left")
