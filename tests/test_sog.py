"""SOG scenes without a GPU: the loader's host side (zip, meta.json, the
lossless WebP decoder, the reference's checks and messages) and the oracle's
restatement of parse_sog (src/sog.rs:97-198), pinned to the sources the
fixtures encode and to the reference's own unit tests (sog.rs:207-238).
Every check here runs before any CUDA call."""
import ctypes as C
import io
import json
import os
import sys
import zipfile

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
import make_sog_fixtures as M  # noqa: E402


def fixture(name):
    with open(os.path.join(HERE, "golden", name), "rb") as f:
        return f.read()


@pytest.mark.parametrize("name", sorted(M.FIXTURES))
def test_oracle_parse_sog_equals_the_encoded_sources(name):
    from oracle import sog as O

    n, bands, seed = M.FIXTURES[name]
    _, src = M.make_sog(n, bands, seed)
    attr, sh = O.parse_sog(fixture(name))
    want_attr, want_sh = M.expected_planes(src, n, bands)
    np.testing.assert_array_equal(attr.view(np.uint32), want_attr.view(np.uint32))
    np.testing.assert_array_equal(sh.view(np.uint32), want_sh.view(np.uint32))


def test_reference_unit_tests():
    """palette_offset, unpack_quat and inv_log/logit (sog.rs:207-238)."""
    from oracle import sog as O

    assert O.palette_offset(20, 128, 8) == (4 * 8, 1)
    for tag in (252, 253, 254, 255):
        q = O.unpack_quat(np.array([200]), np.array([10]), np.array([77]), np.array([tag]))
        assert abs(float((q[:, 0].astype(np.float64) ** 2).sum()) - 1.0) < 1e-5
    for v in (-3.0, -0.5, 0.0, 0.5, 3.0):
        y = np.float32(1.0 / (1.0 + np.exp(-v)))
        assert abs(float(O.logit(np.array([y]))[0]) - v) < 1e-4


@pytest.mark.parametrize("name", sorted(M.FIXTURES))
def test_inspect_reads_count_and_sh_width(built_lib, name):
    import splatfield_b200 as sf

    n, bands, _ = M.FIXTURES[name]
    assert sf.sog_inspect(fixture(name)) == (n, {0: 1, 1: 4, 3: 16}[bands])


@pytest.mark.parametrize("name", sorted(M.FIXTURES))
def test_webp_decoder_equals_pillow_on_every_plane(built_lib, name):
    from PIL import Image

    import splatfield_b200 as sf

    zf = zipfile.ZipFile(io.BytesIO(fixture(name)))
    for entry in zf.namelist():
        if not entry.endswith(".webp"):
            continue
        data = zf.read(entry)
        want = np.array(Image.open(io.BytesIO(data)).convert("RGBA"))
        np.testing.assert_array_equal(sf.webp_decode(data), want, err_msg=entry)


def _webp(pixels, **kw):
    from PIL import Image

    b = io.BytesIO()
    Image.fromarray(np.ascontiguousarray(pixels, np.uint8), "RGBA").save(b, "WEBP", lossless=True, **kw)
    return b.getvalue()


@pytest.mark.parametrize("kind", ["noise", "gradient", "palette2", "palette4", "palette16", "palette200",
                                  "repeat", "smooth", "large"])
@pytest.mark.parametrize("method", [0, 4, 6])
def test_webp_decoder_equals_pillow_across_encoder_choices(built_lib, kind, method):
    """Images that steer the encoder to each tool of the format: literal
    codes and colour caches (noise), predictors and cross-colour (gradient,
    smooth), colour indexing with 8/4/2/1 pixels per byte (palettes), 2-D
    backward references (repeat), meta prefix codes (large)."""
    import splatfield_b200 as sf

    rng = np.random.default_rng(hash(kind) & 0xFFFF)
    if kind == "noise":
        img = rng.integers(0, 256, (37, 53, 4))
    elif kind == "gradient":
        img = np.zeros((64, 96, 4), np.int64)
        img[..., 0] = np.arange(96)[None] * 2
        img[..., 1] = np.arange(64)[:, None] * 3
        img[..., 2] = 77
        img[..., 3] = 255
    elif kind.startswith("palette"):
        k = int(kind[7:])
        img = rng.integers(0, 256, (k, 4))[rng.integers(0, k, (41, 67))]
    elif kind == "repeat":
        img = np.tile(rng.integers(0, 256, (7, 9, 4)), (20, 15, 1))
    elif kind == "smooth":
        img = np.cumsum(rng.integers(-3, 4, (96, 128, 4)), axis=1) % 256
    else:
        x = np.arange(640)[None, :, None]
        img = (np.sin(x / 17.0) * 100 + np.arange(4)[None, None, :] * 20 + 128
               + rng.integers(0, 3, (480, 640, 4)))
    data = _webp(img.astype(np.uint8), method=method, quality=100 if method else 0)
    from PIL import Image

    want = np.array(Image.open(io.BytesIO(data)).convert("RGBA"))
    np.testing.assert_array_equal(sf.webp_decode(data), want)


def test_webp_decoder_refuses_lossy_and_garbage(built_lib):
    from PIL import Image

    import splatfield_b200 as sf

    b = io.BytesIO()
    Image.fromarray(np.zeros((8, 8, 3), np.uint8)).save(b, "WEBP", lossless=False)
    with pytest.raises(sf.SplatfieldError, match="lossy"):
        sf.webp_decode(b.getvalue())
    with pytest.raises(sf.SplatfieldError, match="RIFF"):
        sf.webp_decode(b"not a webp file at all")
    good = _webp(np.zeros((16, 16, 4), np.uint8))
    with pytest.raises(sf.SplatfieldError):
        sf.webp_decode(good[: len(good) // 2])


def _load_error(data: bytes) -> str:
    """sf_sog_load's error on a stand-in context: its checks all run on the
    host before the context is used."""
    import splatfield_b200 as sf
    from splatfield_b200 import _lib

    L = _lib.lib()
    fake_ctx = C.create_string_buffer(64)
    buf = np.frombuffer(data, np.uint8)
    out = C.c_void_p()
    rc = L.sf_sog_load(C.cast(fake_ctx, C.c_void_p), buf.ctypes.data_as(C.c_void_p), buf.size, C.byref(out))
    assert rc == _lib.SF_ERR_ARG and not out.value
    return L.sf_last_error().decode()


def _edit_zip(data: bytes, drop=(), replace=None):
    src = zipfile.ZipFile(io.BytesIO(data))
    out = io.BytesIO()
    with zipfile.ZipFile(out, "w", zipfile.ZIP_DEFLATED) as zf:
        for name in src.namelist():
            if name in drop:
                continue
            zf.writestr(name, (replace or {}).get(name, src.read(name)))
    return out.getvalue()


def test_reference_errors_and_messages(built_lib):
    """parse_sog's failures (sog.rs:44-198), with its messages."""
    base, _ = M.make_sog(50, 1, 9)
    assert "not a SOG archive" in _load_error(b"PK\x05\x06 garbage")
    assert "missing meta.json" in _load_error(_edit_zip(base, drop=("meta.json",)))
    assert "invalid meta.json" in _load_error(_edit_zip(base, replace={"meta.json": b"{not json"}))
    assert "missing scales.webp" in _load_error(_edit_zip(base, drop=("scales.webp",)))
    zero, _ = M.make_sog(50, 0, 9, meta_edit=lambda m: m.update(count=0))
    assert "SOG contains no splats" in _load_error(zero)
    big, _ = M.make_sog(50, 0, 9, meta_edit=lambda m: m.update(count=5000))
    assert "means_l.webp: 64x1 < 5000 pixels" in _load_error(big)
    cb, _ = M.make_sog(50, 0, 9, meta_edit=lambda m: m["scales"].update(codebook=[0.0] * 10))
    assert "scales codebook: 256 floats expected, got 10" in _load_error(cb)
    tag, _ = M.make_sog(50, 0, 9, quat_tags=np.full(50, 17, np.uint8))
    assert "quats: invalid rotation tag 17" in _load_error(tag)
    bands, _ = M.make_sog(50, 1, 9, meta_edit=lambda m: m["shN"].update(bands=4))
    assert "shN.bands 4 outside 1..=3" in _load_error(bands)
    files, _ = M.make_sog(50, 0, 9, meta_edit=lambda m: m["means"].update(files=["means_l.webp"]))
    assert "invalid meta.json" in _load_error(files)


def test_label_outside_the_palette_is_refused(built_lib):
    data, src = M.make_sog(50, 1, 11)
    meta = json.loads(zipfile.ZipFile(io.BytesIO(data)).read("meta.json"))
    n = 50
    lab = np.zeros((n, 4), np.uint8)
    lab[:, 0] = 200  # 96 palettes in the sheet
    lab[:, 3] = 255
    bad = _edit_zip(data, replace={"shN_labels.webp": M.webp_lossless(M.plane(lab, 64))})
    assert "shN label 200 >= palette size" in _load_error(bad)
    assert meta["count"] == n
