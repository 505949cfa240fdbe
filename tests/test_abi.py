"""The C ABI without a GPU: the library loads, exports every entry point the
header declares, and its host-only functions (camera math, the entropy LUT,
bits_for, fractional bits, map_labels, argument validation) agree with the
oracle bit for bit. No kernel is launched here."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from helpers import known_answers

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "splatfield_cuda.h")


def header_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:const\s+)?\w+\*?\s+\**(sf_\w+)\s*\(", text, flags=re.M)))


def test_header_declares_the_bound_functions():
    from splatfield_b200 import _lib

    names = header_functions()
    assert len(names) >= 50
    assert sorted(_lib.SIGNATURES) == names


def test_library_exports_every_header_symbol(built_lib):
    lib = C.CDLL(built_lib)
    missing = [n for n in header_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_abi_version(built_lib):
    from splatfield_b200._lib import lib

    assert lib().sf_abi_version() == 1


def test_bits_for_matches_reference(built_lib):
    import splatfield_b200 as sf

    for v, want in known_answers()["bits_for"]["cases"]:
        assert sf.bits_for(v) == want


def test_fractional_bits(built_lib, oracle_mod):
    import splatfield_b200 as sf

    for w, h in [(512, 512), (1920, 1080), (256, 256), (70, 70), (1, 1), (65536, 65536), (3, 7)]:
        assert sf.fractional_bits(w, h) == oracle_mod.fractional_bits(w, h)


def test_map_labels_ties_are_background(built_lib):
    import splatfield_b200 as sf

    ka = known_answers()["map_labels"]
    assert list(sf.map_labels(ka["a"], ka["b"])) == ka["labels"]
    with pytest.raises(sf.SplatfieldError):
        sf.map_labels([1.0], [1.0, 2.0])


def test_entropy_table_bit_equal_to_oracle(built_lib, oracle_mod):
    import splatfield_b200 as sf

    np.testing.assert_array_equal(sf.entropy_table().view(np.uint32),
                                  oracle_mod.entropy_table().view(np.uint32))


CAMERAS = [
    dict(position=(0.0, 0.0, 0.0), rotation=(0.0, 0.0, 0.0, 1.0), fov=(0.8, 0.8)),
    dict(position=(-2.0, 0.0, 0.0), rotation=(0.0, 0.70710677, 0.0, 0.70710677), fov=(0.8, 0.8)),
    dict(position=(3.0, -2.0, 7.0), rotation=(0.1, -0.2, 0.3, 0.92736185), fov=(1.0471976, 0.6)),
]


@pytest.mark.parametrize("k", range(len(CAMERAS)))
@pytest.mark.parametrize("size", [(64, 64), (1920, 1080), (70, 33)])
def test_view_for_camera_bit_equal_to_oracle(built_lib, oracle_mod, k, size):
    import splatfield_b200 as sf

    c = CAMERAS[k]
    v1 = sf.view_for_camera(sf.make_camera(**c), *size)
    v2 = oracle_mod.view_for_camera(oracle_mod.camera(**c), *size)
    assert bytes(v1) == bytes(v2)


@pytest.mark.parametrize("pos,target", [((0, 0, -3), (0, 0, 0)), ((4, 0, 0), (0, 0, 0)),
                                        ((0, 0, 4), (0, 0, 0)), ((1.5, -2.0, 0.7), (0.1, 0.2, -0.3)),
                                        ((1.2, 0, -3), (1.2, 0, 0))])
def test_look_at_bit_equal_to_oracle(built_lib, oracle_mod, pos, target):
    import splatfield_b200 as sf

    assert bytes(sf.look_at(pos, target)) == bytes(oracle_mod.look_at(pos, target))


def test_errors_without_a_device_are_reported_not_raised_in_c(built_lib):
    """Argument checks run before any CUDA call and come back as status codes."""
    from splatfield_b200 import _lib

    L = _lib.lib()
    out = C.c_void_p()
    assert L.sf_splats_create(None, None, None, 0, 1, C.byref(out)) == _lib.SF_ERR_ARG
    assert L.sf_last_error()
    assert L.sf_radix_argsort(None, None, None, 0, 0, 0, None, None, None) == _lib.SF_ERR_ARG
    assert L.sf_beta_eig(None, None, 0, None, None) == _lib.SF_ERR_ARG
    assert L.sf_map_labels(None, None, 0, None) == _lib.SF_OK


@pytest.mark.parametrize("bad", [0.0, -1.0, float("nan"), float("inf"), float("-inf"), -2.0**60])
def test_beta_create_refuses_bad_parameters_before_any_cuda_call(built_lib, bad):
    """Non-positive or non-finite Beta parameters are refused with SF_ERR_ARG
    before the context is touched (a stand-in context pointer suffices), so
    they can never reach the FP64 entropy kernels."""
    from splatfield_b200 import _lib

    L = _lib.lib()
    fake_ctx = C.create_string_buffer(64)
    good = np.ones(4, np.float32)
    a = good.copy()
    a[2] = bad
    out = C.c_void_p()
    rc = L.sf_beta_create(C.cast(fake_ctx, C.c_void_p), a.ctypes.data_as(C.c_void_p),
                          good.ctypes.data_as(C.c_void_p), 4, C.byref(out))
    assert rc == _lib.SF_ERR_ARG
    assert b"splat 2" in L.sf_last_error()
    rc = L.sf_beta_create(C.cast(fake_ctx, C.c_void_p), good.ctypes.data_as(C.c_void_p),
                          a.ctypes.data_as(C.c_void_p), 4, C.byref(out))
    assert rc == _lib.SF_ERR_ARG
    assert not out.value


@pytest.mark.parametrize("x", [0.0, -1.0, float("-inf"), float("nan"), -2.0**60])
def test_digamma_terminates_on_non_positive_input(oracle_mod, x):
    """The oracle's digamma (the restatement of beta.rs:77-86) returns NaN
    for x <= 0 and NaN instead of running its recurrence without end; the
    device and host copies in the library carry the same guard."""
    assert np.isnan(oracle_mod.digamma(x))
    assert abs(oracle_mod.digamma(1.0) + 0.5772156649015329) < 1e-8
