"""sf_exclusive_scan_gather_noalloc (static device scratch, allocates nothing)
against sf_exclusive_scan_gather (scratch from sf_scan_create), both called
through the C ABI. Integer offsets: the outputs must be identical. Two calls
in a row check that the shared static array's leftover contents from the
first call do not leak into the second."""
import ctypes as C

import numpy as np
import pytest

import splatfield_b200 as sf
from splatfield_b200._lib import SF_ERR_SHAPE, SF_OK, lib

MAX_ELEMS = 1 << 24


def _scan_both(gids, counts, n):
    """(offsets from the no-alloc entry point, offsets from the scratch one)."""
    dg = sf.DeviceBuffer.from_array(gids) if gids is not None else None
    dc = sf.DeviceBuffer.from_array(counts)
    got = sf.DeviceBuffer.empty(n)
    want = sf.DeviceBuffer.empty(n)
    gp = C.c_void_p(dg.ptr) if dg is not None else None
    rc = lib().sf_exclusive_scan_gather_noalloc(gp, C.c_void_p(dc.ptr), C.c_void_p(got.ptr), n, None)
    assert rc == SF_OK, lib().sf_last_error()
    scratch = sf.ScanScratch(n)
    rc = lib().sf_exclusive_scan_gather(scratch.handle, gp, C.c_void_p(dc.ptr), C.c_void_p(want.ptr), n, None)
    assert rc == SF_OK, lib().sf_last_error()
    return got.read(), want.read()


def _cpu(gids, counts):
    c = counts[gids] if gids is not None else counts
    # uint64 throughout (an int64 [0] would promote the sums to float64),
    # then the low word, as the kernel stores it.
    sums = np.cumsum(c.astype(np.uint64))[:-1]
    return np.concatenate([np.zeros(1, np.uint64), sums]).astype(np.uint32)


@pytest.mark.gpu
def test_noalloc_scan_matches_scratch_scan_twice(ctx):
    rng = np.random.default_rng(0x5EED00A1)
    # First call at the maximum size, gathered: every look-back word of the
    # static array is used.
    n1 = MAX_ELEMS
    counts1 = rng.integers(0, 600, n1).astype(np.uint32)
    gids1 = rng.permutation(n1).astype(np.uint32)
    got, want = _scan_both(gids1, counts1, n1)
    np.testing.assert_array_equal(got, want)
    np.testing.assert_array_equal(got, _cpu(gids1, counts1))
    # Second call, smaller and without a gather: the stale status words of
    # the first call must not be read as this call's prefixes.
    n2 = 1_000_003
    counts2 = rng.integers(0, 20, n2).astype(np.uint32)
    got, want = _scan_both(None, counts2, n2)
    np.testing.assert_array_equal(got, want)
    np.testing.assert_array_equal(got, _cpu(None, counts2))


def test_noalloc_scan_rejects_oversize_before_any_cuda_call(built_lib):
    """Sizes beyond the maximum fail with SF_ERR_SHAPE and a message naming
    the limit; the check precedes every CUDA call, so it runs without a GPU."""
    rc = lib().sf_exclusive_scan_gather_noalloc(None, None, None, MAX_ELEMS + 1, None)
    assert rc == SF_ERR_SHAPE
    assert str(MAX_ELEMS) in lib().sf_last_error().decode()
    assert lib().sf_exclusive_scan_gather_noalloc(None, None, None, 0, None) == SF_OK
