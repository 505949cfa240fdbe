"""Bounded look-back waits: a wait that runs out is reported as SF_ERR_TIMEOUT
by the standalone sort and scan calls, and the GPU stays usable.

The reference has no bounded waits (its scan is reduce-then-scan and its sort
counts per pass, crates/sort/src/{scan,sort}.rs), so there is nothing of its to
compare with. The failure is made the way a lost predecessor would look: the
test knob sf_debug_lookback keeps the first partition of the scan and of every
digit pass from publishing its status (a flag that nothing then sets) and caps
each wait at a few polls. Every later partition gives up, records the timeout
in the device error word and returns; all accesses stay inside the buffers.
After the knobs are cleared, the same calls succeed and are exact, which also
shows that the error words were cleared once reported.
"""
import ctypes as C

import numpy as np
import pytest

import splatfield_b200 as sf
from splatfield_b200._lib import SF_ERR_TIMEOUT, SF_OK, lib

pytestmark = pytest.mark.gpu

N = 200_003  # 49 scan partitions of 4096 elements, 25 sort partitions of 8192 keys


def _cpu_scan(counts):
    sums = np.cumsum(counts.astype(np.uint64))[:-1]
    return np.concatenate([np.zeros(1, np.uint64), sums]).astype(np.uint32)


def test_look_back_timeouts_are_reported_then_cleared(ctx):
    rng = np.random.default_rng(0x5EED0071)
    counts = rng.integers(0, 50, N).astype(np.uint32)
    keys = rng.integers(0, 2**32, N, dtype=np.uint64).astype(np.uint32)
    dc = sf.DeviceBuffer.from_array(counts)
    dk = sf.DeviceBuffer.from_array(keys)
    out = sf.DeviceBuffer.empty(N)
    scan = sf.ScanScratch(N)
    radix = sf.RadixScratch(N)
    L = lib()
    assert L.sf_debug_lookback(16, 1) == SF_OK
    try:
        with pytest.raises(sf.SplatfieldError) as e:
            sf.exclusive_scan_gather(None, dc, out, N, scan)
        assert e.value.code == SF_ERR_TIMEOUT
        rc = L.sf_exclusive_scan_gather_noalloc(None, C.c_void_p(dc.ptr), C.c_void_p(out.ptr), N, None)
        assert rc == SF_ERR_TIMEOUT
        assert b"timed out" in L.sf_last_error()
        with pytest.raises(sf.SplatfieldError) as e:
            radix.argsort(dk, None, N, 32)
        assert e.value.code == SF_ERR_TIMEOUT
    finally:
        assert L.sf_debug_lookback(0, 0) == SF_OK
    # Knobs cleared: the same scratches give exact results again.
    sf.exclusive_scan_gather(None, dc, out, N, scan)
    np.testing.assert_array_equal(out.read(), _cpu_scan(counts))
    rc = L.sf_exclusive_scan_gather_noalloc(None, C.c_void_p(dc.ptr), C.c_void_p(out.ptr), N, None)
    assert rc == SF_OK, L.sf_last_error()
    np.testing.assert_array_equal(out.read(), _cpu_scan(counts))
    ko, vo = radix.argsort(dk, None, N, 32)
    np.testing.assert_array_equal(vo.read(), np.argsort(keys, kind="stable").astype(np.uint32))


def test_async_sort_and_scan_report_timeouts_at_status(ctx):
    """sf_radix_argsort_async / sf_exclusive_scan_gather_async only enqueue;
    a wait that ran out in any of several calls is reported once by the
    scratch's status call, which clears it, so the next status is clean."""
    rng = np.random.default_rng(0x5EED0072)
    counts = rng.integers(0, 50, N).astype(np.uint32)
    keys = rng.integers(0, 2**32, N, dtype=np.uint64).astype(np.uint32)
    dc = sf.DeviceBuffer.from_array(counts)
    dk = sf.DeviceBuffer.from_array(keys)
    out = sf.DeviceBuffer.empty(N)
    scan = sf.ScanScratch(N)
    radix = sf.RadixScratch(N)
    L = lib()
    assert L.sf_debug_lookback(16, 1) == SF_OK
    try:
        for _ in range(2):
            sf.exclusive_scan_gather(None, dc, out, N, scan, sync=False)
            radix.argsort(dk, None, N, 32, sync=False)
        with pytest.raises(sf.SplatfieldError) as e:
            scan.status()
        assert e.value.code == SF_ERR_TIMEOUT
        with pytest.raises(sf.SplatfieldError) as e:
            radix.status()
        assert e.value.code == SF_ERR_TIMEOUT
    finally:
        assert L.sf_debug_lookback(0, 0) == SF_OK
    scan.status()
    radix.status()
    sf.exclusive_scan_gather(None, dc, out, N, scan, sync=False)
    scan.status()
    np.testing.assert_array_equal(out.read(), _cpu_scan(counts))
    ko, vo = radix.argsort(dk, None, N, 32, sync=False)
    radix.status()
    np.testing.assert_array_equal(vo.read(), np.argsort(keys, kind="stable").astype(np.uint32))
