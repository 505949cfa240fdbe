"""Onesweep radix sort and decoupled-look-back scan vs the reference's sort and
scan tests (crates/sort/src/sort.rs:383-543, crates/sort/src/scan.rs:278-344),
through the C ABI (GPU). Seeds are new (the reference's Rust StdRng streams
are not reproducible here); the properties are the reference's."""
import numpy as np
import pytest

import splatfield_b200 as sf
from helpers import known_answers

pytestmark = pytest.mark.gpu

KA = known_answers()


def argsort_gpu(keys, vals, bits, write_keys=True):
    keys = np.ascontiguousarray(keys, np.uint32)
    vals = np.ascontiguousarray(vals, np.uint32)
    dk, dv = sf.DeviceBuffer.from_array(keys), sf.DeviceBuffer.from_array(vals)
    scratch = sf.RadixScratch(len(keys))
    ko, vo = scratch.argsort(dk, dv, len(keys), bits, write_keys)
    return ko.read(), vo.read()


def assert_argsort_bits(keys, vals, bits):
    ko, vo = argsort_gpu(keys, vals, bits)
    mask = np.uint32(0xFFFFFFFF if bits >= 32 else (1 << bits) - 1)
    assert np.all(np.diff((ko & mask).astype(np.int64)) >= 0)
    np.testing.assert_array_equal(keys[vo], ko)


@pytest.mark.parametrize("n", KA["sort_sizes"]["stable_n"])
def test_sorting_stable(ctx, n):
    rng = np.random.default_rng(0x5EED0001)
    keys = rng.integers(0, KA["sort_sizes"]["stable_key_range"], n).astype(np.uint32)
    vals = np.arange(n, dtype=np.uint32)
    _, vo = argsort_gpu(keys, vals, 8)
    np.testing.assert_array_equal(vo, np.argsort(keys, kind="stable").astype(np.uint32))


def test_sort_values_only(ctx):
    rng = np.random.default_rng(0x5EED0002)
    keys = rng.integers(0, 2**32, 5000, dtype=np.uint64).astype(np.uint32)
    _, vo = argsort_gpu(keys, np.arange(5000, dtype=np.uint32), 32, write_keys=False)
    np.testing.assert_array_equal(vo, np.argsort(keys, kind="stable").astype(np.uint32))


@pytest.mark.parametrize("mx", KA["sort_sizes"]["partial_bits_max"])
def test_sorting_partial_bits(ctx, mx):
    rng = np.random.default_rng(0x5EED0003)
    keys = rng.integers(0, mx, 5000).astype(np.uint32)
    assert_argsort_bits(keys, np.arange(5000, dtype=np.uint32), sf.bits_for(mx))


def test_sorting_32bit_keys(ctx):
    rng = np.random.default_rng(0x5EED0004)
    clustered = []
    for i in range(10000):
        start = rng.integers(i, i + 150)
        end = rng.integers(start, start + 250)
        run = np.arange(start, end)
        clustered.extend(run[rng.random(run.size) < 0.5].tolist())
    spread = rng.integers(0, 1_000_000, KA["sort_sizes"]["spread_n"])
    for keys in (np.array(clustered, np.uint32), spread.astype(np.uint32)):
        assert_argsort_bits(keys, np.arange(keys.size, dtype=np.uint32), 32)


def test_sort_subset_of_capacity(ctx):
    cap, n = KA["sort_sizes"]["subset_cap"], KA["sort_sizes"]["subset_n"]
    keys = (np.arange(cap, dtype=np.uint64) * 2654435761 % 2**32).astype(np.uint32)
    vals = np.arange(cap, dtype=np.uint32)
    dk, dv = sf.DeviceBuffer.from_array(keys), sf.DeviceBuffer.from_array(vals)
    scratch = sf.RadixScratch(n)
    ko, vo = scratch.argsort(dk, dv, n, 32, True)
    out = ko.read()
    np.testing.assert_array_equal(out, np.sort(keys[:n]))
    np.testing.assert_array_equal(keys[vo.read()], out)
    with pytest.raises(sf.SplatfieldError):
        scratch.argsort(dk, dv, n + 1, 32, True)


def test_sort_trivial_returns_inputs(ctx):
    keys = sf.DeviceBuffer.from_array(np.array([7], np.uint32))
    vals = sf.DeviceBuffer.from_array(np.array([3], np.uint32))
    scratch = sf.RadixScratch(4)
    ko, vo = scratch.argsort(keys, vals, 1, 32)
    assert ko.ptr == keys.ptr and vo.ptr == vals.ptr
    ko, vo = scratch.argsort(keys, vals, 4, 0)
    assert ko.ptr == keys.ptr


def test_sort_large_stable_with_many_partitions(ctx):
    rng = np.random.default_rng(9)
    n = 3_000_001
    keys = rng.integers(0, 8160, n).astype(np.uint32)
    _, vo = argsort_gpu(keys, np.arange(n, dtype=np.uint32), 13)
    np.testing.assert_array_equal(vo, np.argsort(keys, kind="stable").astype(np.uint32))


@pytest.mark.parametrize("n", KA["scan_sizes"]["gather_n"])
def test_scan_gather_matches_cpu(ctx, n):
    rng = np.random.default_rng(0x5EED0005)
    counts = rng.integers(0, 20, n).astype(np.uint32)
    gids = rng.permutation(n).astype(np.uint32)
    dg, dc = sf.DeviceBuffer.from_array(gids), sf.DeviceBuffer.from_array(counts)
    out = sf.DeviceBuffer.empty(n)
    sf.exclusive_scan_gather(dg, dc, out, n, sf.ScanScratch(n))
    want = np.concatenate([[0], np.cumsum(counts[gids].astype(np.uint64))[:-1]]).astype(np.uint32)
    np.testing.assert_array_equal(out.read(), want)


@pytest.mark.parametrize("n", KA["scan_sizes"]["buf_n"] + [4_000_003])
def test_scan_buf_matches_cpu(ctx, n):
    counts = (np.arange(n, dtype=np.uint32) % 4).astype(np.uint32)
    buf = sf.DeviceBuffer.from_array(counts)
    sf.exclusive_scan_buf(buf, n, sf.ScanScratch(n))
    want = np.concatenate([[0], np.cumsum(counts.astype(np.uint64))[:-1]]).astype(np.uint32)
    np.testing.assert_array_equal(buf.read(), want)


def test_scan_zero(ctx):
    gids = sf.DeviceBuffer.from_array(np.array([0], np.uint32))
    counts = sf.DeviceBuffer.from_array(np.array([7], np.uint32))
    offsets = sf.DeviceBuffer.from_array(np.array([0xDEADBEEF], np.uint32))
    sf.exclusive_scan_gather(gids, counts, offsets, 0, sf.ScanScratch(1))
    assert offsets.read()[0] == 0xDEADBEEF


@pytest.mark.parametrize("digit_bits", [4, 5, 6, 7, 8])
@pytest.mark.parametrize("bits", [5, 13, 32])
def test_every_digit_width_sorts_stably(ctx, digit_bits, bits):
    """sf_radix_set_digit_bits: 4..8-bit digits (the reference's is 6,
    sort.rs:11-17) give numpy's stable argsort, at key widths that are and
    are not multiples of the digit."""
    rng = np.random.default_rng(0x5EED0100 + digit_bits * 64 + bits)
    n = 300_001
    keys = rng.integers(0, 2**bits, n, dtype=np.uint64).astype(np.uint32)
    dk = sf.DeviceBuffer.from_array(keys)
    scratch = sf.RadixScratch(n)
    scratch.set_digit_bits(digit_bits)
    ko, vo = scratch.argsort(dk, None, n, bits)
    order = np.argsort(keys, kind="stable").astype(np.uint32)
    np.testing.assert_array_equal(vo.read(), order)
    np.testing.assert_array_equal(ko.read(), keys[order])


def test_async_sorts_and_scans_back_to_back_equal_sync(ctx):
    """Sorts enqueued with sync=False and checked by status, and three scans
    enqueued back to back on one stream with one status after them: the same
    arrays as the synchronous calls (stable order, exact offsets)."""
    rng = np.random.default_rng(0x5EED0009)
    n = 1_000_003
    radix = sf.RadixScratch(n)
    scan = sf.ScanScratch(n)
    results = []
    for bits in (32, 20, 8):
        keys = rng.integers(0, 2**32, n, dtype=np.uint64).astype(np.uint32) & np.uint32((1 << bits) - 1 if bits < 32 else 0xFFFFFFFF)
        dk = sf.DeviceBuffer.from_array(keys)
        _, vo = radix.argsort(dk, None, n, bits, sync=False)
        radix.status()
        results.append((keys, vo.read()))
    for keys, got in results:
        np.testing.assert_array_equal(got, np.argsort(keys, kind="stable").astype(np.uint32))
    counts = rng.integers(0, 20, n).astype(np.uint32)
    gids = rng.permutation(n).astype(np.uint32)
    dg, dc = sf.DeviceBuffer.from_array(gids), sf.DeviceBuffer.from_array(counts)
    outs = [sf.DeviceBuffer.empty(n) for _ in range(3)]
    for o in outs:
        sf.exclusive_scan_gather(dg, dc, o, n, scan, sync=False)
    scan.status()
    want = np.concatenate([[0], np.cumsum(counts[gids].astype(np.uint64))[:-1]]).astype(np.uint32)
    for o in outs:
        np.testing.assert_array_equal(o.read(), want)
