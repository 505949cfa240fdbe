// Binned intersection build: the tile-major, depth-minor (tile id, splat id)
// list without a global sort.
//
// The reference orders intersections with two global sorts
// (src/render.rs:318-352): splats by depth, then a stable sort of the
// emitted (tile, splat) pairs by tile id. Within a tile this yields the
// splats in ascending (depth key, splat id) order, since the depth argsort
// breaks key ties by splat id. This file builds the same list in four
// steps, and no step moves the whole list through a global sort:
//
//   1. bin_count: chunk c of the splats (in id order) is counted per tile in a
//      shared-memory histogram, written as hist[c][tile].
//   2. bin_colscan: per tile, the exclusive prefix of hist over the chunks (in
//      place) and the tile's total; tiles are filed into size classes.
//      An exclusive scan of the totals (sfk::exclusive_scan) gives tile_start.
//   3. bin_place: chunk c re-walks its pairs and drops each (depth key, splat
//      id) at tile_start[t] + hist[c][t] + a shared-memory cursor. The order
//      inside a tile is not yet fixed.
//   4. tile_sort: one CTA per tile sorts its segment in shared memory by
//      (depth key, splat id) with a stable LSD radix sort over only the bits
//      where the segment's keys differ, and writes the splat ids (and, when
//      asked, the tile ids) back in place.
//
// The result is bit-identical to the reference's order: the pair set is the
// same, and a total order on (key, id) has one sorted arrangement.
#include <cuda_runtime.h>
#include <cstdint>
#include "sf_internal.h"

namespace sfk {
namespace {

constexpr uint32_t kBinThreads = 1024;

__device__ __forceinline__ uint32_t lanemask_lt() {
    uint32_t m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// Calls f(splat, tile, payload) for every tile of every splat in [begin,
// end): warps take 32 consecutive splats at a time and spread the pairs over
// their lanes (owner found by a shuffle search over the lanes' inclusive
// ends), so a splat covering many tiles does not stall its warp. payload
// (optional) is a per-splat word loaded once by the splat's lane with its box
// and shuffled to the lanes that emit its pairs. U rounds of 32 pairs are
// handed out per step: their searches and f calls are independent, so their
// shuffle and shared-memory latencies overlap.
template <uint32_t U, typename F>
__device__ __forceinline__ void for_each_pair(uint32_t begin, uint32_t end, const uint2* __restrict__ bbox,
                                              const uint32_t* __restrict__ payload, uint32_t tiles_x, F&& f) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t warp = threadIdx.x >> 5;
    const uint32_t stride = (blockDim.x >> 5) * 32u;
    // The next group's box and payload are loaded while this group's pairs
    // are handed out (a zero box has no pairs).
    uint2 bb_next = make_uint2(0u, 0u);
    uint32_t pay_next = 0;
    uint32_t g0 = begin + warp * 32u;
    if (g0 + lane < end) {
        bb_next = bbox[g0 + lane];
        if (payload) pay_next = payload[g0 + lane];
    }
    for (; g0 < end; g0 += stride) {
        const uint2 bb = bb_next;
        const uint32_t pay = pay_next;
        const uint32_t rn = g0 + stride + lane;
        bb_next = make_uint2(0u, 0u);
        pay_next = 0;
        if (rn < end) {
            bb_next = bbox[rn];
            if (payload) pay_next = payload[rn];
        }
        uint32_t min_x = bb.x & 0xffffu, min_y = bb.x >> 16, width = 1, cnt = 0;
        const uint32_t max_x = bb.y & 0xffffu, max_y = bb.y >> 16;
        if (max_x > min_x && max_y > min_y) {
            width = max_x - min_x;
            cnt = width * (max_y - min_y);
        }
        // 1 / width, shuffled to the pair lanes with the box.
        const float rw = __fdividef(1.0f, (float)width);
        uint32_t incl = cnt;
#pragma unroll
        for (uint32_t d = 1; d < 32; d <<= 1) {
            const uint32_t v = __shfl_up_sync(0xffffffffu, incl, d);
            if (lane >= d) incl += v;
        }
        const uint32_t total = __shfl_sync(0xffffffffu, incl, 31);
        for (uint32_t p0 = 0; p0 < total; p0 += 32u * U) {
            uint32_t o[U];
#pragma unroll
            for (uint32_t u = 0; u < U; ++u) o[u] = 0;
#pragma unroll
            for (uint32_t step = 16; step > 0; step >>= 1) {
#pragma unroll
                for (uint32_t u = 0; u < U; ++u) {
                    const uint32_t v = __shfl_sync(0xffffffffu, incl, o[u] + step - 1);
                    if (v <= p0 + 32u * u + lane) o[u] += step;
                }
            }
#pragma unroll
            for (uint32_t u = 0; u < U; ++u) {
                const uint32_t p = p0 + 32u * u + lane;
                const uint32_t oend = __shfl_sync(0xffffffffu, incl, o[u]);
                const uint32_t ocnt = __shfl_sync(0xffffffffu, cnt, o[u]);
                const uint32_t ow = __shfl_sync(0xffffffffu, width, o[u]);
                const float orw = __shfl_sync(0xffffffffu, rw, o[u]);
                const uint32_t ox = __shfl_sync(0xffffffffu, min_x, o[u]);
                const uint32_t oy = __shfl_sync(0xffffffffu, min_y, o[u]);
                const uint32_t opay = __shfl_sync(0xffffffffu, pay, o[u]);
                if (p < total) {
                    // Row and column of pair k in the owner's box: a float
                    // quotient (k < 2^16, so it is off by at most one) and an
                    // exact integer correction.
                    const uint32_t k = p - (oend - ocnt);
                    uint32_t row = (uint32_t)((float)k * orw);
                    int32_t col = (int32_t)(k - row * ow);
                    if (col < 0) {
                        --row;
                        col += (int32_t)ow;
                    } else if (col >= (int32_t)ow) {
                        ++row;
                        col -= (int32_t)ow;
                    }
                    f(g0 + o[u], (ox + (uint32_t)col) + (oy + row) * tiles_x, opay);
                }
            }
        }
    }
}

// Rounds of 32 pairs per step in the count and place walks. Two rounds in
// place, and two place blocks per SM (32 registers), measured no faster.
constexpr uint32_t kCountUnroll = 1;
constexpr uint32_t kPlaceUnroll = 1;

__global__ __launch_bounds__(kBinThreads) void bin_count_kernel(const uint2* __restrict__ bbox, uint32_t n,
                                                                uint32_t chunk, uint32_t tiles_x,
                                                                uint32_t tiles, uint32_t* __restrict__ hist) {
    pdl_trigger();
    pdl_wait();
    extern __shared__ uint32_t s_hist[];
    for (uint32_t t = threadIdx.x; t < tiles; t += blockDim.x) s_hist[t] = 0;
    __syncthreads();
    const uint32_t begin = min(n, blockIdx.x * chunk);
    const uint32_t end = min(n, begin + chunk);
    for_each_pair<kCountUnroll>(begin, end, bbox, nullptr, tiles_x,
                                [&](uint32_t, uint32_t t, uint32_t) { atomicAdd(&s_hist[t], 1u); });
    __syncthreads();
    uint32_t* row = hist + (size_t)blockIdx.x * tiles;
    for (uint32_t t = threadIdx.x; t < tiles; t += blockDim.x) row[t] = s_hist[t];
}

struct ClassLimits {
    uint32_t max_n[kSortClasses - 1];  // longest list of each class but the last
};

// Block (32, 32): x = tile within the block's 32, y = a group of chunks.
// words: [6] max tile count (atomicMax), [8 + k] tiles in size class k
// (lists[k * tiles + i]); class kSortClasses - 1 holds the lists longer than
// every shared-memory class, "class" kSortClasses the empty tiles.
__global__ __launch_bounds__(1024) void bin_colscan_kernel(uint32_t* __restrict__ hist, uint32_t chunks,
                                                           uint32_t tiles, uint32_t* __restrict__ cnt,
                                                           uint32_t* __restrict__ lists, uint32_t* words,
                                                           ClassLimits lim) {
    pdl_trigger();
    pdl_wait();
    __shared__ uint32_t s_part[32][33];
    const uint32_t tx = threadIdx.x, ty = threadIdx.y;
    const uint32_t t = blockIdx.x * 32u + tx;
    const bool valid = t < tiles;
    const uint32_t per = (chunks + 31u) / 32u;
    const uint32_t c0 = min(chunks, ty * per), c1 = min(chunks, c0 + per);
    uint32_t sum = 0;
    if (valid)
        for (uint32_t c = c0; c < c1; ++c) sum += hist[(size_t)c * tiles + t];
    s_part[ty][tx] = sum;
    __syncthreads();
    if (ty == 0) {
        uint32_t run = 0;
        for (uint32_t y = 0; y < 32; ++y) {
            const uint32_t v = s_part[y][tx];
            s_part[y][tx] = run;
            run += v;
        }
        if (valid) cnt[t] = run;
        if (blockIdx.x == 0 && tx == 0) cnt[tiles] = 0;
        // Size classes (warp-aggregated appends; the list order is free).
        const uint32_t total = valid ? run : 0u;
        uint32_t cls = total == 0 ? kSortClasses : kSortClasses - 1;  // kSortClasses: the empty tiles
        if (total > 0)
            for (int k = kSortClasses - 2; k >= 0; --k)
                if (total <= lim.max_n[k]) cls = (uint32_t)k;
        const uint32_t mx = __reduce_max_sync(0xffffffffu, total);
        if (tx == 0 && mx) atomicMax(words + 6, mx);
#pragma unroll
        for (uint32_t k = 0; k <= kSortClasses; ++k) {
            const uint32_t m = __ballot_sync(0xffffffffu, valid && cls == k);
            if (!m) continue;
            const uint32_t leader = __ffs(m) - 1;
            uint32_t base = 0;
            if (tx == leader) base = atomicAdd(words + 8u + k, __popc(m));
            base = __shfl_sync(0xffffffffu, base, leader);
            if (cls == k) lists[k * tiles + base + __popc(m & lanemask_lt())] = t;
        }
    }
    __syncthreads();
    if (valid) {
        uint32_t run = s_part[ty][tx];
        for (uint32_t c = c0; c < c1; ++c) {
            const size_t i = (size_t)c * tiles + t;
            const uint32_t v = hist[i];
            hist[i] = run;
            run += v;
        }
    }
}

__global__ __launch_bounds__(kBinThreads) void bin_place_kernel(
    const uint2* __restrict__ bbox, const uint32_t* __restrict__ depth_keys, uint32_t n, uint32_t chunk,
    uint32_t tiles_x, uint32_t tiles, const uint32_t* __restrict__ hist, const uint32_t* __restrict__ tile_start,
    uint32_t capacity, uint2* __restrict__ pairs, uint32_t* err) {
    pdl_trigger();
    pdl_wait();
    extern __shared__ uint32_t s_cur[];
    const uint32_t* row = hist + (size_t)blockIdx.x * tiles;
    for (uint32_t t = threadIdx.x; t < tiles; t += blockDim.x) s_cur[t] = tile_start[t] + row[t];
    __syncthreads();
    const uint32_t begin = min(n, blockIdx.x * chunk);
    const uint32_t end = min(n, begin + chunk);
    bool over = false;
    for_each_pair<kPlaceUnroll>(begin, end, bbox, depth_keys, tiles_x, [&](uint32_t s, uint32_t t, uint32_t key) {
        const uint32_t slot = atomicAdd(&s_cur[t], 1u);
        if (slot < capacity) {
            pairs[slot] = make_uint2(key, s);
        } else {
            over = true;
        }
    });
    if (over) atomicOr(err, SF_DEV_ERR_CAPACITY);
}

// ---- per-tile sort
//
// Each tile's placed (depth key, splat id) pairs are sorted by (key, id).
// Main method, a bucket sort: (key - min) >> shift picks one of about 2n
// buckets (monotone in the key); a counting pass and an atomic scatter fill
// them; each entry's final place is its bucket's start plus its rank on
// (key, id) among the bucket's entries, counted by its own thread. A bucket
// past kMaxBucket entries (keys bunched within the tile, or equal keys) sends
// the tile to a stable LSD radix sort on (key, id) in global memory (the
// tile's own ranges of the pair and output buffers, L2-resident).

constexpr uint32_t kMaxBucket = 256;

// One stable LSD pass on digit (x >> shift) & 255, x = key or value, from
// (sk, sv) into (dk, dv). s_base[256], s_wc[WARPS * 256] (zero on entry,
// zero on exit), s_tmp[WARPS].
template <uint32_t THREADS>
__device__ void sort_pass(const uint32_t* sk, const uint32_t* sv, uint32_t* dk, uint32_t* dv, uint32_t n,
                          uint32_t shift, bool by_val, uint32_t* s_base, uint32_t* s_wc, uint32_t* s_tmp) {
    constexpr uint32_t WARPS = THREADS / 32;
    static_assert(THREADS >= 256, "one thread per digit");
    const uint32_t tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5;
    if (tid < 256) s_base[tid] = 0;
    __syncthreads();
    // Digit counts, one shared atomic per distinct digit of each warp (the
    // digits of one tile's keys are far from uniform).
    for (uint32_t c0 = 0; c0 < n; c0 += THREADS) {
        const uint32_t i = c0 + tid;
        const bool valid = i < n;
        const uint32_t d = valid ? ((by_val ? sv[i] : sk[i]) >> shift) & 255u : 0u;
        uint32_t peers = __ballot_sync(0xffffffffu, valid);
#pragma unroll
        for (uint32_t b = 0; b < 8; ++b) {
            const bool bit = (d >> b) & 1u;
            const uint32_t bb = __ballot_sync(0xffffffffu, bit);
            peers &= bit ? bb : ~bb;
        }
        if (valid && (peers & lanemask_lt()) == 0) atomicAdd(&s_base[d], (uint32_t)__popc(peers));
    }
    __syncthreads();
    // Exclusive scan of the 256 digit counts (threads 0..255, warps 0..7).
    uint32_t c = 0, incl = 0;
    if (tid < 256) {
        c = s_base[tid];
        incl = c;
#pragma unroll
        for (uint32_t d = 1; d < 32; d <<= 1) {
            const uint32_t v = __shfl_up_sync(0xffffffffu, incl, d);
            if (lane >= d) incl += v;
        }
        if (lane == 31) s_tmp[warp] = incl;
    }
    __syncthreads();
    if (tid < 256) {
        uint32_t wbase = 0;
        for (uint32_t w = 0; w < warp; ++w) wbase += s_tmp[w];
        s_base[tid] = wbase + incl - c;
    }
    __syncthreads();
    for (uint32_t c0 = 0; c0 < n; c0 += THREADS) {
        const uint32_t i = c0 + tid;
        const bool valid = i < n;
        uint32_t k = 0, v = 0, d = 0;
        if (valid) {
            k = sk[i];
            v = sv[i];
            d = ((by_val ? v : k) >> shift) & 255u;
        }
        uint32_t peers = __ballot_sync(0xffffffffu, valid);
#pragma unroll
        for (uint32_t b = 0; b < 8; ++b) {
            const bool bit = (d >> b) & 1u;
            const uint32_t bb = __ballot_sync(0xffffffffu, bit);
            peers &= bit ? bb : ~bb;
        }
        const uint32_t rank = __popc(peers & lanemask_lt());
        if (valid && rank == 0) s_wc[warp * 256u + d] = __popc(peers);
        __syncthreads();
        if (valid) {
            uint32_t off = s_base[d] + rank;
            for (uint32_t w = 0; w < warp; ++w) off += s_wc[w * 256u + d];
            dk[off] = k;
            dv[off] = v;
        }
        __syncthreads();
        if (tid < 256) {
            uint32_t add = 0;
#pragma unroll
            for (uint32_t w = 0; w < WARPS; ++w) {
                add += s_wc[w * 256u + tid];
                s_wc[w * 256u + tid] = 0;
            }
            s_base[tid] += add;
        }
        __syncthreads();
    }
}

// Block min and max of per-thread partials (uniform result).
template <uint32_t THREADS>
__device__ void block_min_max(uint32_t lo, uint32_t hi, uint32_t* s_tmp, uint32_t& mn, uint32_t& mx) {
    constexpr uint32_t WARPS = THREADS / 32;
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    lo = __reduce_min_sync(0xffffffffu, lo);
    hi = __reduce_max_sync(0xffffffffu, hi);
    __syncthreads();
    if (lane == 0) {
        s_tmp[warp] = lo;
        s_tmp[WARPS + warp] = hi;
    }
    __syncthreads();
    mn = s_tmp[0];
    mx = s_tmp[WARPS];
    for (uint32_t w = 1; w < WARPS; ++w) {
        mn = min(mn, s_tmp[w]);
        mx = max(mx, s_tmp[WARPS + w]);
    }
    __syncthreads();
}

template <uint32_t THREADS>
__device__ void array_min_max(const uint32_t* a, uint32_t n, uint32_t* s_tmp, uint32_t& mn, uint32_t& mx) {
    uint32_t lo = 0xffffffffu, hi = 0;
    for (uint32_t i = threadIdx.x; i < n; i += THREADS) {
        lo = min(lo, a[i]);
        hi = max(hi, a[i]);
    }
    block_min_max<THREADS>(lo, hi, s_tmp, mn, mx);
}

// Stable sort of (k, v) by the bits where [mn, mx] differ; the arrays
// ping-pong through (k2, v2) and the result is copied back when the pass
// count is odd.
template <uint32_t THREADS>
__device__ void sort_bits(uint32_t* k, uint32_t* v, uint32_t* k2, uint32_t* v2, uint32_t n, uint32_t mn,
                          uint32_t mx, bool by_val, uint32_t* s_base, uint32_t* s_wc, uint32_t* s_tmp) {
    const uint32_t bits = mn == mx ? 0u : 32u - __clz(mn ^ mx);
    bool in_2 = false;
    for (uint32_t shift = 0; shift < bits; shift += 8) {
        if (!in_2) sort_pass<THREADS>(k, v, k2, v2, n, shift, by_val, s_base, s_wc, s_tmp);
        else sort_pass<THREADS>(k2, v2, k, v, n, shift, by_val, s_base, s_wc, s_tmp);
        in_2 = !in_2;
    }
    if (in_2) {
        for (uint32_t i = threadIdx.x; i < n; i += THREADS) {
            k[i] = k2[i];
            v[i] = v2[i];
        }
        __syncthreads();
    }
}

// The radix fallback on global memory: (ka, va) hold the tile's entries and
// receive the result, (kb, vb) are scratch. scratch: 256 + WARPS * 256 words.
template <uint32_t THREADS>
__device__ void radix_tile(uint32_t* ka, uint32_t* va, uint32_t* kb, uint32_t* vb, uint32_t n, uint32_t mn,
                           uint32_t mx, uint32_t* scratch, uint32_t* s_tmp) {
    constexpr uint32_t WARPS = THREADS / 32;
    uint32_t* s_base = scratch;
    uint32_t* s_wc = scratch + 256;
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < WARPS * 256; i += THREADS) s_wc[i] = 0;
    __syncthreads();
    sort_bits<THREADS>(ka, va, kb, vb, n, mn, mx, false, s_base, s_wc, s_tmp);
    int tie = 0;
    for (uint32_t i = threadIdx.x; i + 1 < n; i += THREADS) tie |= ka[i] == ka[i + 1];
    if (__syncthreads_or(tie)) {
        uint32_t imn, imx;
        array_min_max<THREADS>(va, n, s_tmp, imn, imx);
        sort_bits<THREADS>(ka, va, kb, vb, n, imn, imx, true, s_base, s_wc, s_tmp);
        sort_bits<THREADS>(ka, va, kb, vb, n, mn, mx, false, s_base, s_wc, s_tmp);
    }
}

struct BucketPlan {
    uint32_t shift, nbins;
};

__device__ __forceinline__ BucketPlan bucket_plan(uint32_t n, uint32_t mn, uint32_t mx, uint32_t max_bins) {
    const uint32_t range = mx - mn;
    const uint32_t rbits = range == 0 ? 0u : 32u - __clz(range);
    uint32_t lbits = 8;
    while (lbits < 31 && (1u << lbits) < 2u * n) ++lbits;
    while ((1u << lbits) > max_bins) --lbits;
    const uint32_t shift = rbits > lbits ? rbits - lbits : 0u;
    return {shift, (range >> shift) + 1u};  // nbins <= 2^lbits <= max_bins
}

// Clears the counts of buckets [0, nbins) in 16-byte words (bins is 16-byte
// aligned and holds a whole number of them past nbins).
template <uint32_t THREADS>
__device__ __forceinline__ void bucket_clear(uint32_t* bins, uint32_t nbins) {
    uint4* b4 = reinterpret_cast<uint4*>(bins);
    for (uint32_t q = threadIdx.x; q < (nbins + 3u) / 4u; q += THREADS) b4[q] = make_uint4(0u, 0u, 0u, 0u);
}

// Turns bucket counts into bucket starts (exclusive scan, each thread a
// consecutive run of 16-byte words, cleared by bucket_clear); returns the
// largest bucket (uniform). The counts of a word's buckets past nbins are
// zero, so their starts (never read) do not disturb the others.
template <uint32_t THREADS>
__device__ uint32_t bucket_starts(uint32_t* bins, uint32_t nbins, uint32_t* s_tmp) {
    constexpr uint32_t WARPS = THREADS / 32;
    static_assert(WARPS <= 32, "one total per lane");
    const uint32_t tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5;
    uint4* b4 = reinterpret_cast<uint4*>(bins);
    const uint32_t nq = (nbins + 3u) / 4u;
    const uint32_t per = (nq + THREADS - 1) / THREADS;
    const uint32_t q0 = min(nq, tid * per), q1 = min(nq, q0 + per);
    uint32_t run = 0, big = 0;
    for (uint32_t q = q0; q < q1; ++q) {
        const uint4 c = b4[q];
        run += (c.x + c.y) + (c.z + c.w);
        big = max(big, max(max(c.x, c.y), max(c.z, c.w)));
    }
    uint32_t incl = run;
#pragma unroll
    for (uint32_t d = 1; d < 32; d <<= 1) {
        const uint32_t v = __shfl_up_sync(0xffffffffu, incl, d);
        if (lane >= d) incl += v;
    }
    big = __reduce_max_sync(0xffffffffu, big);
    if (lane == 31) s_tmp[2 * WARPS + warp] = incl;
    if (lane == 0) s_tmp[3 * WARPS + warp] = big;
    __syncthreads();
    // Lane w holds warp w's total and largest bucket: the warps before this
    // one add up to its base.
    const uint32_t tot = lane < warp ? s_tmp[2 * WARPS + lane] : 0u;
    const uint32_t wb = lane < WARPS ? s_tmp[3 * WARPS + lane] : 0u;
    uint32_t base = incl - run + __reduce_add_sync(0xffffffffu, tot);
    big = __reduce_max_sync(0xffffffffu, wb);
    if (big <= kMaxBucket) {
        for (uint32_t q = q0; q < q1; ++q) {
            const uint4 c = b4[q];
            uint4 st;
            st.x = base;
            base += c.x;
            st.y = base;
            base += c.y;
            st.z = base;
            base += c.z;
            st.w = base;
            base += c.w;
            b4[q] = st;
        }
    }
    __syncthreads();
    return big;
}

// Ranks of the bucketed entries (kb, vb), written as splat ids to
// out[rank] and the tile id to tids_out.
template <uint32_t THREADS>
__device__ void bucket_rank_store(const uint32_t* kb, const uint32_t* vb, const uint32_t* bins, uint32_t n,
                                  uint32_t mn, uint32_t shift, uint32_t* out, uint32_t* tids_out, uint32_t t) {
    for (uint32_t i = threadIdx.x; i < n; i += THREADS) {
        const uint32_t k = kb[i], v = vb[i];
        const uint32_t b = (k - mn) >> shift;
        const uint32_t lo = b ? bins[b - 1] : 0u, hi = bins[b];
        uint32_t rank = lo;
        for (uint32_t j = lo; j < hi; ++j) {
            const uint32_t kj = kb[j];
            rank += (kj < k) || (kj == k && vb[j] < v);
        }
        out[rank] = v;
        if (tids_out) tids_out[i] = t;
    }
}

// Shared form: the n <= MAXN entries of slots [start, start + n) of tile t,
// held in registers (ITEMS per thread, all loads in flight together); shared
// memory holds the bucketed copy (kb, vb) and the buckets. load(i) gives
// entry i as (depth key, splat id); the sorted splat ids go to
// ids[start, start + n) (and t to tids_out there). Every load completes
// before the first write, so the input may be (keys_tmp, ids) themselves.
template <uint32_t MAXN, uint32_t BINS, uint32_t THREADS, typename Load>
__device__ void sort_range_shared(uint32_t t, uint32_t start, uint32_t n, Load load, uint2* pairs, uint32_t* ids,
                                  uint32_t* tids_out, uint32_t* keys_tmp, uint32_t* sm) {
    constexpr uint32_t ITEMS = MAXN / THREADS;
    constexpr uint32_t WARPS = THREADS / 32;
    static_assert(MAXN % THREADS == 0 && BINS >= 256 + WARPS * 256, "sort shape");
    uint32_t* kb = sm;
    uint32_t* vb = kb + MAXN;
    uint32_t* bins = vb + MAXN;
    uint32_t* s_tmp = bins + BINS;
    const uint32_t tid = threadIdx.x;
    uint32_t k[ITEMS], v[ITEMS];
    uint32_t lo = 0xffffffffu, hi = 0;
#pragma unroll
    for (uint32_t j = 0; j < ITEMS; ++j) {
        const uint32_t i = tid + j * THREADS;
        k[j] = 0;
        v[j] = 0;
        if (i < n) {
            const uint2 p = load(i);
            k[j] = p.x;
            v[j] = p.y;
        }
    }
#pragma unroll
    for (uint32_t j = 0; j < ITEMS; ++j)
        if (tid + j * THREADS < n) {
            lo = min(lo, k[j]);
            hi = max(hi, k[j]);
        }
    uint32_t mn, mx;
    block_min_max<THREADS>(lo, hi, s_tmp, mn, mx);
    const BucketPlan bp = bucket_plan(n, mn, mx, BINS);
    bucket_clear<THREADS>(bins, bp.nbins);
    __syncthreads();
#pragma unroll
    for (uint32_t j = 0; j < ITEMS; ++j)
        if (tid + j * THREADS < n) atomicAdd(&bins[(k[j] - mn) >> bp.shift], 1u);
    __syncthreads();
    const uint32_t big = bucket_starts<THREADS>(bins, bp.nbins, s_tmp);
    if (big > kMaxBucket) {
        // Bunched keys: radix sort in the tile's global ranges.
        uint32_t* ka = keys_tmp + start;
        uint32_t* va = ids + start;
#pragma unroll
        for (uint32_t j = 0; j < ITEMS; ++j) {
            const uint32_t i = tid + j * THREADS;
            if (i < n) {
                ka[i] = k[j];
                va[i] = v[j];
            }
        }
        uint32_t* gkb = reinterpret_cast<uint32_t*>(pairs + start);
        radix_tile<THREADS>(ka, va, gkb, gkb + n, n, mn, mx, bins, s_tmp);
        if (tids_out)
            for (uint32_t i = tid; i < n; i += THREADS) tids_out[start + i] = t;
        return;
    }
#pragma unroll
    for (uint32_t j = 0; j < ITEMS; ++j)
        if (tid + j * THREADS < n) {
            const uint32_t pos = atomicAdd(&bins[(k[j] - mn) >> bp.shift], 1u);
            kb[pos] = k[j];
            vb[pos] = v[j];
        }
    __syncthreads();
    // bins[b] is now the end of bucket b.
    bucket_rank_store<THREADS>(kb, vb, bins, n, mn, bp.shift, ids + start, tids_out ? tids_out + start : nullptr,
                               t);
}

// One tile's whole list from the placed pairs.
template <uint32_t MAXN, uint32_t BINS, uint32_t THREADS>
__device__ void sort_tile_shared(uint32_t t, const uint32_t* __restrict__ tile_start, uint32_t capacity,
                                 uint2* pairs, uint32_t* ids, uint32_t* tids_out, uint32_t* keys_tmp,
                                 uint32_t* sm) {
    const uint32_t start = tile_start[t], end = tile_start[t + 1];
    const uint32_t n = end - start;
    // The size class and the capacity check before this launch keep both
    // conditions false; they guard the shared and global bounds regardless.
    if (n > MAXN || end > capacity || end < start) return;
    const uint2* pr = pairs + start;
    sort_range_shared<MAXN, BINS, THREADS>(t, start, n, [pr](uint32_t i) { return pr[i]; }, pairs, ids, tids_out,
                                           keys_tmp, sm);
}

// Persistent: each CTA takes the class's tiles in turn.
template <uint32_t MAXN, uint32_t BINS, uint32_t THREADS>
__global__ __launch_bounds__(THREADS) void tile_sort_kernel(const uint32_t* __restrict__ list,
                                                            const uint32_t* list_n,
                                                            const uint32_t* __restrict__ tile_start,
                                                            uint32_t capacity, uint2* pairs, uint32_t* ids,
                                                            uint32_t* tids_out, uint32_t* keys_tmp) {
    extern __shared__ __align__(16) uint32_t sm[];
    const uint32_t count = *list_n;
    for (uint32_t idx = blockIdx.x; idx < count; idx += gridDim.x) {
        sort_tile_shared<MAXN, BINS, THREADS>(list[idx], tile_start, capacity, pairs, ids, tids_out, keys_tmp, sm);
        __syncthreads();
    }
}

// Lists longer than the largest register-held class.
// Up to SMAX entries (shared form): the bucket sort with the bucketed copy
// (kb, vb) in shared memory; the entries are read from the tile's placed
// pairs (L2-resident) in each of the three passes instead of being held in
// registers, and SBINS buckets share the space. Longer lists, or bunched keys
// (a bucket past kMaxBucket), go to the global form: the entries stay in the
// tile's global ranges ((keys_tmp, ids) and the pair buffer as scratch), only
// the BINS buckets are in shared memory.
// Shared memory: [s_tmp: 128 words][buckets ...][kb: SMAX][vb: SMAX].
// The same for slots [start, start + n) of tile t with entry i given by
// load(i) (the placed pairs, or (keys_tmp, ids) themselves: the global form
// copies its input into (keys_tmp, ids) before it uses the pair slots
// [start, start + n) as scratch).
template <uint32_t BINS, uint32_t SBINS, uint32_t SMAX, uint32_t THREADS, typename Load>
__device__ void sort_range_global(uint32_t t, uint32_t start, uint32_t n, Load load, uint2* pairs, uint32_t* ids,
                                  uint32_t* tids_out, uint32_t* keys_tmp, uint32_t* sm) {
    static_assert(4 * (THREADS / 32) <= 128, "s_tmp size");
    uint32_t* s_tmp = sm;
    uint32_t* bins = sm + 128;
    const uint32_t tid = threadIdx.x;
    if (n <= SMAX) {
        uint32_t* kb = bins + SBINS;
        uint32_t* vb = kb + SMAX;
        uint32_t lo = 0xffffffffu, hi = 0;
        for (uint32_t i = tid; i < n; i += THREADS) {
            const uint32_t k = load(i).x;
            lo = min(lo, k);
            hi = max(hi, k);
        }
        uint32_t mn, mx;
        block_min_max<THREADS>(lo, hi, s_tmp, mn, mx);
        const BucketPlan bp = bucket_plan(n, mn, mx, SBINS);
        bucket_clear<THREADS>(bins, bp.nbins);
        __syncthreads();
        for (uint32_t i = tid; i < n; i += THREADS) atomicAdd(&bins[(load(i).x - mn) >> bp.shift], 1u);
        __syncthreads();
        const uint32_t big = bucket_starts<THREADS>(bins, bp.nbins, s_tmp);
        if (big <= kMaxBucket) {
            for (uint32_t i = tid; i < n; i += THREADS) {
                const uint2 q = load(i);
                const uint32_t pos = atomicAdd(&bins[(q.x - mn) >> bp.shift], 1u);
                kb[pos] = q.x;
                vb[pos] = q.y;
            }
            __syncthreads();
            bucket_rank_store<THREADS>(kb, vb, bins, n, mn, bp.shift, ids + start,
                                       tids_out ? tids_out + start : nullptr, t);
            return;
        }
        // Bunched keys: the global form below (its first loop reads the
        // pairs again).
        __syncthreads();
    }
    uint32_t* ka = keys_tmp + start;
    uint32_t* va = ids + start;
    uint32_t* kb = reinterpret_cast<uint32_t*>(pairs + start);
    uint32_t* vb = kb + n;
    uint32_t lo = 0xffffffffu, hi = 0;
    for (uint32_t i = tid; i < n; i += THREADS) {
        const uint2 p = load(i);
        ka[i] = p.x;
        va[i] = p.y;
        lo = min(lo, p.x);
        hi = max(hi, p.x);
    }
    uint32_t mn, mx;
    block_min_max<THREADS>(lo, hi, s_tmp, mn, mx);  // its barriers also order the copies above
    const BucketPlan bp = bucket_plan(n, mn, mx, BINS);
    bucket_clear<THREADS>(bins, bp.nbins);
    __syncthreads();
    for (uint32_t i = tid; i < n; i += THREADS) atomicAdd(&bins[(ka[i] - mn) >> bp.shift], 1u);
    __syncthreads();
    const uint32_t big = bucket_starts<THREADS>(bins, bp.nbins, s_tmp);
    if (big > kMaxBucket) {
        radix_tile<THREADS>(ka, va, kb, vb, n, mn, mx, bins, s_tmp);
        if (tids_out)
            for (uint32_t i = tid; i < n; i += THREADS) tids_out[start + i] = t;
        return;
    }
    for (uint32_t i = tid; i < n; i += THREADS) {
        const uint32_t pos = atomicAdd(&bins[(ka[i] - mn) >> bp.shift], 1u);
        kb[pos] = ka[i];
        vb[pos] = va[i];
    }
    __syncthreads();
    bucket_rank_store<THREADS>(kb, vb, bins, n, mn, bp.shift, va, tids_out ? tids_out + start : nullptr, t);
}

template <uint32_t BINS, uint32_t SBINS, uint32_t SMAX, uint32_t THREADS>
__device__ void sort_tile_global(uint32_t t, const uint32_t* __restrict__ tile_start, uint32_t capacity,
                                 uint2* pairs, uint32_t* ids, uint32_t* tids_out, uint32_t* keys_tmp,
                                 uint32_t* sm) {
    const uint32_t start = tile_start[t], end = tile_start[t + 1];
    if (end > capacity || end < start) return;
    const uint2* pr = pairs + start;
    sort_range_global<BINS, SBINS, SMAX, THREADS>(t, start, end - start, [pr](uint32_t i) { return pr[i]; }, pairs,
                                                  ids, tids_out, keys_tmp, sm);
}

// taken (may be null): entries of the class list the segmented sort took.
template <uint32_t BINS, uint32_t SBINS, uint32_t SMAX, uint32_t THREADS>
__global__ __launch_bounds__(THREADS, 1) void tile_sort_global_kernel(const uint32_t* __restrict__ list,
                                                                   const uint32_t* list_n,
                                                                   const uint32_t* __restrict__ tile_start,
                                                                   uint32_t capacity, uint2* pairs, uint32_t* ids,
                                                                   uint32_t* tids_out, uint32_t* keys_tmp,
                                                                   const uint32_t* taken) {
    extern __shared__ __align__(16) uint32_t sm[];
    const uint32_t count = *list_n;
    for (uint32_t idx = blockIdx.x; idx < count; idx += gridDim.x) {
        if (taken && taken[idx]) continue;  // uniform
        sort_tile_global<BINS, SBINS, SMAX, THREADS>(list[idx], tile_start, capacity, pairs, ids, tids_out,
                                                     keys_tmp, sm);
        __syncthreads();
    }
}

// Lists of up to 64 entries: one warp per tile, the 64-bit (key, id) values
// two per lane, a bitonic network over lanes (shuffles) and the lane's two
// slots; 8 tiles per 256-thread CTA, persistent over the class's tiles.
__global__ __launch_bounds__(256) void tile_sort_warp_kernel(const uint32_t* __restrict__ list,
                                                             const uint32_t* list_n,
                                                             const uint32_t* __restrict__ tile_start,
                                                             uint32_t capacity, uint2* pairs, uint32_t* ids,
                                                             uint32_t* tids_out, uint32_t*) {
    const uint32_t lane = threadIdx.x & 31u, wib = threadIdx.x >> 5;
    const uint32_t count = *list_n;
    for (uint32_t idx = blockIdx.x * 8u + wib; idx < count; idx += gridDim.x * 8u) {
        const uint32_t t = list[idx];
        const uint32_t start = tile_start[t], end = tile_start[t + 1];
        const uint32_t n = end - start;
        // The class and the capacity clamp keep these false (warp-uniform).
        if (n > 64 || end > capacity || end < start) continue;
        unsigned long long v0 = ~0ull, v1 = ~0ull;
        if (lane < n) {
            const uint2 p = pairs[start + lane];
            v0 = ((unsigned long long)p.x << 32) | p.y;
        }
        if (lane + 32 < n) {
            const uint2 p = pairs[start + lane + 32];
            v1 = ((unsigned long long)p.x << 32) | p.y;
        }
#pragma unroll
        for (uint32_t k = 2; k <= 64; k <<= 1) {
#pragma unroll
            for (uint32_t j = k >> 1; j > 0; j >>= 1) {
                if (j == 32) {
                    // Element lane against element lane + 32, ascending.
                    const unsigned long long lo = min(v0, v1), hi = max(v0, v1);
                    v0 = lo;
                    v1 = hi;
                } else {
                    const unsigned long long p0 = __shfl_xor_sync(0xffffffffu, v0, j);
                    const unsigned long long p1 = __shfl_xor_sync(0xffffffffu, v1, j);
                    const bool lower = (lane & j) == 0;
                    const bool asc0 = (lane & k) == 0, asc1 = ((lane + 32u) & k) == 0;
                    v0 = (lower == asc0) ? min(v0, p0) : max(v0, p0);
                    v1 = (lower == asc1) ? min(v1, p1) : max(v1, p1);
                }
            }
        }
        if (lane < n) {
            ids[start + lane] = (uint32_t)v0;
            if (tids_out) tids_out[start + lane] = t;
        }
        if (lane + 32 < n) {
            ids[start + lane + 32] = (uint32_t)v1;
            if (tids_out) tids_out[start + lane + 32] = t;
        }
    }
}

template <uint32_t MAXN, uint32_t BINS, uint32_t THREADS>
constexpr size_t sort_smem() {
    return (2ull * MAXN + BINS + 4 * (THREADS / 32)) * 4;
}

// Size classes (longest list): a warp per tile up to 64 entries, then the
// shared-memory bucket sorts (entries, buckets, threads); longer lists take
// the global form.
constexpr uint32_t kClassWarp = 64, kClassS = 512, kClass0 = 2048, kClassM = 4096, kClass1 = 6144,
                   kClass2 = kBinSharedMax;
constexpr uint32_t kBinsS = 2304, kBins0 = 4096, kBinsM = 8192, kBins1 = 8192, kBins2 = 16384, kBinsGiant = 32768;
// The longest lists: up to kGiantShared entries sorted in shared memory
// (8448 buckets, two 24576-entry arrays), longer ones with 32768 buckets over
// global scratch; 1024 threads, one CTA per SM.
constexpr uint32_t kThreadsGiant = 1024, kBinsGiantShared = 8448, kGiantShared = 24576;
constexpr size_t kGiantSmem = std::max<size_t>((128 + kBinsGiant) * 4, (128 + kBinsGiantShared + 2 * kGiantShared) * 4);
static_assert(kGiantSmem <= 232448, "shared memory per block");
constexpr uint32_t kThreadsS = 256, kThreads0 = 256, kThreadsM = 512, kThreads1 = 512, kThreads2 = 1024;
static_assert(sort_smem<kClass2, kBins2, kThreads2>() <= 227 * 1024, "per-tile sort exceeds shared memory");
static_assert(kSortClasses == 7, "class table");

// ---- segmented sort of the longest lists
//
// One CTA sorting a list of 10^5 entries takes milliseconds. Lists of the
// longest class past kGiantMinList entries (the first GiantState::lists of
// them) are instead sorted over all SMs:
//   0. giant_select (one CTA): picks those lists, gives each its first chunk
//      of kGiantChunk entries in one numbering over the picked lists, resets
//      their key ranges and marks them taken for the one-CTA form.
//   1. giant_minmax: the key range of each picked list (CTAs take chunks
//      round-robin; each finds its list in a shared copy of the chunk bases);
//      the lists' bucket counts are cleared on the way.
//   2. giant_hist: a kGiantBins-bucket histogram of (key - min) >> shift per
//      list (monotone in the key).
//   3. giant_plan (a CTA per list): the buckets' exclusive prefix (their
//      first slots) and the segments: runs of buckets whose first slot has
//      the same quotient by kGiantSegTarget. Segments are contiguous in key,
//      so the list sorted is its segments sorted, one after the other.
//   4. giant_scatter: each entry to its bucket's slots in (keys_tmp, ids).
//   5. giant_seg_sort: each segment of up to kClass1 entries sorted by one
//      CTA in shared memory (entries in registers); giant_seg_big: longer
//      ones (bunched keys) by the global form; ids and tile ids in place.
// Every list comes out in the same total (key, id) order as a sort of the
// whole list, so the result is bit-identical whichever form sorted it.

constexpr uint32_t kGiantThreads = 256, kGiantItems = 8, kGiantChunk = kGiantThreads * kGiantItems;
constexpr uint32_t kGiantPlanThreads = 1024;
static_assert(kGiantBins == 2 * kGiantPlanThreads, "two buckets per plan thread");
static_assert(kGiantMinList >= kClass2, "the segmented lists belong to the longest class");

__device__ __forceinline__ uint32_t giant_shift(uint32_t mn, uint32_t mx) {
    const uint32_t range = mx - mn;
    const uint32_t rbits = range == 0 ? 0u : 32u - __clz(range);
    constexpr uint32_t lbits = 11;  // log2(kGiantBins)
    static_assert((1u << lbits) == kGiantBins, "bucket bits");
    return rbits > lbits ? rbits - lbits : 0u;
}

__device__ __forceinline__ uint32_t giant_bucket(uint32_t k, uint32_t mn, uint32_t shift) {
    return min((k - mn) >> shift, kGiantBins - 1);
}

// Block-wide exclusive scan of one value per thread; s32 holds 32 words.
// Returns the exclusive prefix; total gets the sum (uniform).
template <uint32_t THREADS>
__device__ __forceinline__ uint32_t block_scan(uint32_t x, uint32_t* s32, uint32_t& total) {
    constexpr uint32_t WARPS = THREADS / 32;
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    uint32_t incl = x;
#pragma unroll
    for (uint32_t d = 1; d < 32; d <<= 1) {
        const uint32_t v = __shfl_up_sync(0xffffffffu, incl, d);
        if (lane >= d) incl += v;
    }
    __syncthreads();
    if (lane == 31) s32[warp] = incl;
    __syncthreads();
    uint32_t wbase = 0, tot = 0;
    for (uint32_t w = 0; w < WARPS; ++w) {
        const uint32_t v = s32[w];
        if (w < warp) wbase += v;
        tot += v;
    }
    total = tot;
    return wbase + incl - x;
}

__global__ __launch_bounds__(1024) void giant_select_kernel(const uint32_t* __restrict__ list, const uint32_t* list_n,
                                                            const uint32_t* __restrict__ tile_start,
                                                            uint32_t capacity, GiantState gs) {
    __shared__ uint32_t s32[32];
    const uint32_t count = *list_n;
    const uint32_t tid = threadIdx.x;
    uint32_t picked = 0, chunks = 0;
    for (uint32_t i0 = 0; i0 < count; i0 += 1024) {
        const uint32_t idx = i0 + tid;
        uint32_t t = 0, start = 0, n = 0;
        bool big = false;
        if (idx < count) {
            t = list[idx];
            start = tile_start[t];
            const uint32_t end = tile_start[t + 1];
            n = end - start;
            big = end <= capacity && end >= start && n > kGiantMinList;
        }
        uint32_t nbig;
        const uint32_t r = picked + block_scan<1024>(big ? 1u : 0u, s32, nbig);
        const bool take = big && r < gs.lists;
        const uint32_t nch = take ? (n + kGiantChunk - 1) / kGiantChunk : 0u;
        uint32_t tch;
        const uint32_t cb = chunks + block_scan<1024>(nch, s32, tch);
        if (idx < count) gs.taken[idx] = take ? 1u : 0u;
        if (take) {
            gs.sel[r] = make_uint4(t, start, n, cb);
            gs.mm[2 * r] = 0xffffffffu;
            gs.mm[2 * r + 1] = 0u;
        }
        picked += nbig;
        chunks += tch;
    }
    if (tid == 0) {
        gs.ctrl[0] = min(picked, gs.lists);
        gs.ctrl[1] = chunks;
        gs.ctrl[2] = 0;
        gs.ctrl[3] = 0;
    }
}

// The picked lists' first chunks, in shared memory (s_cb[lists] = chunks);
// returns the picked list count. s_cb holds kGiantMaxLists + 1 words.
__device__ __forceinline__ uint32_t giant_load_bases(const GiantState& gs, uint32_t* s_cb, uint32_t& chunks) {
    const uint32_t m = min(gs.ctrl[0], gs.lists);
    chunks = gs.ctrl[1];
    for (uint32_t r = threadIdx.x; r < m; r += blockDim.x) s_cb[r] = gs.sel[r].w;
    if (threadIdx.x == 0) s_cb[m] = chunks;
    __syncthreads();
    return m;
}

// The picked list holding global chunk g, searching forward from r (the
// chunks a CTA takes rise, so its search only moves forward).
__device__ __forceinline__ uint32_t giant_list_of(const uint32_t* s_cb, uint32_t m, uint32_t r, uint32_t g) {
    while (r + 1 < m && s_cb[r + 1] <= g) ++r;
    return r;
}

__global__ __launch_bounds__(kGiantThreads) void giant_minmax_kernel(const uint2* __restrict__ pairs, GiantState gs) {
    __shared__ uint32_t s_cb[kGiantMaxLists + 1];
    __shared__ uint32_t s_tmp[2 * (kGiantThreads / 32)];
    uint32_t chunks;
    const uint32_t m = giant_load_bases(gs, s_cb, chunks);
    const uint32_t tid = threadIdx.x;
    // Clear the picked lists' bucket counts.
    const size_t words = (size_t)m * kGiantBins;
    for (size_t b = (size_t)blockIdx.x * kGiantThreads + tid; b < words; b += (size_t)gridDim.x * kGiantThreads)
        gs.hist[b] = 0;
    uint32_t r = 0;
    for (uint32_t g = blockIdx.x; g < chunks; g += gridDim.x) {
        r = giant_list_of(s_cb, m, r, g);
        const uint4 sl = gs.sel[r];
        const uint32_t c = g - sl.w;
        uint32_t lo = 0xffffffffu, hi = 0;
#pragma unroll
        for (uint32_t j = 0; j < kGiantItems; ++j) {
            const uint32_t i = c * kGiantChunk + j * kGiantThreads + tid;
            if (i < sl.z) {
                const uint32_t k = pairs[sl.y + i].x;
                lo = min(lo, k);
                hi = max(hi, k);
            }
        }
        uint32_t mn, mx;
        block_min_max<kGiantThreads>(lo, hi, s_tmp, mn, mx);
        if (tid == 0) {
            atomicMin(gs.mm + 2 * r, mn);
            atomicMax(gs.mm + 2 * r + 1, mx);
        }
    }
}

__global__ __launch_bounds__(kGiantThreads) void giant_hist_kernel(const uint2* __restrict__ pairs, GiantState gs) {
    __shared__ uint32_t s_cb[kGiantMaxLists + 1];
    __shared__ uint32_t s_h[kGiantBins];
    uint32_t chunks;
    const uint32_t m = giant_load_bases(gs, s_cb, chunks);
    const uint32_t tid = threadIdx.x;
    for (uint32_t b = tid; b < kGiantBins; b += kGiantThreads) s_h[b] = 0;
    __syncthreads();
    uint32_t r = 0;
    for (uint32_t g = blockIdx.x; g < chunks; g += gridDim.x) {
        r = giant_list_of(s_cb, m, r, g);
        const uint4 sl = gs.sel[r];
        const uint32_t c = g - sl.w;
        const uint32_t mn = gs.mm[2 * r], shift = giant_shift(mn, gs.mm[2 * r + 1]);
#pragma unroll
        for (uint32_t j = 0; j < kGiantItems; ++j) {
            const uint32_t i = c * kGiantChunk + j * kGiantThreads + tid;
            if (i < sl.z) atomicAdd(&s_h[giant_bucket(pairs[sl.y + i].x, mn, shift)], 1u);
        }
        __syncthreads();
        uint32_t* row = gs.hist + (size_t)r * kGiantBins;
        for (uint32_t b = tid; b < kGiantBins; b += kGiantThreads) {
            const uint32_t v = s_h[b];
            if (v) {
                atomicAdd(row + b, v);
                s_h[b] = 0;
            }
        }
        __syncthreads();
    }
}

// A CTA per picked list (persistent). ctrl[2] counts the segments of up to
// kClass1 entries (filed from the front of gs.segs), ctrl[3] the longer ones
// (filed from the back).
__global__ __launch_bounds__(kGiantPlanThreads) void giant_plan_kernel(GiantState gs) {
    __shared__ uint32_t s_ex[kGiantBins + 1];
    __shared__ uint32_t s_off[kGiantBins], s_end[kGiantBins];
    __shared__ uint32_t s32[32];
    const uint32_t m = min(gs.ctrl[0], gs.lists);
    const uint32_t tid = threadIdx.x;
    for (uint32_t r = blockIdx.x; r < m; r += gridDim.x) {
        const uint4 sl = gs.sel[r];
        uint32_t* row = gs.hist + (size_t)r * kGiantBins;
        const uint32_t b0 = 2 * tid, b1 = b0 + 1;
        const uint32_t c0 = row[b0], c1 = row[b1];
        uint32_t total;
        const uint32_t e0 = block_scan<kGiantPlanThreads>(c0 + c1, s32, total);
        const uint32_t e1 = e0 + c0;
        row[b0] = e0;
        row[b1] = e1;
        s_ex[b0] = e0;
        s_ex[b1] = e1;
        if (tid == 0) s_ex[kGiantBins] = total;
        __syncthreads();
        const uint32_t T = kGiantSegTarget;
        // Bucket b starts a run when its first slot's quotient differs from
        // the previous bucket's.
        const bool f0 = b0 == 0 || e0 / T != s_ex[b0 - 1] / T;
        const bool f1 = e1 / T != e0 / T;
        uint32_t nruns;
        const uint32_t r0 = block_scan<kGiantPlanThreads>((uint32_t)f0 + (uint32_t)f1, s32, nruns);
        // Run of each bucket: the starts up to and including it, minus one.
        const uint32_t ri0 = r0 + (uint32_t)f0 - 1u, ri1 = ri0 + (uint32_t)f1;
        if (f0) s_off[ri0] = e0;
        if (f1) s_off[ri1] = e1;
        // Bucket b ends its run when it is the last bucket or b + 1 starts one.
        const bool l1 = b1 == kGiantBins - 1 || s_ex[b1 + 1] / T != e1 / T;
        if (f1) s_end[ri0] = e1;
        if (l1) s_end[ri1] = s_ex[b1 + 1];
        __syncthreads();
        // total == entries always (every chunk was counted); the test guards
        // the scatter's slots regardless.
        if (total == sl.z)
            for (uint32_t q = tid; q < nruns; q += kGiantPlanThreads) {
                const uint32_t off = s_off[q], len = s_end[q] - off;
                if (len == 0) continue;
                const uint32_t slot = len <= kClass1 ? atomicAdd(gs.ctrl + 2, 1u)
                                                     : gs.seg_cap - 1u - atomicAdd(gs.ctrl + 3, 1u);
                if (slot < gs.seg_cap) gs.segs[slot] = make_uint4(sl.x, sl.y + off, len, 0u);
            }
        __syncthreads();
    }
}

__global__ __launch_bounds__(kGiantThreads) void giant_scatter_kernel(const uint2* __restrict__ pairs, GiantState gs,
                                                                      uint32_t* keys_tmp, uint32_t* ids) {
    __shared__ uint32_t s_cb[kGiantMaxLists + 1];
    __shared__ uint32_t s_cnt[kGiantBins], s_base[kGiantBins];
    uint32_t chunks;
    const uint32_t m = giant_load_bases(gs, s_cb, chunks);
    const uint32_t tid = threadIdx.x;
    for (uint32_t b = tid; b < kGiantBins; b += kGiantThreads) s_cnt[b] = 0;
    __syncthreads();
    uint32_t r = 0;
    for (uint32_t g = blockIdx.x; g < chunks; g += gridDim.x) {
        r = giant_list_of(s_cb, m, r, g);
        const uint4 sl = gs.sel[r];
        const uint32_t c = g - sl.w;
        const uint32_t mn = gs.mm[2 * r], shift = giant_shift(mn, gs.mm[2 * r + 1]);
        uint32_t* row = gs.hist + (size_t)r * kGiantBins;
        uint32_t k[kGiantItems], v[kGiantItems], q[kGiantItems];
#pragma unroll
        for (uint32_t j = 0; j < kGiantItems; ++j) {
            const uint32_t i = c * kGiantChunk + j * kGiantThreads + tid;
            q[j] = 0xffffffffu;
            if (i < sl.z) {
                const uint2 p = pairs[sl.y + i];
                k[j] = p.x;
                v[j] = p.y;
                q[j] = atomicAdd(&s_cnt[giant_bucket(p.x, mn, shift)], 1u);
            }
        }
        __syncthreads();
        for (uint32_t b = tid; b < kGiantBins; b += kGiantThreads) {
            const uint32_t cnt = s_cnt[b];
            if (cnt) {
                s_base[b] = atomicAdd(row + b, cnt);
                s_cnt[b] = 0;
            }
        }
        __syncthreads();
#pragma unroll
        for (uint32_t j = 0; j < kGiantItems; ++j)
            if (q[j] != 0xffffffffu) {
                const uint32_t pos = s_base[giant_bucket(k[j], mn, shift)] + q[j];
                if (pos < sl.z) {
                    keys_tmp[sl.y + pos] = k[j];
                    ids[sl.y + pos] = v[j];
                }
            }
    }
}

__global__ __launch_bounds__(kThreads1) void giant_seg_sort_kernel(GiantState gs, uint2* pairs, uint32_t* ids,
                                                                   uint32_t* tids_out, uint32_t* keys_tmp) {
    extern __shared__ __align__(16) uint32_t sm[];
    const uint32_t count = min(gs.ctrl[2], gs.seg_cap);
    for (uint32_t i = blockIdx.x; i < count; i += gridDim.x) {
        const uint4 sg = gs.segs[i];
        if (sg.z > kClass1) continue;
        const uint32_t* kk = keys_tmp + sg.y;
        const uint32_t* vv = ids + sg.y;
        sort_range_shared<kClass1, kBins1, kThreads1>(
            sg.x, sg.y, sg.z, [kk, vv](uint32_t j) { return make_uint2(kk[j], vv[j]); }, pairs, ids, tids_out,
            keys_tmp, sm);
        __syncthreads();
    }
}

__global__ __launch_bounds__(kThreadsGiant, 1) void giant_seg_big_kernel(GiantState gs, uint2* pairs, uint32_t* ids,
                                                                         uint32_t* tids_out, uint32_t* keys_tmp) {
    extern __shared__ __align__(16) uint32_t sm[];
    const uint32_t count = min(gs.ctrl[3], gs.seg_cap);
    for (uint32_t i = blockIdx.x; i < count; i += gridDim.x) {
        const uint4 sg = gs.segs[gs.seg_cap - 1u - i];
        const uint32_t* kk = keys_tmp + sg.y;
        const uint32_t* vv = ids + sg.y;
        sort_range_global<kBinsGiant, kBinsGiantShared, kGiantShared, kThreadsGiant>(
            sg.x, sg.y, sg.z, [kk, vv](uint32_t j) { return make_uint2(kk[j], vv[j]); }, pairs, ids, tids_out,
            keys_tmp, sm);
        __syncthreads();
    }
}

// grid: the class's tile count when the host knows it, else an upper bound;
// capped at the CTAs resident at once (the kernels loop over their tiles).
template <typename K>
cudaError_t launch_sort_kernel(K kernel, uint32_t threads, size_t smem, uint32_t grid, int sm_count,
                               const uint32_t* list, const uint32_t* list_n, const uint32_t* tile_start,
                               uint32_t capacity, uint2* pairs, uint32_t* ids, uint32_t* tids_out,
                               uint32_t* keys_tmp, cudaStream_t st) {
    if (grid == 0) return cudaSuccess;
    const uint32_t per_sm = std::max<uint32_t>(
        1u, std::min<uint32_t>(2048u / threads, (uint32_t)(233472 / (smem + 1024))));
    grid = std::min(grid, per_sm * (uint32_t)std::max(sm_count, 1));
    if (smem > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
    }
    kernel<<<grid, threads, smem, st>>>(list, list_n, tile_start, capacity, pairs, ids, tids_out, keys_tmp);
    note_launches(1);
    return cudaGetLastError();
}

cudaError_t smem_opt_in(const void* fn, size_t smem) {
    if (smem <= 48 * 1024) return cudaSuccess;
    return cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
}

}  // namespace

uint32_t bin_chunks(uint32_t n, int sm_count) {
    const uint32_t c = (uint32_t)std::max(1, 2 * sm_count);
    return std::max(1u, std::min(c, (n + 31) / 32));
}

uint32_t bin_chunk_size(uint32_t n, uint32_t chunks) { return ((n + chunks - 1) / chunks + 31) / 32 * 32; }

namespace {
uint32_t g_giant_max_lists = kGiantMaxLists;  // lowered only by sf_debug_giant_lists
}  // namespace

uint32_t giant_lists(uint32_t tiles) { return std::min(tiles, g_giant_max_lists); }

void set_giant_max_lists(uint32_t lists) { g_giant_max_lists = std::min(lists, kGiantMaxLists); }

uint32_t giant_seg_cap(uint32_t lists) { return (1u << 30) / kGiantSegTarget + lists + 1u; }

uint32_t bin_class_limit(int k) {
    const uint32_t lim[kSortClasses - 1] = {kClassWarp, kClassS, kClass0, kClassM, kClass1, kClass2};
    return k >= 0 && k < kSortClasses - 1 ? lim[k] : 0xffffffffu;
}

cudaError_t launch_bin_count(const uint2* bbox, uint32_t n, uint32_t tiles_x, uint32_t tiles, uint32_t chunks,
                             uint32_t* hist, cudaStream_t st) {
    const size_t smem = (size_t)tiles * 4;
    cudaError_t e = smem_opt_in((const void*)bin_count_kernel, smem);
    if (e != cudaSuccess) return e;
    e = launch_pdl(bin_count_kernel, chunks, kBinThreads, smem, st, bbox, n, bin_chunk_size(n, chunks), tiles_x,
                   tiles, hist);
    note_launches(1);
    return e;
}

cudaError_t launch_bin_colscan(uint32_t* hist, uint32_t chunks, uint32_t tiles, uint32_t* cnt, uint32_t* lists,
                               uint32_t* words, cudaStream_t st) {
    const ClassLimits lim{{kClassWarp, kClassS, kClass0, kClassM, kClass1, kClass2}};
    const cudaError_t e =
        launch_pdl(bin_colscan_kernel, (tiles + 31) / 32, dim3(32, 32), 0, st, hist, chunks, tiles, cnt, lists, words, lim);
    note_launches(1);
    return e;
}

cudaError_t launch_bin_place(const uint2* bbox, const uint32_t* depth_keys, uint32_t n, uint32_t tiles_x,
                             uint32_t tiles, uint32_t chunks, const uint32_t* hist, const uint32_t* tile_start,
                             uint32_t capacity, uint2* pairs, uint32_t* err, cudaStream_t st) {
    const size_t smem = (size_t)tiles * 4;
    cudaError_t e = smem_opt_in((const void*)bin_place_kernel, smem);
    if (e != cudaSuccess) return e;
    e = launch_pdl(bin_place_kernel, chunks, kBinThreads, smem, st, bbox, depth_keys, n, bin_chunk_size(n, chunks),
                   tiles_x, tiles, hist, tile_start, capacity, pairs, err);
    note_launches(1);
    return e;
}

namespace {

__global__ void clamp_count_kernel(const unsigned long long* total, uint32_t cap, uint32_t* n32, uint32_t* err) {
    pdl_trigger();
    pdl_wait();
    const unsigned long long t = *total;
    if (t > cap) atomicOr(err, SF_DEV_ERR_CAPACITY);
    *n32 = (uint32_t)(t < cap ? t : cap);
}

__global__ void save_words_kernel(const uint32_t* __restrict__ words, uint32_t* __restrict__ ring,
                                  uint32_t* counter, uint32_t ring_frames) {
    const uint32_t idx = *counter;
    if (idx < ring_frames)
        for (uint32_t k = 0; k < 16; ++k) ring[(size_t)idx * 16 + k] = words[k];
    *counter = idx + 1;
}

__global__ void clamp_starts_kernel(uint32_t* tile_start, uint32_t count, uint32_t cap) {
    pdl_trigger();
    pdl_wait();
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < count && tile_start[i] > cap) tile_start[i] = cap;
}

}  // namespace

cudaError_t launch_clamp_count(const unsigned long long* total, uint32_t cap, uint32_t* n32, uint32_t* err,
                               cudaStream_t st) {
    const cudaError_t e = launch_pdl(clamp_count_kernel, 1, 1, 0, st, total, cap, n32, err);
    note_launches(1);
    return e;
}

cudaError_t launch_save_words(const uint32_t* words, uint32_t* ring, uint32_t* counter, uint32_t ring_frames,
                              cudaStream_t st) {
    save_words_kernel<<<1, 1, 0, st>>>(words, ring, counter, ring_frames);
    note_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_clamp_starts(uint32_t* tile_start, uint32_t count, uint32_t cap, cudaStream_t st) {
    const cudaError_t e = launch_pdl(clamp_starts_kernel, (count + 255) / 256, 256, 0, st, tile_start, count, cap);
    note_launches(1);
    return e;
}

cudaError_t sort_streams_create(SortStreams* ss) {
    for (int k = 0; k < 4; ++k) {
        cudaError_t e = cudaStreamCreateWithFlags(&ss->s[k], cudaStreamNonBlocking);
        if (e != cudaSuccess) return e;
    }
    for (int k = 0; k < 5; ++k) {
        cudaError_t e = cudaEventCreateWithFlags(&ss->e[k], cudaEventDisableTiming);
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

void sort_streams_destroy(SortStreams* ss) {
    for (int k = 0; k < 4; ++k) {
        if (ss->s[k]) cudaStreamDestroy(ss->s[k]);
        ss->s[k] = nullptr;
    }
    for (int k = 0; k < 5; ++k) {
        if (ss->e[k]) cudaEventDestroy(ss->e[k]);
        ss->e[k] = nullptr;
    }
}

namespace {

template <typename K>
cudaError_t smem_attr(K kernel, size_t smem) {
    if (smem <= 48 * 1024) return cudaSuccess;
    return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
}

// The longest class: the segmented sort for its lists past kGiantMinList
// entries (the first gs->lists of them), the one-CTA global form for the
// rest. grid: the class's tile count (or an upper bound); 0 leaves the class
// unsorted.
cudaError_t launch_giant_sorts(uint32_t grid, const uint32_t* list, const uint32_t* words,
                               const uint32_t* tile_start, uint32_t capacity, uint2* pairs, uint32_t* ids,
                               uint32_t* tids_out, uint32_t* keys_tmp, int sm_count, cudaStream_t st,
                               const GiantState* gs) {
    if (grid == 0) return cudaSuccess;
    const uint32_t* n = words + 8 + (kSortClasses - 1);
    const uint32_t sms = (uint32_t)std::max(sm_count, 1);
    auto global_form = tile_sort_global_kernel<kBinsGiant, kBinsGiantShared, kGiantShared, kThreadsGiant>;
    cudaError_t e = smem_attr(global_form, kGiantSmem);
    if (e != cudaSuccess) return e;
    const bool seg = gs && gs->sel && gs->lists > 0;
    if (seg) {
        const GiantState g = *gs;
        const uint32_t wide = 4 * sms;
        giant_select_kernel<<<1, 1024, 0, st>>>(list, n, tile_start, capacity, g);
        giant_minmax_kernel<<<wide, kGiantThreads, 0, st>>>(pairs, g);
        giant_hist_kernel<<<wide, kGiantThreads, 0, st>>>(pairs, g);
        giant_plan_kernel<<<std::min(std::min(grid, g.lists), 2 * sms), kGiantPlanThreads, 0, st>>>(g);
        giant_scatter_kernel<<<wide, kGiantThreads, 0, st>>>(pairs, g, keys_tmp, ids);
        constexpr size_t seg_smem = sort_smem<kClass1, kBins1, kThreads1>();
        if ((e = smem_attr(giant_seg_sort_kernel, seg_smem)) != cudaSuccess) return e;
        giant_seg_sort_kernel<<<2 * sms, kThreads1, seg_smem, st>>>(g, pairs, ids, tids_out, keys_tmp);
        if ((e = smem_attr(giant_seg_big_kernel, kGiantSmem)) != cudaSuccess) return e;
        giant_seg_big_kernel<<<sms, kThreadsGiant, kGiantSmem, st>>>(g, pairs, ids, tids_out, keys_tmp);
        note_launches(7);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
    }
    global_form<<<std::min(grid, sms), kThreadsGiant, kGiantSmem, st>>>(list, n, tile_start, capacity, pairs, ids,
                                                                         tids_out, keys_tmp,
                                                                         seg ? gs->taken : nullptr);
    note_launches(1);
    return cudaGetLastError();
}

}  // namespace

cudaError_t launch_tile_sorts(const uint32_t grids[kSortClasses], const uint32_t* lists, const uint32_t* words,
                              uint32_t tiles, const uint32_t* tile_start, uint32_t capacity, uint2* pairs,
                              uint32_t* ids, uint32_t* tids_out, uint32_t* keys_tmp, int sm_count,
                              cudaStream_t st, const SortStreams* side, const GiantState* gs) {
    cudaError_t e;
    // Each form reads and overwrites only its own tiles' ranges, so the
    // classes may run concurrently.
    cudaStream_t s1 = st, s2 = st, s3 = st, s4 = st;
    if (side && side->s[0]) {
        if ((e = cudaEventRecord(side->e[0], st)) != cudaSuccess) return e;
        for (int k = 0; k < 4; ++k)
            if ((e = cudaStreamWaitEvent(side->s[k], side->e[0], 0)) != cudaSuccess) return e;
        s1 = side->s[0];
        s2 = side->s[1];
        s3 = side->s[2];
        s4 = side->s[3];
    }
    auto L = [&](int k) { return lists + (size_t)k * tiles; };
    auto N = [&](int k) { return words + 8 + k; };
    e = launch_giant_sorts(grids[6], L(6), words, tile_start, capacity, pairs, ids, tids_out, keys_tmp, sm_count,
                           s3, gs);
    if (e != cudaSuccess) return e;
    e = launch_sort_kernel(tile_sort_kernel<kClass1, kBins1, kThreads1>, kThreads1,
                           sort_smem<kClass1, kBins1, kThreads1>(), grids[4], sm_count, L(4), N(4), tile_start,
                           capacity, pairs, ids, tids_out, keys_tmp, s1);
    if (e != cudaSuccess) return e;
    e = launch_sort_kernel(tile_sort_kernel<kClass2, kBins2, kThreads2>, kThreads2,
                           sort_smem<kClass2, kBins2, kThreads2>(), grids[5], sm_count, L(5), N(5), tile_start,
                           capacity, pairs, ids, tids_out, keys_tmp, s2);
    if (e != cudaSuccess) return e;
    e = launch_sort_kernel(tile_sort_kernel<kClassM, kBinsM, kThreadsM>, kThreadsM,
                           sort_smem<kClassM, kBinsM, kThreadsM>(), grids[3], sm_count, L(3), N(3), tile_start,
                           capacity, pairs, ids, tids_out, keys_tmp, s4);
    if (e != cudaSuccess) return e;
    e = launch_sort_kernel(tile_sort_warp_kernel, 256, 0, (grids[0] + 7) / 8, sm_count, L(0), N(0), tile_start,
                           capacity, pairs, ids, tids_out, keys_tmp, s2);
    if (e != cudaSuccess) return e;
    e = launch_sort_kernel(tile_sort_kernel<kClassS, kBinsS, kThreadsS>, kThreadsS,
                           sort_smem<kClassS, kBinsS, kThreadsS>(), grids[1], sm_count, L(1), N(1), tile_start,
                           capacity, pairs, ids, tids_out, keys_tmp, s3);
    if (e != cudaSuccess) return e;
    e = launch_sort_kernel(tile_sort_kernel<kClass0, kBins0, kThreads0>, kThreads0,
                           sort_smem<kClass0, kBins0, kThreads0>(), grids[2], sm_count, L(2), N(2), tile_start,
                           capacity, pairs, ids, tids_out, keys_tmp, st);
    if (e != cudaSuccess) return e;
    if (side && side->s[0]) {
        for (int k = 0; k < 4; ++k) {
            if ((e = cudaEventRecord(side->e[1 + k], side->s[k])) != cudaSuccess) return e;
            if ((e = cudaStreamWaitEvent(st, side->e[1 + k], 0)) != cudaSuccess) return e;
        }
    }
    return cudaSuccess;
}

}  // namespace sfk
