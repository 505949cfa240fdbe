// Onesweep LSD radix sort and decoupled-look-back prefix scan (sm_100a).
//
// Replaces crates/sort/src/sort.rs (count_kernel + scan + scatter_plane_kernel
// per 6-bit digit, 3 launches a digit) and crates/sort/src/scan.rs
// (block_sums + scan_serial + apply_block_offsets). Design (Adinets & Merrill,
// "Onesweep: A Faster Least Significant Digit Radix Sort for GPUs", 2022):
//  * one upfront kernel reads the keys once and builds the 256-bin histogram
//    of every 8-bit digit position;
//  * one kernel per digit: a partition of 4096 keys (8192 from 2M keys on)
//    is ranked in registers and shared memory (stable warp ranking by one
//    ballot per digit bit), publishes its digit
//    counts, resolves its global digit offsets by decoupled look-back over the
//    preceding partitions, and scatters through shared memory so each digit's
//    run is written contiguously.
// Partition indices come from an atomic ticket in launch order, so a block
// only ever waits on blocks that already hold a ticket (forward progress).
// Every wait is bounded: after kSpinLimit polls the block records
// SF_DEV_ERR_TIMEOUT in the error word and carries on, so a lost predecessor
// can corrupt the result but never hang the GPU.
#include <cstdint>
#include <type_traits>
#include <string>
#include "sf_handles.h"

namespace sfk {

namespace {

// Digit width: 4 to 8 bits (a template parameter of the kernels); the
// scratch is laid out for the widest case, 256 bins, 4 passes of 32 bits.
constexpr int kRadixBits = 8;
constexpr int kRadix = 1 << kRadixBits;
constexpr int kHistWords = 1024;  // passes x bins <= 1024 for every width
constexpr int kThreads = 256;
constexpr int kItems = 16;
constexpr int kWarps = kThreads / 32;
// Digit passes: partitions of THREADS x 16 keys. The look-back chain across
// partitions bounds a large pass (a partition publishes its inclusive prefix
// only after its own look-back), so from kWidePassN keys on the partitions
// are 8192 keys of 512 threads (half the chain: 10M keys 0.47 -> 0.44 ms);
// smaller sorts keep 4096-key partitions of 256 threads, whose single
// partitions finish sooner (1k-500k keys 12-17% faster than the wide form).
// The keys and values staged for the scatter are dynamic shared memory.
constexpr uint32_t kWidePassN = 1u << 21;
constexpr int kMinPassTile = 256 * kItems;  // look-back space is sized for it
template <int THREADS>
constexpr size_t pass_smem() { return 2 * (size_t)THREADS * kItems * 4; }
constexpr uint32_t kFlagAgg = 1u << 30;
constexpr uint32_t kFlagPrefix = 2u << 30;
constexpr uint32_t kCountMask = (1u << 30) - 1u;
constexpr uint32_t kSpinLimit = 1u << 22;

// Test knobs of the look-back waits, set by sf_debug_lookback and passed to
// the kernels only by the standalone sort and scan entry points (the frame
// and round paths always pass zeros). spin_limit caps the polls of one wait
// (0: kSpinLimit). withhold = 1 keeps partition 0 of the scan and of every
// digit pass from publishing its status, a flag that nothing then sets: every
// later partition's wait runs out after spin_limit polls, records
// SF_DEV_ERR_TIMEOUT and returns, and the host reports SF_ERR_TIMEOUT. Every
// access stays inside the buffers either way; only the values are wrong.
LookbackKnobs g_test_knobs = {0u, 0u};

__device__ __forceinline__ uint32_t ld_relaxed(const uint32_t* p) {
    uint32_t v;
    asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_relaxed(uint32_t* p, uint32_t v) {
    asm volatile("st.relaxed.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ unsigned long long ld_relaxed64(const unsigned long long* p) {
    unsigned long long v;
    asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_relaxed64(unsigned long long* p, unsigned long long v) {
    asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

__device__ __forceinline__ uint32_t ld_status(const uint32_t* p) { return ld_relaxed(p); }
__device__ __forceinline__ unsigned long long ld_status(const unsigned long long* p) {
    return ld_relaxed64(p);
}

// Decoupled look-back from partition `part` over status words stat[p * stride]
// (flag in the top two bits: 0 = not ready, aggregate, inclusive prefix).
// kWindow predecessors are loaded at once, so a chain of aggregates costs one
// L2 round trip per kWindow partitions instead of one per partition. Returns
// the exclusive prefix. A poll that finds nothing new backs off with
// __nanosleep (32 ns, doubling to 256 ns), so waiting blocks leave issue
// slots and L2 bandwidth to the partitions still ranking (10M-key sorts
// 0.52 -> 0.49 ms); a wait that outlasts kSpinLimit polls (about a second
// with the naps) records SF_DEV_ERR_TIMEOUT and returns what it has.
constexpr int kWindow = 8;
template <typename W>
__device__ __forceinline__ W lookback_window(const W* stat, size_t stride, uint32_t part, W flag_prefix,
                                             W value_mask, uint32_t* err, uint32_t spin_limit) {
    W excl = 0;
    int64_t p = (int64_t)part - 1;
    uint32_t spins = 0, nap = 32;
    const uint32_t limit = spin_limit ? spin_limit : kSpinLimit;
    while (p >= 0) {
        W s[kWindow];
#pragma unroll
        for (int w = 0; w < kWindow; ++w)
            s[w] = (p - w >= 0) ? ld_status(stat + (size_t)(p - w) * stride) : flag_prefix;
        int used = 0;
        bool found = false;
        for (; used < kWindow; ++used) {
            const W flag = s[used] & ~value_mask;
            if (flag == 0) break;
            excl += s[used] & value_mask;
            if (flag == flag_prefix) {
                found = true;
                break;
            }
        }
        if (found) break;
        if (used == 0) {
            if (++spins > limit) {
                atomicOr(err, SF_DEV_ERR_TIMEOUT);
                break;
            }
            __nanosleep(nap);
            nap = min(nap * 2u, 256u);
        }
        p -= used;
    }
    return excl;
}

__device__ __forceinline__ uint32_t lanemask_lt() {
    uint32_t m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// Lanes holding the same BITS-bit digit (and the same validity) as this
// lane: one ballot per digit bit, inverted where this lane's bit is clear,
// ANDed. Fixed cost of BITS + 1 votes, far cheaper on this part than
// match.any.
template <int BITS>
__device__ __forceinline__ uint32_t match_digit(uint32_t d, bool valid) {
    uint32_t peers = __ballot_sync(0xffffffffu, valid);
    if (!valid) peers = ~peers;
#pragma unroll
    for (int b = 0; b < BITS; ++b) {
        const bool bit = (d >> b) & 1u;
        const uint32_t v = __ballot_sync(0xffffffffu, bit);
        peers &= bit ? v : ~v;
    }
    return peers;
}

__device__ __forceinline__ uint32_t load_n(const uint32_t* n_dev, uint32_t n_static) {
    return n_dev ? *n_dev : n_static;
}

// Upfront digit histograms: hist[pass * 2^BITS + digit] over all n keys.
template <int BITS>
__global__ __launch_bounds__(kThreads) void radix_histogram_kernel(
    const uint32_t* __restrict__ keys, const uint32_t* n_dev, uint32_t n_static,
    uint32_t num_passes, uint32_t bits, uint32_t* __restrict__ hist) {
    constexpr uint32_t R = 1u << BITS;
    __shared__ uint32_t s_hist[kHistWords];
    const uint32_t n = load_n(n_dev, n_static);
    for (uint32_t i = threadIdx.x; i < num_passes * R; i += kThreads) s_hist[i] = 0;
    __syncthreads();
    // Whole warps iterate together (the bound is rounded up) so that runs of
    // equal digits in neighbouring lanes are merged before the shared atomic:
    // emitted tile ids come in runs, and 32 lanes on one bin would otherwise
    // serialise. A lane whose digit differs from its left neighbour's adds the
    // length of its run.
    // Each warp takes 128 consecutive keys per step (4 loads in flight per
    // lane, each covering 32 consecutive keys across the lanes).
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t warp_global = (blockIdx.x * kThreads + threadIdx.x) >> 5;
    const uint32_t warps_total = (gridDim.x * kThreads) >> 5;
    for (uint32_t base = warp_global * 128u; base < n; base += warps_total * 128u) {
        uint32_t kk[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const uint32_t i = base + u * 32u + lane;
            kk[u] = i < n ? keys[i] : 0u;
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const bool valid = base + u * 32u + lane < n;
            for (uint32_t p = 0; p < num_passes; ++p) {
                const uint32_t shift = p * BITS;
                const uint32_t w = bits - shift < (uint32_t)BITS ? bits - shift : (uint32_t)BITS;
                const uint32_t d = valid ? ((kk[u] >> shift) & ((1u << w) - 1u)) : R;
                const uint32_t left = __shfl_up_sync(0xffffffffu, d, 1);
                const bool head = lane == 0 || left != d;
                const uint32_t heads = __ballot_sync(0xffffffffu, head);
                if (valid && head) {
                    const uint32_t above = heads & ~((2u << lane) - 1u);
                    const uint32_t next = above ? (uint32_t)(__ffs(above) - 1) : 32u;
                    atomicAdd(&s_hist[p * R + d], next - lane);
                }
            }
        }
    }
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < num_passes * R; i += kThreads)
        if (s_hist[i]) atomicAdd(&hist[i], s_hist[i]);
}

// One BITS-bit digit pass. `vals_iota` substitutes vals_in[i] = i.
template <int BITS, int THREADS>
__global__ __launch_bounds__(THREADS, THREADS >= 512 ? 2 : 4) void onesweep_pass_kernel(
    const uint32_t* __restrict__ keys_in, const uint32_t* __restrict__ vals_in,
    uint32_t* __restrict__ keys_out, uint32_t* __restrict__ vals_out, const uint32_t* n_dev,
    uint32_t n_static, uint32_t shift, uint32_t digit_mask, const uint32_t* __restrict__ pass_hist,
    uint32_t* lookback, uint32_t* ticket, uint32_t* err, int vals_iota, int write_keys, LookbackKnobs knobs) {
    constexpr uint32_t R = 1u << BITS;
    constexpr int kPassThreads = THREADS, kPassWarps = THREADS / 32, kPassTile = THREADS * kItems;
    __shared__ uint32_t s_part;
    __shared__ uint32_t s_warp_hist[kPassWarps][R];
    __shared__ uint32_t s_local_start[R];
    __shared__ uint32_t s_global_base[R];
    __shared__ uint32_t s_scan[kPassWarps];
    extern __shared__ __align__(16) uint32_t s_stage[];
    uint32_t* s_keys = s_stage;
    uint32_t* s_vals = s_stage + kPassTile;

    const uint32_t tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5;
    const uint32_t n = load_n(n_dev, n_static);
    const uint32_t num_parts = (n + kPassTile - 1) / kPassTile;
    if (tid == 0) s_part = atomicAdd(ticket, 1u);
    for (uint32_t i = tid; i < kPassWarps * R; i += kPassThreads) (&s_warp_hist[0][0])[i] = 0;
    __syncthreads();
    const uint32_t part = s_part;
    if (part >= num_parts) return;
    const uint32_t base = part * kPassTile;
    const uint32_t wbase = base + warp * (kItems * 32);

    // Keys and values are loaded together, before the ranking and the
    // look-back, so no global load waits behind them.
    uint32_t k[kItems], rank[kItems], vv[kItems];
#pragma unroll
    for (int i = 0; i < kItems; ++i) {
        const uint32_t idx = wbase + i * 32 + lane;
        k[i] = idx < n ? keys_in[idx] : 0u;
        vv[i] = idx < n ? (vals_iota ? idx : vals_in[idx]) : 0u;
    }
    // Stable warp ranking: items in index order, lanes in lane order.
    const uint32_t lt = lanemask_lt();
#pragma unroll
    for (int i = 0; i < kItems; ++i) {
        const uint32_t idx = wbase + i * 32 + lane;
        const bool valid = idx < n;
        const uint32_t d = valid ? ((k[i] >> shift) & digit_mask) : R;
        const uint32_t peers = match_digit<BITS>(d, valid);
        const uint32_t leader = __ffs(peers) - 1;
        uint32_t prev = 0;
        if (valid && lane == leader) {
            prev = s_warp_hist[warp][d];
            s_warp_hist[warp][d] = prev + __popc(peers);
        }
        prev = __shfl_sync(0xffffffffu, prev, leader);
        rank[i] = prev + __popc(peers & lt);
        __syncwarp();
    }
    __syncthreads();

    // Per digit: exclusive prefix over warps, block total, publish.
    uint32_t digit_total = 0;
    if (tid < R) {
        uint32_t sum = 0;
#pragma unroll
        for (int w = 0; w < kPassWarps; ++w) {
            const uint32_t c = s_warp_hist[w][tid];
            s_warp_hist[w][tid] = sum;
            sum += c;
        }
        digit_total = sum;
        if (part > 0 || !knobs.withhold)
            st_relaxed(&lookback[(size_t)part * R + tid], (part == 0 ? kFlagPrefix : kFlagAgg) | sum);
    }
    // Block exclusive scan of digit totals (digit order) -> local starts.
    {
        uint32_t v = digit_total;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t t = __shfl_up_sync(0xffffffffu, v, o);
            if (lane >= (uint32_t)o) v += t;
        }
        if (lane == 31) s_scan[warp] = v;
        __syncthreads();
        if (tid < 32) {
            uint32_t w = tid < (uint32_t)kPassWarps ? s_scan[tid] : 0u;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t t = __shfl_up_sync(0xffffffffu, w, o);
                if (lane >= (uint32_t)o) w += t;
            }
            if (tid < (uint32_t)kPassWarps) s_scan[tid] = w;
        }
        __syncthreads();
        if (tid < R) s_local_start[tid] = v - digit_total + (warp ? s_scan[warp - 1] : 0u);
    }
    // Global digit offsets of this pass (exclusive over digits of pass_hist).
    uint32_t gstart = 0;
    {
        const uint32_t h = tid < R ? pass_hist[tid] : 0u;
        uint32_t v = h;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t t = __shfl_up_sync(0xffffffffu, v, o);
            if (lane >= (uint32_t)o) v += t;
        }
        __syncthreads();
        if (lane == 31) s_scan[warp] = v;
        __syncthreads();
        if (tid < 32) {
            uint32_t w = tid < (uint32_t)kPassWarps ? s_scan[tid] : 0u;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t t = __shfl_up_sync(0xffffffffu, w, o);
                if (lane >= (uint32_t)o) w += t;
            }
            if (tid < (uint32_t)kPassWarps) s_scan[tid] = w;
        }
        __syncthreads();
        gstart = v - h + (warp ? s_scan[warp - 1] : 0u);
    }
    // Decoupled look-back, one digit per thread, kWindow predecessors per step.
    if (tid < R) {
        uint32_t excl = 0;
        if (part > 0) {
            excl = lookback_window<uint32_t>(lookback + tid, R, part, kFlagPrefix, kCountMask, err,
                                            knobs.spin_limit);
            st_relaxed(&lookback[(size_t)part * R + tid], kFlagPrefix | ((excl + digit_total) & kCountMask));
        }
        s_global_base[tid] = gstart + excl - s_local_start[tid];
    }
    __syncthreads();

    // Scatter into shared memory at the partition-local sorted position.
#pragma unroll
    for (int i = 0; i < kItems; ++i) {
        const uint32_t idx = wbase + i * 32 + lane;
        if (idx < n) {
            const uint32_t d = (k[i] >> shift) & digit_mask;
            const uint32_t pos = s_local_start[d] + s_warp_hist[warp][d] + rank[i];
            s_keys[pos] = k[i];
            s_vals[pos] = vv[i];
        }
    }
    __syncthreads();
    const uint32_t cnt = min((uint32_t)kPassTile, n - base);
    for (uint32_t j = tid; j < cnt; j += kPassThreads) {
        const uint32_t key = s_keys[j];
        const uint32_t d = (key >> shift) & digit_mask;
        const uint32_t out = s_global_base[d] + j;
        if (out >= n) continue;  // only after a timed-out look-back
        if (write_keys) keys_out[out] = key;
        vals_out[out] = s_vals[j];
    }
}

// The scan's look-back done by one whole warp: lane l reads the status of
// partition p - l (p the newest predecessor not yet summed), so one L2 round
// trip covers 32 predecessors. If some lane finds an inclusive prefix and
// every lane before it an aggregate, the warp sums those lanes and stops;
// otherwise it sums the aggregates before the first lane whose partition
// has published nothing and reads again from there, with the same backoff
// and bound as lookback_window. Lanes past partition 0 read a zero prefix.
// Returns the exclusive prefix in every lane.
__device__ unsigned long long lookback_warp64(const unsigned long long* stat, uint32_t part, uint32_t* err,
                                              uint32_t spin_limit, unsigned long long flag_prefix,
                                              unsigned long long value_mask) {
    const uint32_t lane = threadIdx.x & 31u;
    unsigned long long excl = 0;
    int64_t p = (int64_t)part - 1;
    uint32_t spins = 0, nap = 32;
    const uint32_t limit = spin_limit ? spin_limit : kSpinLimit;
    while (p >= 0) {
        const int64_t q = p - (int64_t)lane;
        const unsigned long long st = q >= 0 ? ld_relaxed64(stat + q) : flag_prefix;
        const unsigned long long flag = st & ~value_mask;
        const uint32_t not_ready = __ballot_sync(0xffffffffu, flag == 0);
        const uint32_t prefix = __ballot_sync(0xffffffffu, flag == flag_prefix);
        const uint32_t first_nr = not_ready ? (uint32_t)(__ffs(not_ready) - 1) : 32u;
        const uint32_t first_pf = prefix ? (uint32_t)(__ffs(prefix) - 1) : 32u;
        const bool done = first_pf < first_nr;
        const uint32_t take = done ? first_pf + 1 : first_nr;
        unsigned long long v = lane < take ? (st & value_mask) : 0ull;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        excl += v;
        if (done) break;
        if (take == 0) {
            if (++spins > limit) {
                if (lane == 0) atomicOr(err, SF_DEV_ERR_TIMEOUT);
                break;
            }
            __nanosleep(nap);
            nap = min(nap * 2u, 256u);
        }
        p -= take;
    }
    return excl;
}

// Single-pass exclusive scan with optional gather:
// out[i] = sum_{j<i} counts[gids ? gids[j] : j], 64-bit running sums, the
// u32 low word stored; *total_out = the 64-bit total.
constexpr int kScanItems = 16;
constexpr int kScanTile = kThreads * kScanItems;
constexpr unsigned long long kScanFlagAgg = 1ull << 62;
constexpr unsigned long long kScanFlagPrefix = 2ull << 62;
constexpr unsigned long long kScanValMask = (1ull << 62) - 1ull;

__global__ __launch_bounds__(kThreads) void scan_kernel(
    const uint32_t* __restrict__ gids, const uint32_t* counts, uint32_t* out, const uint32_t* n_dev,
    uint32_t n_static, unsigned long long* lookback, uint32_t* ticket,
    unsigned long long* total_out, uint32_t* err, LookbackKnobs knobs) {
    pdl_trigger();
    pdl_wait();
    __shared__ uint32_t s_part;
    __shared__ unsigned long long s_warp[kWarps];
    __shared__ unsigned long long s_prefix;
    __shared__ uint32_t s_tile[kThreads * (kScanItems + 1)];
    const uint32_t tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5;
    const uint32_t n = load_n(n_dev, n_static);
    const uint32_t num_parts = (n + kScanTile - 1) / kScanTile;
    if (tid == 0) s_part = atomicAdd(ticket, 1u);
    __syncthreads();
    const uint32_t part = s_part;
    if (n == 0) {
        if (part == 0 && tid == 0 && total_out) *total_out = 0ull;
        return;
    }
    if (part >= num_parts) return;
    // Coalesced striped loads, transposed through shared memory so each
    // thread scans kScanItems consecutive elements (row pitch 17 words keeps
    // the transposed reads conflict-free).
    const uint32_t tile0 = part * kScanTile;
#pragma unroll
    for (int i = 0; i < kScanItems; ++i) {
        const uint32_t e = i * kThreads + tid;
        const uint32_t idx = tile0 + e;
        uint32_t c = 0;
        if (idx < n) c = counts[gids ? gids[idx] : idx];
        s_tile[(e / kScanItems) * (kScanItems + 1) + e % kScanItems] = c;
    }
    __syncthreads();
    const uint32_t base = tile0 + tid * kScanItems;
    uint32_t v[kScanItems];
    unsigned long long local = 0;
#pragma unroll
    for (int i = 0; i < kScanItems; ++i) {
        v[i] = s_tile[tid * (kScanItems + 1) + i];
        local += v[i];
    }
    // Block exclusive scan of the per-thread sums.
    unsigned long long incl = local;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned long long t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= (uint32_t)o) incl += t;
    }
    if (lane == 31) s_warp[warp] = incl;
    __syncthreads();
    unsigned long long warp_prefix = 0, block_total = 0;
#pragma unroll
    for (int w = 0; w < kWarps; ++w) {
        if ((uint32_t)w < warp) warp_prefix += s_warp[w];
        block_total += s_warp[w];
    }
    if (warp == 0) {
        unsigned long long excl = 0;
        if (part == 0) {
            if (lane == 0 && !knobs.withhold) st_relaxed64(&lookback[0], kScanFlagPrefix | block_total);
        } else {
            if (lane == 0) st_relaxed64(&lookback[part], kScanFlagAgg | block_total);
            excl = lookback_warp64(lookback, part, err, knobs.spin_limit, kScanFlagPrefix, kScanValMask);
            if (lane == 0) st_relaxed64(&lookback[part], kScanFlagPrefix | (excl + block_total));
        }
        if (lane == 0) {
            s_prefix = excl;
            if (part == num_parts - 1 && total_out) *total_out = excl + block_total;
        }
    }
    __syncthreads();
    unsigned long long running = s_prefix + warp_prefix + (incl - local);
#pragma unroll
    for (int i = 0; i < kScanItems; ++i) {
        s_tile[tid * (kScanItems + 1) + i] = (uint32_t)running;
        running += v[i];
    }
    (void)base;
    __syncthreads();
#pragma unroll
    for (int i = 0; i < kScanItems; ++i) {
        const uint32_t e = i * kThreads + tid;
        const uint32_t idx = tile0 + e;
        if (idx < n) out[idx] = s_tile[(e / kScanItems) * (kScanItems + 1) + e % kScanItems];
    }
}

}  // namespace

uint32_t radix_passes(uint32_t bits, uint32_t digit_bits) { return (bits + digit_bits - 1) / digit_bits; }

size_t radix_temp_bytes(uint32_t max_elems, uint32_t max_passes) {
    const size_t parts = (max_elems + kMinPassTile - 1) / kMinPassTile;
    // hist [1024] + tickets [16] + lookback [passes][parts][256]: 32-bit keys
    // at 8-bit digits (4 passes x 256 bins) need the most, and every narrower
    // digit (passes x bins <= 1024) fits the same space.
    return kHistWords * 4 + 64 + (size_t)max_passes * parts * kRadix * 4;
}

namespace {

template <int BITS>
cudaError_t radix_sort_bits(const uint32_t* keys_in, const uint32_t* vals_in, uint32_t* keys_a, uint32_t* vals_a,
                            uint32_t* keys_b, uint32_t* vals_b, uint32_t n, const uint32_t* n_dev, uint32_t max_n,
                            uint32_t bits, bool write_keys, bool vals_iota, void* temp, uint32_t* err,
                            int sm_count, cudaStream_t stream, int* out_in_b, LookbackKnobs knobs) {
    constexpr uint32_t R = 1u << BITS;
    const uint32_t passes = radix_passes(bits, BITS);
    const uint32_t grid_n = n_dev ? max_n : n;
    uint8_t* t = static_cast<uint8_t*>(temp);
    uint32_t* hist = reinterpret_cast<uint32_t*>(t);
    uint32_t* tickets = reinterpret_cast<uint32_t*>(t + kHistWords * 4);
    uint32_t* lookback = reinterpret_cast<uint32_t*>(t + kHistWords * 4 + 64);
    const bool wide = grid_n >= kWidePassN;
    const uint32_t tile = (wide ? 512u : 256u) * kItems;
    const size_t parts = (grid_n + tile - 1) / tile;
    cudaError_t e = cudaMemsetAsync(temp, 0, kHistWords * 4 + 64 + passes * parts * R * 4, stream);
    if (e != cudaSuccess) return e;
    if (parts == 0) { *out_in_b = 0; return cudaSuccess; }
    const uint32_t hist_blocks = (uint32_t)std::min<size_t>((grid_n + kThreads * 8 - 1) / (kThreads * 8),
                                                             (size_t)sm_count * 4);
    radix_histogram_kernel<BITS><<<std::max(hist_blocks, 1u), kThreads, 0, stream>>>(
        keys_in, n_dev, n, passes, bits, hist);
    int in_b = 0;
    auto run_passes = [&](auto threads) -> cudaError_t {
        constexpr int TH = decltype(threads)::value;
        cudaError_t e2 = cudaFuncSetAttribute(onesweep_pass_kernel<BITS, TH>,
                                              cudaFuncAttributeMaxDynamicSharedMemorySize, (int)pass_smem<TH>());
        if (e2 != cudaSuccess) return e2;
        const uint32_t* kin = keys_in;
        const uint32_t* vin = vals_in;
        for (uint32_t p = 0; p < passes; ++p) {
            const uint32_t shift = p * BITS;
            const uint32_t w = std::min<uint32_t>(bits - shift, BITS);
            uint32_t* kout = (p % 2 == 0) ? keys_a : keys_b;
            uint32_t* vout = (p % 2 == 0) ? vals_a : vals_b;
            const bool wk = write_keys || (p + 1 < passes);
            onesweep_pass_kernel<BITS, TH><<<(uint32_t)parts, TH, pass_smem<TH>(), stream>>>(
                kin, vin, kout, vout, n_dev, n, shift, (1u << w) - 1u, hist + p * R,
                lookback + (size_t)p * parts * R, tickets + p, err, (vals_iota && p == 0) ? 1 : 0,
                wk ? 1 : 0, knobs);
            kin = kout;
            vin = vout;
            in_b = (p % 2 == 1);
        }
        return cudaSuccess;
    };
    e = wide ? run_passes(std::integral_constant<int, 512>{}) : run_passes(std::integral_constant<int, 256>{});
    if (e != cudaSuccess) return e;
    *out_in_b = in_b;
    note_launches(1 + passes);
    return cudaGetLastError();
}

}  // namespace

cudaError_t radix_sort_pairs(const uint32_t* keys_in, const uint32_t* vals_in, uint32_t* keys_a,
                             uint32_t* vals_a, uint32_t* keys_b, uint32_t* vals_b, uint32_t n,
                             const uint32_t* n_dev, uint32_t max_n, uint32_t bits, bool write_keys,
                             bool vals_iota, void* temp, uint32_t* err, int sm_count,
                             cudaStream_t stream, int* out_in_b, LookbackKnobs knobs, uint32_t digit_bits) {
    switch (digit_bits) {
#define SF_RADIX_CASE(B)                                                                                      \
    case B:                                                                                                   \
        return radix_sort_bits<B>(keys_in, vals_in, keys_a, vals_a, keys_b, vals_b, n, n_dev, max_n, bits,   \
                                  write_keys, vals_iota, temp, err, sm_count, stream, out_in_b, knobs);
        SF_RADIX_CASE(4)
        SF_RADIX_CASE(5)
        SF_RADIX_CASE(6)
        SF_RADIX_CASE(7)
        SF_RADIX_CASE(8)
#undef SF_RADIX_CASE
        default: return cudaErrorInvalidValue;
    }
}

size_t scan_temp_bytes(uint32_t max_elems) {
    const size_t parts = (max_elems + kScanTile - 1) / kScanTile;
    return 64 + std::max<size_t>(parts, 1) * 8;
}

cudaError_t exclusive_scan(const uint32_t* gids, const uint32_t* counts, uint32_t* out, uint32_t n,
                           const uint32_t* n_dev, uint32_t max_n, void* temp,
                           unsigned long long* total_out, uint32_t* err, cudaStream_t stream,
                           LookbackKnobs knobs) {
    const uint32_t grid_n = n_dev ? max_n : n;
    const size_t parts = std::max<size_t>((grid_n + kScanTile - 1) / kScanTile, 1);
    uint8_t* t = static_cast<uint8_t*>(temp);
    uint32_t* ticket = reinterpret_cast<uint32_t*>(t);
    unsigned long long* lookback = reinterpret_cast<unsigned long long*>(t + 64);
    cudaError_t e = cudaMemsetAsync(temp, 0, 64 + parts * 8, stream);
    if (e != cudaSuccess) return e;
    scan_kernel<<<(uint32_t)parts, kThreads, 0, stream>>>(gids, counts, out, n_dev, n, lookback,
                                                           ticket, total_out, err, knobs);
    note_launches(1);
    return cudaGetLastError();
}

}  // namespace sfk

namespace sfk {
LookbackKnobs lookback_test_knobs() { return g_test_knobs; }
}  // namespace sfk

extern "C" int sf_debug_lookback(uint32_t spin_limit, int withhold) {
    sfk::g_test_knobs = sfk::LookbackKnobs{spin_limit, withhold ? 1u : 0u};
    return SF_OK;
}

extern "C" int sf_debug_giant_lists(uint32_t lists) {
    sfk::set_giant_max_lists(lists);
    return SF_OK;
}
