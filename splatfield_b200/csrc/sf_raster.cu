// Tile rasterizer for sm_100a: rasterize_kernel (src/raster.rs:88-230) in its
// RGB, total-responsibility and evidence modes, plus a transmittance-only
// mode (3) that keeps each pixel's final T and last contributor for the
// adjoint of a per-splat scalar feature (sf_backward.cu).
//
// A CTA owns all (CTAS = 1) or part (CTAS = 2, 4) of one 16x16 tile: warp w of
// the tile covers the 8x4 pixel block at ((w & 1) * 8, (w >> 1) * 4), and a
// CTA of 256 / CTAS threads takes 8 / CTAS consecutive warps of it. Every
// CTA walks the tile's whole list in order for its own pixels, so splitting a
// tile changes no pixel's walk and no result; a long, unsaturated list is
// then walked by several SMs at once.
//
// Staging: the splat records of the list are gathered 256 entries at a time
// into shared memory with cp.async (16-byte global -> shared copies that
// need no registers), double-buffered: chunk c + 1 is in flight while chunk c
// is composited, and the ids of chunk c + 2 are loaded a chunk ahead, so the
// gather latency overlaps the walk instead of stalling every warp between two
// barriers. Two barriers per chunk: one before reusing a buffer, one (with the
// saturation count) before compositing it.
//
// Per pair: the power of the splat's quadratic form at the pixel; a pair with
// power above the splat's power_max (alpha < 1/255 for sure) skips the
// exponential; alpha = min(opacity * exp(-power), 0.999), pairs below 1/255
// are skipped, and the pixel stops after the contributor that takes T below
// 1/255 (src/raster.rs:173-221). The f32 operations are the oracle's, in the
// same order (sf_math.cuh), so images and words are bit-identical to it.
//
// CULL: each warp walks only the entries whose power_max box (with margin,
// from the projection) reaches its 8x4 block, 32 candidates per ballot; a
// pair outside the box has power above power_max, which the per-pixel test
// skips anyway, so nothing changes but the work.
//
// Responsibility / evidence words: the 32 pixels' fixed-point shares of an
// entry are summed by the warp (redux.sync) only when one of them is non-zero,
// added to a per-entry shared accumulator, and the chunk's accumulators go to
// global memory with one atomic per splat per CTA. Integer sums are
// order-independent, so the words equal the reference's per-pixel atomics.
//
// LAZY: the tile's list comes unsorted (the binned build's placed (depth key,
// splat id) pairs) and is put in order here, slab by slab, only as far as the
// pixels need: a 256-bin histogram over the 64-bit (key, id) values left
// picks a run of bins holding at most kSlab entries, that slab is gathered and
// bitonic-sorted in shared memory and composited, and the next slab starts
// after the last bin taken. (key, id) values are distinct and slabs end on bin
// boundaries, so the composite order is exactly the sorted list's.
#include <cstdint>
#include "sf_internal.h"
#include "sf_math.cuh"

namespace sfk {

namespace {

using namespace sfm;

constexpr uint32_t kChunk = 256;
constexpr uint32_t kSlab = 2048;
constexpr uint32_t kFirstSlab = 256;

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
    const uint32_t s = (uint32_t)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async8(void* smem, const void* gmem) {
    const uint32_t s = (uint32_t)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// CULL's second test, for an entry whose power_max box reaches the warp's
// 8x4 block: whether the splat's quadratic form q(dx, dy) = hx dx^2 +
// cy dx dy + hz dy^2 stays above power_max at every pixel of the block. The
// pixel offsets (splat centre minus pixel centre) lie in [X0 - 7, X0] x
// [Y0 - 3, Y0], widened by 1e-3 for the rounding of X0 and Y0. The form is
// convex, so its minimum over that rectangle is 0 with the centre inside it,
// else the least of its minima along the four edges (each a 1-D quadratic,
// minimised at a clamped point; an approximate minimiser only raises q by
// the square of its error). The entry is skipped only when that minimum
// exceeds power_max by 1e-5 of the largest sum of |terms| over the block
// plus 1e-5: both this minimum and the per-pixel power are a few roundings
// of such terms (error below 1e-6 of their sum), so every pixel's computed
// power is then above power_max and the pixel would skip the pair itself.
// A form that is not positive definite has no box (ext infinite) and is
// never skipped.
__device__ __forceinline__ bool block_misses(const float4 g0, const float4 g1, const float2 e, float wxf,
                                             float wyf) {
    if (!(e.x < INFINITY)) return false;
    const float hx = g0.z, cy = g0.w, hz = g1.x, pmax = g1.z;
    const float x0 = g0.x - wxf, y0 = g0.y - wyf;
    const float xlo = x0 - 7.001f, xhi = x0 + 0.001f, ylo = y0 - 3.001f, yhi = y0 + 0.001f;
    if (xlo <= 0.0f && xhi >= 0.0f && ylo <= 0.0f && yhi >= 0.0f) return false;
    const float ky = __fdividef(-0.5f * cy, hz), kx = __fdividef(-0.5f * cy, hx);
    auto q = [&](float x, float y) { return fmaf(hx * x, x, fmaf(hz * y, y, (cy * x) * y)); };
    const float y1 = fminf(fmaxf(ky * xlo, ylo), yhi), y2 = fminf(fmaxf(ky * xhi, ylo), yhi);
    const float x1 = fminf(fmaxf(kx * ylo, xlo), xhi), x2 = fminf(fmaxf(kx * yhi, xlo), xhi);
    const float qmin = fminf(fminf(q(xlo, y1), q(xhi, y2)), fminf(q(x1, ylo), q(x2, yhi)));
    const float dx = fmaxf(fabsf(xlo), fabsf(xhi)), dy = fmaxf(fabsf(ylo), fabsf(yhi));
    const float smax = fmaf(hx * dx, dx, fmaf(hz * dy, dy, (fabsf(cy) * dx) * dy));
    return qmin > fmaf(1e-5f, smax, pmax + 1e-5f);
}

// Modes: 0 RGB, 1 total responsibility words, 2 evidence (fg / bg) words,
// 3 transmittance only (final T and last contributor per pixel).
template <int MODE>
struct ModeOf {
    static constexpr bool kColor = MODE == 0;
    static constexpr bool kWords = MODE == 1 || MODE == 2;
};

// Shared staging of one CTA: two buffers of kChunk records each.
template <int MODE, bool CULL>
struct Stage {
    static constexpr bool kC = ModeOf<MODE>::kColor, kW = ModeOf<MODE>::kWords;
    float4 g0[2][kChunk];
    float4 g1[2][kChunk];
    float4 col[kC ? 2 : 1][kC ? kChunk : 1];
    float2 ext[CULL ? 2 : 1][CULL ? kChunk : 1];
    uint32_t gid[kW ? 2 : 1][kW ? kChunk : 1];
    uint32_t acc0[kW ? 2 : 1][kW ? kChunk : 1];
    uint32_t acc1[MODE == 2 ? 2 : 1][MODE == 2 ? kChunk : 1];
};

struct PixelState {
    float T, pr, pg, pb;
    uint32_t last;
    bool done;
    uint32_t n_eval, n_hit, n_proc;
};

// Composites list entries [0, count) in order for this CTA's pixels; id(i)
// gives entry i's splat id, list_off the entry's position in the tile's
// whole sorted list. (wxf, wyf): the first pixel centre of this warp's 8x4
// block. Returns true once every pixel of the CTA is saturated (uniform).
// STATE: ps.last tracks the last contributor (for the adjoint); otherwise
// only the entry that saturated the pixel.
template <int MODE, bool CULL, bool DETAIL, bool STATE, uint32_t NT, typename IdOf>
__device__ bool composite_list(const RasterArgs& a, Stage<MODE, CULL>& sm, IdOf id, uint32_t count,
                               uint32_t list_off, float fx, float fy, float wxf, float wyf, uint32_t inside,
                               PixelState& ps) {
    constexpr uint32_t kPer = kChunk / NT;
    constexpr bool kColor = ModeOf<MODE>::kColor, kWords = ModeOf<MODE>::kWords;
    const uint32_t tid = threadIdx.x, lane = tid & 31u;
    const float inv255 = 1.0f / 255.0f;
    const uint32_t nchunks = (count + kChunk - 1) / kChunk;
    if (nchunks == 0) return false;
    uint32_t g_next[kPer];
    auto load_ids = [&](uint32_t c) {
#pragma unroll
        for (uint32_t k = 0; k < kPer; ++k) {
            const uint32_t idx = c * kChunk + k * NT + tid;
            g_next[k] = idx < count ? id(idx) : 0u;
        }
    };
    auto issue = [&](uint32_t c, uint32_t b) {
#pragma unroll
        for (uint32_t k = 0; k < kPer; ++k) {
            const uint32_t e = k * NT + tid;
            if (c * kChunk + e < count) {
                const uint32_t g = g_next[k];
                cp_async16(&sm.g0[b][e], a.geo0 + g);
                cp_async16(&sm.g1[b][e], a.geo1 + g);
                if (kColor) cp_async16(&sm.col[b][e], a.color + g);
                if (CULL) cp_async8(&sm.ext[b][e], a.ext + g);
                if (kWords) sm.gid[b][e] = g;
            }
        }
    };
    // Sums of buffer b's first cnt entries to global memory; the
    // accumulators are left at zero for the buffer's next chunk.
    auto flush = [&](uint32_t b, uint32_t cnt) {
#pragma unroll
        for (uint32_t k = 0; k < kPer; ++k) {
            const uint32_t e = k * NT + tid;
            if (e < cnt) {
                const uint32_t g = sm.gid[b][e];
                const uint32_t v0 = sm.acc0[b][e];
                if (v0) {
                    atomicAdd((MODE == 1 ? a.resp : a.fg) + g, v0);
                    sm.acc0[b][e] = 0u;
                }
                if (MODE == 2) {
                    const uint32_t v1 = sm.acc1[b][e];
                    if (v1) {
                        atomicAdd(a.bg + g, v1);
                        sm.acc1[b][e] = 0u;
                    }
                }
            }
        }
    };
    // One (warp, entry) step: every lane of the warp runs it together.
    auto step = [&](uint32_t b, uint32_t j, uint32_t pos) {
        if (DETAIL) ++ps.n_proc;
        uint32_t q = 0;
        // CULL: a warp whose pixels are all done has left the chunk, so the
        // power is formed unconditionally and one branch tests both.
        if (CULL || !ps.done) {
            const float4 g0 = sm.g0[b][j];
            const float4 g1 = sm.g1[b][j];
            const float dx = g0.x - fx, dy = g0.y - fy;
            const float power = fma_(g0.z * dx, dx, fma_(g1.x * dy, dy, (g0.w * dx) * dy));
            if ((!CULL || !ps.done) && !(power > g1.z)) {
                if (DETAIL) ++ps.n_eval;
                const float alpha = fminf(g1.y * exp_neg_(-power), 0.999f);
                if (alpha >= inv255) {
                    if (DETAIL) ++ps.n_hit;
                    const float vis = alpha * ps.T;
                    if (kColor) {
                        const float4 c = sm.col[b][j];
                        ps.pr = fma_(c.x, vis, ps.pr);
                        ps.pg = fma_(c.y, vis, ps.pg);
                        ps.pb = fma_(c.z, vis, ps.pb);
                    } else if (kWords) {
                        q = sat_u32(vis * a.scale);
                    }
                    ps.T = ps.T * (1.0f - alpha);
                    if (STATE) ps.last = pos;
                    if (ps.T < inv255) {
                        ps.done = true;
                        if (!STATE) ps.last = pos;
                    }
                }
            }
        }
        if (kWords) {
            if (__any_sync(0xffffffffu, q != 0u)) {
                if (MODE == 1) {
                    const uint32_t s = __reduce_add_sync(0xffffffffu, q);
                    if (lane == 0) atomicAdd(&sm.acc0[b][j], s);
                } else {
                    const uint32_t qf = inside ? q : 0u;
                    const uint32_t sf = __reduce_add_sync(0xffffffffu, qf);
                    const uint32_t st = __reduce_add_sync(0xffffffffu, q);
                    if (lane == 0) {
                        if (sf) atomicAdd(&sm.acc0[b][j], sf);
                        if (st - sf) atomicAdd(&sm.acc1[b][j], st - sf);
                    }
                }
            }
        }
    };

    load_ids(0);
    issue(0, 0);
    cp_async_commit();
    if (nchunks > 1) load_ids(1);
    for (uint32_t c = 0; c < nchunks; ++c) {
        const uint32_t b = c & 1u;
        // The walk of chunk c - 1 is over: its buffer may be refilled and
        // its sums are complete.
        __syncthreads();
        if (kWords && c > 0) flush(b ^ 1u, kChunk);
        if (c + 1 < nchunks) {
            issue(c + 1, b ^ 1u);
            if (c + 2 < nchunks) load_ids(c + 2);
        }
        cp_async_commit();
        cp_async_wait<1>();  // this thread's copies of chunk c have landed
        if (__syncthreads_count(ps.done) == NT) {
            cp_async_wait<0>();
            return true;
        }
        const uint32_t cnt = min(kChunk, count - c * kChunk);
        const uint32_t pos0 = list_off + c * kChunk + 1;
        if (CULL) {
            for (uint32_t g32 = 0; g32 < cnt; g32 += 32) {
                if (__all_sync(0xffffffffu, ps.done)) break;
                const uint32_t j = g32 + lane;
                bool hit = false;
                if (j < cnt) {
                    const float4 g0 = sm.g0[b][j];
                    const float2 e = sm.ext[b][j];
                    const float lx = (g0.x - e.x) - wxf, hx = (g0.x + e.x) - wxf;
                    const float ly = (g0.y - e.y) - wyf, hy = (g0.y + e.y) - wyf;
                    hit = lx <= 7.0f && hx >= 0.0f && ly <= 3.0f && hy >= 0.0f;
                    if (hit) hit = !block_misses(g0, sm.g1[b][j], e, wxf, wyf);
                }
                uint32_t word = __ballot_sync(0xffffffffu, hit);
                while (word) {
                    const uint32_t jj = g32 + (uint32_t)(__ffs(word) - 1);
                    word &= word - 1u;
                    step(b, jj, pos0 + jj);
                }
            }
        } else {
            for (uint32_t j = 0; j < cnt; ++j) step(b, j, pos0 + j);
        }
    }
    __syncthreads();
    if (kWords) flush((nchunks - 1) & 1u, count - (nchunks - 1) * kChunk);
    return false;
}

__device__ __forceinline__ unsigned long long pair_value(uint2 p) {
    return ((unsigned long long)p.x << 32) | p.y;
}

// Block min / max of 64-bit values (uniform); s64 holds 2 * 8 words.
template <uint32_t NT>
__device__ void block_minmax64(unsigned long long lo, unsigned long long hi, unsigned long long* s64,
                               unsigned long long& mn, unsigned long long& mx) {
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
#pragma unroll
    for (uint32_t d = 16; d > 0; d >>= 1) {
        lo = min(lo, __shfl_xor_sync(0xffffffffu, lo, d));
        hi = max(hi, __shfl_xor_sync(0xffffffffu, hi, d));
    }
    __syncthreads();
    if (lane == 0) {
        s64[warp] = lo;
        s64[8 + warp] = hi;
    }
    __syncthreads();
    mn = s64[0];
    mx = s64[8];
    for (uint32_t w = 1; w < NT / 32; ++w) {
        mn = min(mn, s64[w]);
        mx = max(mx, s64[8 + w]);
    }
    __syncthreads();
}

// Bitonic sort of v[0, m) ascending in shared memory (m <= kSlab), padded to
// a power of two with the largest value.
template <uint32_t NT>
__device__ void bitonic_sort64(unsigned long long* v, uint32_t m) {
    uint32_t p = 1;
    while (p < m) p <<= 1;
    for (uint32_t i = m + threadIdx.x; i < p; i += NT) v[i] = ~0ull;
    __syncthreads();
    for (uint32_t k = 2; k <= p; k <<= 1) {
        for (uint32_t j = k >> 1; j > 0; j >>= 1) {
            for (uint32_t i = threadIdx.x; i < p; i += NT) {
                const uint32_t ixj = i ^ j;
                if (ixj > i) {
                    const unsigned long long x = v[i], y = v[ixj];
                    const bool up = (i & k) == 0;
                    if ((x > y) == up) {
                        v[i] = y;
                        v[ixj] = x;
                    }
                }
            }
            __syncthreads();
        }
    }
}

// This CTA's part `sub` of one tile (block-uniform).
template <int MODE, bool CULL, bool DETAIL, bool STATE, bool LAZY, uint32_t NT>
__device__ __forceinline__ void raster_tile(const RasterArgs& a, const uint32_t tile, const uint32_t sub) {
    __shared__ Stage<MODE, CULL> sm;
    __shared__ unsigned long long s_slab[LAZY ? kSlab : 1];
    __shared__ uint32_t s_hist[LAZY ? 256 : 1];
    __shared__ unsigned long long s_64[16];
    __shared__ uint32_t s_ctl[4];

    const uint32_t tx = tile % a.tiles_x, ty = tile / a.tiles_x;
    const uint32_t tid = threadIdx.x, lane = tid & 31u;
    const uint32_t wt = sub * (NT / 32) + (tid >> 5);  // warp of the tile
    const uint32_t wx0 = tx * 16 + (wt & 1u) * 8, wy0 = ty * 16 + (wt >> 1) * 4;
    const uint32_t px = wx0 + (lane & 7u);
    const uint32_t py = wy0 + (lane >> 3);
    const bool in_bounds = px < a.w && py < a.h;
    const float fx = (float)px + 0.5f, fy = (float)py + 0.5f;
    const float wxf = (float)wx0 + 0.5f, wyf = (float)wy0 + 0.5f;
    uint32_t inside = 0;
    if (MODE == 2 && in_bounds) inside = (a.mask[px / 32 + py * a.mask_wpr] >> (px % 32)) & 1u;
    const uint32_t start = a.tile_start[tile], end = a.tile_start[tile + 1];
    PixelState ps{1.0f, 0.0f, 0.0f, 0.0f, 0u, !in_bounds, 0u, 0u, 0u};
    if (ModeOf<MODE>::kWords) {
        for (uint32_t e = tid; e < kChunk; e += NT) {
            sm.acc0[0][e] = sm.acc0[1][e] = 0u;
            if (MODE == 2) sm.acc1[0][e] = sm.acc1[1][e] = 0u;
        }
    }

    if (!LAZY || end - start <= a.lazy_min) {
        const uint32_t* ids = a.gaussian_ids + start;
        composite_list<MODE, CULL, DETAIL, STATE, NT>(
            a, sm, [&](uint32_t i) { return __ldg(ids + i); }, end - start, 0, fx, fy, wxf, wyf, inside, ps);
    } else if (end > start) {
        const uint2* pairs = a.pairs + start;
        const uint32_t n = end - start;
        unsigned long long lo = ~0ull, hi = 0;
        for (uint32_t i = tid; i < n; i += NT) {
            const unsigned long long v = pair_value(pairs[i]);
            lo = min(lo, v);
            hi = max(hi, v);
        }
        unsigned long long vmin, vmax;
        block_minmax64<NT>(lo, hi, s_64, vmin, vmax);
        auto slab_id = [&](uint32_t i) { return (uint32_t)s_slab[i]; };
        if (n <= kFirstSlab) {
            for (uint32_t i = tid; i < n; i += NT) s_slab[i] = pair_value(pairs[i]);
            __syncthreads();
            bitonic_sort64<NT>(s_slab, n);
            composite_list<MODE, CULL, DETAIL, STATE, NT>(a, sm, slab_id, n, 0, fx, fy, wxf, wyf, inside, ps);
        } else {
            unsigned long long cur = vmin;
            uint32_t pos = 0;
            // The first slab aims at kFirstSlab entries (most tiles saturate
            // well inside it), later ones at the full kSlab.
            uint32_t target = kFirstSlab;
            for (;;) {
                // Pick [cur, sel] holding at most `target` of the values left
                // (one whole bin of up to kSlab when the first bin alone is
                // past the target).
                unsigned long long top = vmax, sel = vmax;
                for (;;) {
                    const unsigned long long width = top - cur;
                    const uint32_t wbits = width == 0 ? 0u : 64u - (uint32_t)__clzll(width);
                    const uint32_t shift = wbits > 8 ? wbits - 8 : 0u;
                    for (uint32_t i = tid; i < 256; i += NT) s_hist[i] = 0;
                    __syncthreads();
                    for (uint32_t i = tid; i < n; i += NT) {
                        const unsigned long long v = pair_value(pairs[i]);
                        if (v >= cur && v <= top) atomicAdd(&s_hist[(uint32_t)((v - cur) >> shift)], 1u);
                    }
                    __syncthreads();
                    if (tid < 32) {
                        // Warp 0: prefix over the 256 bins (8 per lane), the
                        // last bin whose running total stays within target.
                        const uint32_t nb = (uint32_t)(width >> shift) + 1u;
                        uint32_t c[8], run = 0;
#pragma unroll
                        for (uint32_t q = 0; q < 8; ++q) {
                            const uint32_t bn = lane * 8 + q;
                            c[q] = bn < nb ? s_hist[bn] : 0u;
                            run += c[q];
                        }
                        uint32_t incl = run;
#pragma unroll
                        for (uint32_t d = 1; d < 32; d <<= 1) {
                            const uint32_t x = __shfl_up_sync(0xffffffffu, incl, d);
                            if (lane >= d) incl += x;
                        }
                        uint32_t acc = incl - run, best = 0u;
                        bool any = false;
#pragma unroll
                        for (uint32_t q = 0; q < 8; ++q) {
                            acc += c[q];
                            const uint32_t bn = lane * 8 + q;
                            if (bn < nb && acc <= target) {
                                best = bn;
                                any = true;
                            }
                        }
                        const uint32_t e = __reduce_max_sync(0xffffffffu, any ? best + 1u : 0u);
                        if (lane == 0) {
                            const uint32_t h0 = s_hist[0];
                            // e == 0: even bin 0 is past the target.
                            s_ctl[0] = e > 0 ? 1u : (h0 <= kSlab ? 1u : 0u);
                            s_ctl[1] = e > 0 ? e - 1u : 0u;
                            s_ctl[2] = nb;
                        }
                    }
                    __syncthreads();
                    const uint32_t e = s_ctl[1], bins = s_ctl[2];
                    if (!s_ctl[0]) {
                        // The first bin holds more than kSlab: narrow to it.
                        top = cur + ((1ull << shift) - 1ull);
                        continue;
                    }
                    sel = (e + 1 >= bins) ? top : cur + (((unsigned long long)(e + 1)) << shift) - 1ull;
                    break;
                }
                if (tid == 0) s_ctl[3] = 0;
                __syncthreads();
                for (uint32_t i = tid; i < n; i += NT) {
                    const unsigned long long v = pair_value(pairs[i]);
                    if (v >= cur && v <= sel) s_slab[atomicAdd(&s_ctl[3], 1u)] = v;
                }
                __syncthreads();
                const uint32_t m = s_ctl[3];
                bitonic_sort64<NT>(s_slab, m);
                if (composite_list<MODE, CULL, DETAIL, STATE, NT>(a, sm, slab_id, m, pos, fx, fy, wxf, wyf,
                                                                  inside, ps))
                    break;
                pos += m;
                if (sel == vmax) break;
                cur = sel + 1;
                target = kSlab;
                __syncthreads();
            }
        }
    }
    if (a.stats) {
        if (DETAIL) {
            const uint32_t e = __reduce_add_sync(0xffffffffu, ps.n_eval);
            const uint32_t c = __reduce_add_sync(0xffffffffu, ps.n_hit);
            const uint32_t pr_ = __reduce_add_sync(0xffffffffu, ps.n_proc);
            if (lane == 0) {
                atomicAdd(a.stats + 1, (unsigned long long)e);
                atomicAdd(a.stats + 2, (unsigned long long)c);
                atomicAdd(a.stats + 3, (unsigned long long)pr_);
            }
        }
        // Algorithmic pairs: this CTA's pixels times the entries of the
        // sorted list that a walk in 256-entry chunks covers until every one
        // of them is saturated — the entry that saturates its last pixel,
        // rounded up to a chunk (the whole list if a pixel never saturates).
        // With one CTA per tile, 256 per entry the tile walks. The same
        // count for either list order.
        const uint32_t n_list = end - start;
        uint32_t e = ps.done ? ps.last : n_list;
        e = __reduce_max_sync(0xffffffffu, e);
        __syncthreads();
        if (tid == 0) s_ctl[0] = 0;
        __syncthreads();
        if (lane == 0) atomicMax(&s_ctl[0], e);
        __syncthreads();
        if (tid == 0) {
            const uint32_t emax = s_ctl[0];
            const uint64_t chunks = ((uint64_t)emax + kChunk - 1) / kChunk * kChunk;
            const uint64_t walked = chunks < n_list ? chunks : (uint64_t)n_list;
            atomicAdd(a.stats, (unsigned long long)NT * walked);
        }
    }
    if (!in_bounds) return;
    const size_t pix = (size_t)py * a.w + px;
    if (MODE == 0) {
        if (a.bitmap) {
            const uint32_t r = sat_u32(clamp_(ps.pr * 255.0f, 0.0f, 255.0f));
            const uint32_t g = sat_u32(clamp_(ps.pg * 255.0f, 0.0f, 255.0f));
            const uint32_t b = sat_u32(clamp_(ps.pb * 255.0f, 0.0f, 255.0f));
            const uint32_t al = sat_u32(clamp_((1.0f - ps.T) * 255.0f, 0.0f, 255.0f));
            a.bitmap[(size_t)py * a.row_stride + px] = r | (g << 8) | (b << 16) | (al << 24);
        }
        if (a.rgba) a.rgba[pix] = make_float4(ps.pr, ps.pg, ps.pb, 1.0f - ps.T);
    }
    if (STATE) {
        if (a.final_t) a.final_t[pix] = ps.T;
        if (a.n_contrib) a.n_contrib[pix] = ps.last;
    }
}

// 256 / NT CTAs per tile: block i takes part i % (256 / NT) of tile i /
// (256 / NT), or with class lists of the tile of that rank in longest-list-
// first order.
template <int MODE, bool CULL, bool DETAIL, bool STATE, bool LAZY, uint32_t NT>
__global__ __launch_bounds__(NT) void raster_kernel(RasterArgs a) {
    constexpr uint32_t kSplit = 256 / NT;
    const uint32_t rank = blockIdx.x / kSplit, sub = blockIdx.x % kSplit;
    uint32_t tile = rank;
    if (a.class_lists) {
        const uint32_t tiles = a.tiles_x * a.tiles_y;
        uint32_t j = rank;
        int k = kSortClasses - 1;
        for (; k >= 0; --k) {
            const uint32_t c = a.class_n[k];
            if (j < c) break;
            j -= c;
        }
        // k < 0: the empty tiles (the counts sum to the tile count).
        tile = a.class_lists[(size_t)(k < 0 ? kSortClasses : k) * tiles + j];
    }
    raster_tile<MODE, CULL, DETAIL, STATE, LAZY, NT>(a, tile, sub);
}

template <int MODE, bool CULL, bool LAZY>
void raster_go(const RasterArgs& a, uint32_t tiles, cudaStream_t st) {
    if constexpr (MODE == 3) {
        // The per-pixel state is the mode's only output: one CTA per tile.
        if (a.detail) raster_kernel<3, CULL, true, true, LAZY, 256><<<tiles, 256, 0, st>>>(a);
        else raster_kernel<3, CULL, false, true, LAZY, 256><<<tiles, 256, 0, st>>>(a);
    } else {
        const bool state = MODE == 0 && (a.final_t || a.n_contrib);
        constexpr bool kState = MODE == 0;
        // The diagnostic and adjoint-state forms run one CTA per tile.
        const uint32_t split = (a.detail || state) ? 1u : a.split;
        if (split == 4) {
            raster_kernel<MODE, CULL, false, false, LAZY, 64><<<tiles * 4, 64, 0, st>>>(a);
        } else if (split == 2) {
            raster_kernel<MODE, CULL, false, false, LAZY, 128><<<tiles * 2, 128, 0, st>>>(a);
        } else if (a.detail) {
            if (state) raster_kernel<MODE, CULL, true, kState, LAZY, 256><<<tiles, 256, 0, st>>>(a);
            else raster_kernel<MODE, CULL, true, false, LAZY, 256><<<tiles, 256, 0, st>>>(a);
        } else {
            if (state) raster_kernel<MODE, CULL, false, kState, LAZY, 256><<<tiles, 256, 0, st>>>(a);
            else raster_kernel<MODE, CULL, false, false, LAZY, 256><<<tiles, 256, 0, st>>>(a);
        }
    }
}

template <int MODE>
void raster_dispatch(const RasterArgs& a, uint32_t tiles, cudaStream_t st) {
    if (a.pairs) {
        if (a.cull) raster_go<MODE, true, true>(a, tiles, st);
        else raster_go<MODE, false, true>(a, tiles, st);
    } else {
        if (a.cull) raster_go<MODE, true, false>(a, tiles, st);
        else raster_go<MODE, false, false>(a, tiles, st);
    }
}

}  // namespace

cudaError_t launch_raster(int mode, const RasterArgs& args, cudaStream_t stream) {
    const uint32_t tiles = args.tiles_x * args.tiles_y;
    if (tiles == 0) return cudaSuccess;
    RasterArgs a = args;
    if (a.split == 0) a.split = 1;
    if (a.split != 1 && a.split != 2 && a.split != 4) return cudaErrorInvalidValue;
    switch (mode) {
        case 0: raster_dispatch<0>(a, tiles, stream); break;
        case 1: raster_dispatch<1>(a, tiles, stream); break;
        case 2: raster_dispatch<2>(a, tiles, stream); break;
        case 3:
            if (!a.final_t || !a.n_contrib) return cudaErrorInvalidValue;
            raster_dispatch<3>(a, tiles, stream);
            break;
        default: return cudaErrorInvalidValue;
    }
    note_launches(1);
    return cudaGetLastError();
}

}  // namespace sfk
