// Segmentation-evidence kernels: analytic EIG over Beta posteriors (f32 LUT
// and on-GPU FP64 entropy) and the conjugate Beta update.
//
// Reference: src/seg/beta.rs:55-212. The reference sums per-workgroup f32
// partials on the host after a blocking read-back (beta.rs:265-267); here the
// sum is an f64 two-level reduction on the device in a fixed order, so the
// result is deterministic and a batched round needs no host sync per view.
#include <cmath>
#include <math_constants.h>
#include <cstdint>
#include "sf_internal.h"
#include "sf_math.cuh"

namespace sfk {

// ---- host: the f64 entropy formulas and the LUT (beta.rs:55-112)
namespace {
double lgamma_h(double x) {
    const double z = x - 1.0;
    static const double c[8] = {676.5203681218851,    -1259.1392167224028, 771.3234287776531,
                                -176.6150291621406,   12.507343278686905,  -0.13857109526572012,
                                9.984369578019572e-6, 1.5056327351493116e-7};
    double series = 0.9999999999998099;
    for (int k = 0; k < 8; ++k) series += c[k] / (z + (double)k + 1.0);
    const double t = z + 7.5;
    return 0.5 * std::log(2.0 * 3.141592653589793) + (z + 0.5) * std::log(t) - t + std::log(series);
}
// The recurrence runs at most six steps for x > 0. Beta parameters are
// positive, so x <= 0 and NaN return NaN instead of recurring (the
// reference's loop, beta.rs:77-86, would take about |x| steps there and never
// end for x <= -2^53).
double digamma_h(double x) {
    if (!(x > 0.0)) return NAN;
    double r = 0.0;
    while (x < 6.0) { r -= 1.0 / x; x += 1.0; }
    const double inv = 1.0 / x, inv2 = inv * inv;
    return r + std::log(x) - 0.5 * inv - inv2 / 12.0 + inv2 * inv2 / 120.0 -
           inv2 * inv2 * inv2 / 252.0;
}
}  // namespace

double beta_entropy_host(double a, double b) {
    const double s = a + b;
    return lgamma_h(a) + lgamma_h(b) - lgamma_h(s) - (a - 1.0) * digamma_h(a) -
           (b - 1.0) * digamma_h(b) + (s - 2.0) * digamma_h(s);
}

void build_entropy_table(float* table) {
    double axis[kGridPts];
    for (int i = 0; i < kGridPts; ++i) axis[i] = std::exp((double)((float)i * kLnStep));
    for (int i = 0; i < kGridPts; ++i)
        for (int j = 0; j < kGridPts; ++j)
            table[i * kGridPts + j] = (float)beta_entropy_host(axis[i], axis[j]);
}

namespace {

using namespace sfm;

// ---- device f64 entropy: the same formulas as the host (beta.rs:55-86),
// CUDA double log. The per-term forms below are the plain statement;
// beta_entropy_d, which the EIG kernels use, arranges the lgamma part for
// the FP64 pipe without moving any evaluation point, so it agrees with the
// per-term form to rounding:
//   - each Lanczos series c0 + sum_k c_k / (z + k) is summed as one
//     fraction N / D (one division instead of eight);
//   - the three series logs of H(a, b) are one log of their ratio, and the
//     0.5 ln(2 pi) terms of the three lgammas leave one constant.
// psi keeps its recurrence (no division for x >= 6, most arguments).
// Arguments past 2^32 take the per-term forms (the fractions' products of
// eight factors stay below 2^260 under that bound). Measured on the
// 20-view FP64 round: 3.68 -> 3.48 ms, with the EIG kernels held to five
// blocks per SM (the fractions raise register use; at two blocks per SM
// the round took 3.71 ms, at three 3.54, at four 3.52).
__device__ __forceinline__ double lgamma_terms(double x) {
    const double z = x - 1.0;
    double series = 0.9999999999998099;
    series += 676.5203681218851 / (z + 1.0);
    series += -1259.1392167224028 / (z + 2.0);
    series += 771.3234287776531 / (z + 3.0);
    series += -176.6150291621406 / (z + 4.0);
    series += 12.507343278686905 / (z + 5.0);
    series += -0.13857109526572012 / (z + 6.0);
    series += 9.984369578019572e-6 / (z + 7.0);
    series += 1.5056327351493116e-7 / (z + 8.0);
    const double t = z + 7.5;
    return 0.5 * log(2.0 * 3.141592653589793) + (z + 0.5) * log(t) - t + log(series);
}
// As digamma_h: x <= 0 and NaN give NaN, so the recurrence is at most six
// steps for every input (a posterior word of -inf cannot hold the kernel).
__device__ __forceinline__ double digamma_terms(double x) {
    if (!(x > 0.0)) return CUDART_NAN;
    double r = 0.0;
    while (x < 6.0) { r -= 1.0 / x; x += 1.0; }
    const double inv = 1.0 / x, inv2 = inv * inv;
    return r + log(x) - 0.5 * inv - inv2 / 12.0 + inv2 * inv2 / 120.0 - inv2 * inv2 * inv2 / 252.0;
}
__device__ __forceinline__ double beta_entropy_terms(double a, double b) {
    const double s = a + b;
    return lgamma_terms(a) + lgamma_terms(b) - lgamma_terms(s) - (a - 1.0) * digamma_terms(a) -
           (b - 1.0) * digamma_terms(b) + (s - 2.0) * digamma_terms(s);
}

// The Lanczos series of lgamma(x), z = x - 1, as num / den.
__device__ __forceinline__ void lanczos_fraction(double x, double& num, double& den) {
    const double z = x - 1.0;
    double n = 0.9999999999998099, d = 1.0, zk;
    zk = z + 1.0; n = fma(n, zk, 676.5203681218851 * d); d *= zk;
    zk = z + 2.0; n = fma(n, zk, -1259.1392167224028 * d); d *= zk;
    zk = z + 3.0; n = fma(n, zk, 771.3234287776531 * d); d *= zk;
    zk = z + 4.0; n = fma(n, zk, -176.6150291621406 * d); d *= zk;
    zk = z + 5.0; n = fma(n, zk, 12.507343278686905 * d); d *= zk;
    zk = z + 6.0; n = fma(n, zk, -0.13857109526572012 * d); d *= zk;
    zk = z + 7.0; n = fma(n, zk, 9.984369578019572e-6 * d); d *= zk;
    zk = z + 8.0; n = fma(n, zk, 1.5056327351493116e-7 * d); d *= zk;
    num = n;
    den = d;
}
__device__ __forceinline__ double beta_entropy_d(double a, double b) {
    const double s = a + b;
    if (!(a > 0.0) || !(b > 0.0) || !(s < 4294967296.0)) return beta_entropy_terms(a, b);
    double na, da, nb, db, ns, ds;
    lanczos_fraction(a, na, da);
    lanczos_fraction(b, nb, db);
    lanczos_fraction(s, ns, ds);
    // lgamma(x) = 0.5 ln(2 pi) + (x - 0.5) ln(x + 6.5) - (x + 6.5) + ln(series);
    // the three -(x + 6.5) add up to -6.5 exactly.
    const double lg = 0.91893853320467274178 + (a - 0.5) * log(a + 6.5) + (b - 0.5) * log(b + 6.5) -
                      (s - 0.5) * log(s + 6.5) - 6.5 + log(((na / da) * (nb / db)) * (ds / ns));
    return lg - (a - 1.0) * digamma_terms(a) - (b - 1.0) * digamma_terms(b) + (s - 2.0) * digamma_terms(s);
}

// table_entropy (beta.rs:128-144).
__device__ __forceinline__ float table_entropy_d(float a, float b, const float* __restrict__ t) {
    const float xa = log_(a) / kLnStep;
    const float xb = log_(b) / kLnStep;
    const float ia = min_(max_(floorf(xa), 0.0f), (float)(kGridPts - 2));
    const float ib = min_(max_(floorf(xb), 0.0f), (float)(kGridPts - 2));
    const float ta = clamp_(xa - ia, 0.0f, 1.0f);
    const float tb = clamp_(xb - ib, 0.0f, 1.0f);
    const uint32_t row = sat_u32(ia) * kGridPts + sat_u32(ib);
    const float h00 = __ldg(t + row), h10 = __ldg(t + row + kGridPts);
    const float h01 = __ldg(t + row + 1), h11 = __ldg(t + row + kGridPts + 1);
    return (((h00 * (1.0f - ta)) * (1.0f - tb) + (h10 * ta) * (1.0f - tb)) + (h01 * (1.0f - ta)) * tb) +
           (h11 * ta) * tb;
}

constexpr int kEigThreads = 256;

__device__ __forceinline__ double block_sum(double v, double* s_warp) {
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (lane == 0) s_warp[warp] = v;
    __syncthreads();
    double total = 0.0;
    if (threadIdx.x == 0)
        for (int w = 0; w < kEigThreads / 32; ++w) total += s_warp[w];
    return total;
}

// entropy_delta_kernel (beta.rs:152-201): per splat with eps > 0,
// dH = max(0, H(a,b) - H(k a, k b)), k = 1 + eps/(a+b).
template <int MODE>
__global__ __launch_bounds__(kEigThreads, 5) void eig_kernel(const float* __restrict__ a,
                                                          const float* __restrict__ b,
                                                          const uint32_t* __restrict__ resp,
                                                          const uint32_t* __restrict__ resp2,
                                                          uint32_t n, float scale,
                                                          const float* __restrict__ table,
                                                          double* __restrict__ partials,
                                                          const void* __restrict__ h0) {
    __shared__ double s_warp[kEigThreads / 32];
    double acc = 0.0;
    const uint32_t stride = gridDim.x * kEigThreads;
    for (uint32_t i = blockIdx.x * kEigThreads + threadIdx.x; i < n; i += stride) {
        // eps words; with an evidence split, eps = fg + bg exactly.
        const uint32_t bits = resp[i] + (resp2 ? resp2[i] : 0u);
        if (bits == 0u) continue;
        const float ai = a[i], bi = b[i];
        if (MODE == SF_EIG_LUT_F32) {
            const float eps = (float)bits / scale;
            const float k = 1.0f + eps / (ai + bi);
            const float hab = h0 ? static_cast<const float*>(h0)[i] : table_entropy_d(ai, bi, table);
            const float d = max_(hab - table_entropy_d(ai * k, bi * k, table), 0.0f);
            acc += (double)d;
        } else {
            const double eps = (double)bits / (double)scale;
            const double ad = ai, bd = bi;
            const double k = 1.0 + eps / (ad + bd);
            const double hab = h0 ? static_cast<const double*>(h0)[i] : beta_entropy_d(ad, bd);
            const double d = hab - beta_entropy_d(ad * k, bd * k);
            acc += d > 0.0 ? d : 0.0;
        }
    }
    const double total = block_sum(acc, s_warp);
    if (threadIdx.x == 0) partials[blockIdx.x] = total;
}

// entropy_delta_kernel over real-valued responsibilities (the adjoint of a
// per-splat scalar feature, sf_backward.cu): eps = fg + bg directly, with no
// fixed-point scale; the LUT form adds in f32, the FP64 form in f64.
template <int MODE>
__global__ __launch_bounds__(kEigThreads, 5) void eig_real_kernel(const float* __restrict__ a,
                                                               const float* __restrict__ b,
                                                               const float* __restrict__ fg,
                                                               const float* __restrict__ bg, uint32_t n,
                                                               const float* __restrict__ table,
                                                               double* __restrict__ partials,
                                                               const void* __restrict__ h0) {
    __shared__ double s_warp[kEigThreads / 32];
    double acc = 0.0;
    const uint32_t stride = gridDim.x * kEigThreads;
    for (uint32_t i = blockIdx.x * kEigThreads + threadIdx.x; i < n; i += stride) {
        const float f = fg[i], g = bg ? bg[i] : 0.0f;
        if (!(f + g > 0.0f)) continue;
        const float ai = a[i], bi = b[i];
        if (MODE == SF_EIG_LUT_F32) {
            const float k = 1.0f + (f + g) / (ai + bi);
            const float hab = h0 ? static_cast<const float*>(h0)[i] : table_entropy_d(ai, bi, table);
            const float d = max_(hab - table_entropy_d(ai * k, bi * k, table), 0.0f);
            acc += (double)d;
        } else {
            const double eps = (double)f + (double)g;
            const double ad = ai, bd = bi;
            const double k = 1.0 + eps / (ad + bd);
            const double hab = h0 ? static_cast<const double*>(h0)[i] : beta_entropy_d(ad, bd);
            const double d = hab - beta_entropy_d(ad * k, bd * k);
            acc += d > 0.0 ? d : 0.0;
        }
    }
    const double total = block_sum(acc, s_warp);
    if (threadIdx.x == 0) partials[blockIdx.x] = total;
}

// H(a_i, b_i) of every splat, once per batched round: every view's EIG term
// is H(a, b) - H(k a, k b) over the same posterior, so the views read the
// first half instead of each recomputing it (the same value, bit for bit, as
// the per-view kernel computes). LUT: f32 values; FP64: f64 values.
template <int MODE>
__global__ void entropy_kernel(const float* __restrict__ a, const float* __restrict__ b, uint32_t n,
                               const float* __restrict__ table, void* __restrict__ out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (MODE == SF_EIG_LUT_F32) static_cast<float*>(out)[i] = table_entropy_d(a[i], b[i], table);
    else static_cast<double*>(out)[i] = beta_entropy_d((double)a[i], (double)b[i]);
}

__global__ __launch_bounds__(kEigThreads) void eig_final_kernel(const double* __restrict__ partials,
                                                                uint32_t nb, double* out) {
    __shared__ double s_warp[kEigThreads / 32];
    double acc = 0.0;
    for (uint32_t i = threadIdx.x; i < nb; i += kEigThreads) acc += partials[i];
    const double total = block_sum(acc, s_warp);
    if (threadIdx.x == 0) *out = total;
}

// localize (src/seg/views.rs:24-66) over the foreground set {a > b} with
// weights m = a / (a + b): pass 0 sums (m, m x, m y, m z), pass 1 sums
// m |p - c| for the centre c of pass 0. Per-splat products in f32 as the
// reference computes them; sums in f64 over a fixed partition (deterministic).
__global__ __launch_bounds__(kEigThreads) void localize_kernel(const float* __restrict__ attr,
                                                               const float* __restrict__ a,
                                                               const float* __restrict__ b, uint32_t n,
                                                               int pass, const double* __restrict__ out,
                                                               double* __restrict__ partials) {
    __shared__ double s_warp[kEigThreads / 32];
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    float cx = 0.0f, cy = 0.0f, cz = 0.0f;
    if (pass == 1) {
        cx = (float)out[4];
        cy = (float)out[5];
        cz = (float)out[6];
    }
    const uint32_t stride = gridDim.x * kEigThreads;
    for (uint32_t i = blockIdx.x * kEigThreads + threadIdx.x; i < n; i += stride) {
        const float ai = a[i], bi = b[i];
        if (!(ai > bi)) continue;
        const float m = ai / (ai + bi);
        const float px = attr[i], py = attr[(size_t)n + i], pz = attr[2 * (size_t)n + i];
        if (pass == 0) {
            acc[0] += (double)m;
            acc[1] += (double)(m * px);
            acc[2] += (double)(m * py);
            acc[3] += (double)(m * pz);
        } else {
            const float dx = px - cx, dy = py - cy, dz = pz - cz;
            const float d = sqrtf((dx * dx + dy * dy) + dz * dz);
            acc[0] += (double)(m * d);
        }
    }
    const int sums = pass == 0 ? 4 : 1;
    for (int j = 0; j < sums; ++j) {
        const double total = block_sum(acc[j], s_warp);
        if (threadIdx.x == 0) partials[blockIdx.x * 4 + j] = total;
        __syncthreads();
    }
}

// out: [0..3] pass-0 sums, [4..6] centre (f32 values), [7] radius.
__global__ __launch_bounds__(kEigThreads) void localize_final_kernel(const double* __restrict__ partials,
                                                                     uint32_t nb, int pass, double* out) {
    __shared__ double s_warp[kEigThreads / 32];
    const int sums = pass == 0 ? 4 : 1;
    for (int j = 0; j < sums; ++j) {
        double acc = 0.0;
        for (uint32_t i = threadIdx.x; i < nb; i += kEigThreads) acc += partials[i * 4 + j];
        const double total = block_sum(acc, s_warp);
        if (threadIdx.x == 0) {
            if (pass == 0) out[j] = total;
            else out[7] = (double)(float)(total / out[0]);
        }
        __syncthreads();
    }
    if (pass == 0 && threadIdx.x == 0) {
        const double sw = out[0];
        for (int k = 0; k < 3; ++k) out[4 + k] = sw > 0.0 ? (double)(float)(out[1 + k] / sw) : 0.0;
    }
}

// paint_posterior (src/seg/paint.rs:104-114): each splat's projected colour
// becomes its posterior mean m = a / (a + b) as grey, with no +0.5 offset.
__global__ void paint_posterior_kernel(const float* __restrict__ a, const float* __restrict__ b, uint32_t n,
                                       float4* __restrict__ color) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float m = a[i] / (a[i] + b[i]);
    color[i] = make_float4(m, m, m, 0.0f);
}

// tint_colors (src/seg/paint.rs:116-126): DC planes of foreground splats
// (a > b) set to (r, g, b).
__global__ void tint_kernel(float* __restrict__ sh, const float* __restrict__ a, const float* __restrict__ b,
                            uint32_t n, float r, float g, float bl) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || !(a[i] > b[i])) return;
    sh[i] = r;
    sh[(size_t)n + i] = g;
    sh[2 * (size_t)n + i] = bl;
}

__global__ void beta_update_kernel(float scale, const uint32_t* __restrict__ fg,
                                   const uint32_t* __restrict__ bg, float* __restrict__ a,
                                   float* __restrict__ b, uint32_t n) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    a[i] = a[i] + (float)fg[i] / scale;
    b[i] = b[i] + (float)bg[i] / scale;
}

// Conjugate update from real-valued responsibilities: a += fg, b += bg.
__global__ void beta_update_real_kernel(const float* __restrict__ fg, const float* __restrict__ bg,
                                        float* __restrict__ a, float* __restrict__ b, uint32_t n) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    a[i] = a[i] + fg[i];
    b[i] = b[i] + bg[i];
}

__global__ void table_probe_kernel(const float* a, const float* b, uint32_t n, const float* table,
                                   float* out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = table_entropy_d(a[i], b[i], table);
}

}  // namespace

cudaError_t launch_paint_posterior(const float* a, const float* b, uint32_t n, float4* color,
                                   cudaStream_t stream) {
    if (n == 0) return cudaSuccess;
    paint_posterior_kernel<<<(n + 255) / 256, 256, 0, stream>>>(a, b, n, color);
    note_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_tint(float* sh, const float* a, const float* b, uint32_t n, float r, float g, float bl,
                        cudaStream_t stream) {
    if (n == 0) return cudaSuccess;
    tint_kernel<<<(n + 255) / 256, 256, 0, stream>>>(sh, a, b, n, r, g, bl);
    note_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_localize(const float* attr, const float* a, const float* b, uint32_t n, double* partials,
                            uint32_t blocks, double* out, cudaStream_t stream) {
    for (int pass = 0; pass < 2; ++pass) {
        localize_kernel<<<blocks, kEigThreads, 0, stream>>>(attr, a, b, n, pass, out, partials);
        localize_final_kernel<<<1, kEigThreads, 0, stream>>>(partials, blocks, pass, out);
    }
    note_launches(4);
    return cudaGetLastError();
}

uint32_t eig_blocks(uint32_t n, int sm_count) {
    const uint32_t want = (n + kEigThreads * 4 - 1) / (kEigThreads * 4);
    return std::max(1u, std::min(want, (uint32_t)sm_count * 8));
}

cudaError_t launch_eig(int mode, const float* a, const float* b, const uint32_t* resp, uint32_t n,
                       float scale, const float* table, double* partials, uint32_t blocks,
                       double* out, cudaStream_t stream, const uint32_t* resp2, const void* h0) {
    if (mode == SF_EIG_LUT_F32)
        eig_kernel<SF_EIG_LUT_F32><<<blocks, kEigThreads, 0, stream>>>(a, b, resp, resp2, n, scale, table, partials,
                                                                      h0);
    else
        eig_kernel<SF_EIG_FP64><<<blocks, kEigThreads, 0, stream>>>(a, b, resp, resp2, n, scale, table, partials, h0);
    eig_final_kernel<<<1, kEigThreads, 0, stream>>>(partials, blocks, out);
    note_launches(2);
    return cudaGetLastError();
}

cudaError_t launch_entropy(int mode, const float* a, const float* b, uint32_t n, const float* table, void* out,
                           cudaStream_t stream) {
    if (n == 0) return cudaSuccess;
    if (mode == SF_EIG_LUT_F32) entropy_kernel<SF_EIG_LUT_F32><<<(n + 255) / 256, 256, 0, stream>>>(a, b, n, table, out);
    else entropy_kernel<SF_EIG_FP64><<<(n + 255) / 256, 256, 0, stream>>>(a, b, n, table, out);
    note_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_eig_real(int mode, const float* a, const float* b, const float* fg, const float* bg,
                            uint32_t n, const float* table, double* partials, uint32_t blocks, double* out,
                            cudaStream_t stream, const void* h0) {
    if (mode == SF_EIG_LUT_F32)
        eig_real_kernel<SF_EIG_LUT_F32><<<blocks, kEigThreads, 0, stream>>>(a, b, fg, bg, n, table, partials, h0);
    else
        eig_real_kernel<SF_EIG_FP64><<<blocks, kEigThreads, 0, stream>>>(a, b, fg, bg, n, table, partials, h0);
    eig_final_kernel<<<1, kEigThreads, 0, stream>>>(partials, blocks, out);
    note_launches(2);
    return cudaGetLastError();
}

cudaError_t launch_beta_update_real(const float* fg, const float* bg, float* a, float* b, uint32_t n,
                                    cudaStream_t stream) {
    if (n == 0) return cudaSuccess;
    beta_update_real_kernel<<<(n + 255) / 256, 256, 0, stream>>>(fg, bg, a, b, n);
    note_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_beta_update(float scale, const uint32_t* fg, const uint32_t* bg, float* a,
                               float* b, uint32_t n, cudaStream_t stream) {
    if (n == 0) return cudaSuccess;
    beta_update_kernel<<<(n + 255) / 256, 256, 0, stream>>>(scale, fg, bg, a, b, n);
    note_launches(1);
    return cudaGetLastError();
}

cudaError_t launch_table_probe(const float* a, const float* b, uint32_t n, const float* table,
                               float* out, cudaStream_t stream) {
    if (n == 0) return cudaSuccess;
    table_probe_kernel<<<(n + 255) / 256, 256, 0, stream>>>(a, b, n, table, out);
    note_launches(1);
    return cudaGetLastError();
}

}  // namespace sfk
