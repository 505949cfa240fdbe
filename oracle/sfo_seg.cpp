// Oracle segmentation-evidence math (TEST INFRASTRUCTURE ONLY).
// Restates src/seg/mod.rs:31-34, 118-143 and src/seg/beta.rs:55-212.
#include <cmath>
#include <cstring>
#include <omp.h>
#include "sfo.h"
#include "sfo_math.h"

using namespace sfo;

namespace {
constexpr int kGridPts = 445;              // beta.rs:47
constexpr float kLnStep = 0.015611423f;    // beta.rs:50
}  // namespace

// fractional_bits (seg/mod.rs:31-34): 32 - log2(next_pow2(pixels)), saturating.
extern "C" uint32_t sfo_fractional_bits(uint32_t w, uint32_t h) {
    const uint64_t pixels = (uint64_t)w * (uint64_t)h;
    uint64_t p2 = 1;
    uint32_t tz = 0;
    while (p2 < pixels) { p2 <<= 1; ++tz; }
    return tz >= 32 ? 0u : 32u - tz;
}

// acc.scale = (1 << bits) as f32 (seg/mod.rs:178).
extern "C" float sfo_scale_for(uint32_t w, uint32_t h) {
    return (float)((uint64_t)1 << sfo_fractional_bits(w, h));
}

// Mask::from_bytes (seg/mod.rs:118-143): LSB-first words, ceil(w/32) per row.
extern "C" uint32_t sfo_mask_pack(const uint8_t* bytes, uint32_t w, uint32_t h, uint32_t* bits) {
    const uint32_t wpr = (w + 31) / 32;
    std::memset(bits, 0, (size_t)wpr * h * 4);
    uint32_t fg = 0;
    for (uint32_t p = 0; p < w * h; ++p)
        if (bytes[p]) {
            const uint32_t y = p / w, x = p % w;
            bits[y * wpr + x / 32] |= 1u << (x % 32);
            ++fg;
        }
    return fg;
}

// lgamma, Lanczos g = 7, 9 terms (beta.rs:55-73).
extern "C" double sfo_lgamma(double x) {
    const double z = x - 1.0;
    static const double c[8] = {676.5203681218851,     -1259.1392167224028,
                                771.3234287776531,     -176.6150291621406,
                                12.507343278686905,    -0.13857109526572012,
                                9.984369578019572e-6,  1.5056327351493116e-7};
    double series = 0.9999999999998099;
    for (int k = 0; k < 8; ++k) series += c[k] / (z + (double)k + 1.0);
    const double t = z + 7.5;
    return 0.5 * std::log(2.0 * 3.141592653589793) + (z + 0.5) * std::log(t) - t + std::log(series);
}

// digamma: recurrence to x >= 6, then the asymptotic series (beta.rs:77-86).
// Departure: x <= 0 and NaN return NaN (Beta parameters are positive); the
// reference's recurrence would run about |x| steps there, forever below -2^53.
extern "C" double sfo_digamma(double x) {
    if (!(x > 0.0)) return std::nan("");
    double r = 0.0;
    while (x < 6.0) { r -= 1.0 / x; x += 1.0; }
    const double inv = 1.0 / x, inv2 = inv * inv;
    return r + std::log(x) - 0.5 * inv - inv2 / 12.0 + inv2 * inv2 / 120.0 -
           inv2 * inv2 * inv2 / 252.0;
}

// beta_entropy (beta.rs:92-96).
extern "C" double sfo_beta_entropy(double a, double b) {
    const double s = a + b;
    return sfo_lgamma(a) + sfo_lgamma(b) - sfo_lgamma(s) - (a - 1.0) * sfo_digamma(a) -
           (b - 1.0) * sfo_digamma(b) + (s - 2.0) * sfo_digamma(s);
}

// build_entropy_table (beta.rs:100-112): axis_i = exp(f64(f32(i) * LN_STEP)).
extern "C" void sfo_entropy_table(float* table) {
    double axis[kGridPts];
    for (int i = 0; i < kGridPts; ++i) axis[i] = std::exp((double)((float)i * kLnStep));
#pragma omp parallel for schedule(static)
    for (int i = 0; i < kGridPts; ++i)
        for (int j = 0; j < kGridPts; ++j)
            table[i * kGridPts + j] = (float)sfo_beta_entropy(axis[i], axis[j]);
}

// table_entropy (beta.rs:128-144): bilinear in (ln a, ln b)/LN_STEP, edge-clamped.
extern "C" float sfo_table_entropy(float a, float b, const float* table) {
    const float xa = logf_c(a) / kLnStep;
    const float xb = logf_c(b) / kLnStep;
    const float ia = minf(maxf(std::floor(xa), 0.0f), (float)(kGridPts - 2));
    const float ib = minf(maxf(std::floor(xb), 0.0f), (float)(kGridPts - 2));
    const float ta = clampf(xa - ia, 0.0f, 1.0f);
    const float tb = clampf(xb - ib, 0.0f, 1.0f);
    const size_t row = (size_t)sat_u32(ia) * kGridPts + sat_u32(ib);
    const float h00 = table[row], h10 = table[row + kGridPts];
    const float h01 = table[row + 1], h11 = table[row + kGridPts + 1];
    return (((h00 * (1.0f - ta)) * (1.0f - tb) + (h10 * ta) * (1.0f - tb)) +
            (h01 * (1.0f - ta)) * tb) + (h11 * ta) * tb;
}

// entropy_delta_kernel per-splat body (beta.rs:170-186).
extern "C" float sfo_delta_lut(float a, float b, uint32_t resp_bits, float scale,
                               const float* table) {
    const float eps = (float)resp_bits / scale;
    if (!(eps > 0.0f)) return 0.0f;
    const float k = 1.0f + eps / (a + b);
    const float a2 = a * k, b2 = b * k;
    return maxf(sfo_table_entropy(a, b, table) - sfo_table_entropy(a2, b2, table), 0.0f);
}

// Same delta from the f64 formulas, posterior scale form in f64.
extern "C" double sfo_delta_f64(float a, float b, uint32_t resp_bits, float scale) {
    const double eps = (double)resp_bits / (double)scale;
    if (!(eps > 0.0)) return 0.0;
    const double ad = a, bd = b;
    const double k = 1.0 + eps / (ad + bd);
    const double d = sfo_beta_entropy(ad, bd) - sfo_beta_entropy(ad * k, bd * k);
    return d > 0.0 ? d : 0.0;
}

extern "C" double sfo_eig(int mode, const float* a, const float* b, const uint32_t* resp,
                          uint32_t n, float scale, const float* table) {
    double total = 0.0;
#pragma omp parallel for schedule(static) reduction(+ : total)
    for (int64_t i = 0; i < (int64_t)n; ++i) {
        if (mode == 0)
            total += (double)sfo_delta_lut(a[i], b[i], resp[i], scale, table);
        else
            total += sfo_delta_f64(a[i], b[i], resp[i], scale);
    }
    return total;
}

// beta_update_kernel (beta.rs:206-212).
extern "C" void sfo_beta_update(float scale, const uint32_t* fg, const uint32_t* bg, float* a,
                                float* b, uint32_t n) {
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)n; ++i) {
        a[i] = a[i] + (float)fg[i] / scale;
        b[i] = b[i] + (float)bg[i] / scale;
    }
}
