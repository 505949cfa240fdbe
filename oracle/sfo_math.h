// Oracle scalar arithmetic: the canonical f32 operations of the splat path.
//
// TEST INFRASTRUCTURE ONLY. This directory is the CPU restatement of the
// reference's render + segmentation-evidence path; only the test suite, the
// smoke check and the benchmark's CPU-baseline leg may load it, and only as the
// checker.
//
// The reference (suous/splatfield, Rust/cubecl on wgpu) evaluates `exp`, `ln`,
// `sqrt`, `inverse_sqrt` and `recip` with WGSL builtins whose rounding is left
// to each GPU driver (src/project.rs:264-268, :277, :313-318;
// src/raster.rs:187). Bit parity between a CPU oracle and a CUDA kernel needs
// one definition of those functions, so both sides use the methods below:
//
//  * exp: Cody–Waite range reduction x = k·ln2 + r with ln2 split into a
//    16-bit head and a tail (Cody & Waite, "Software Manual for the Elementary
//    Functions", 1980), then the degree-7 Taylor polynomial of e^r on
//    |r| <= ln2/2 (truncation < 6e-9 relative), then scaling by 2^k in two
//    exact steps.
//  * log: x = 2^e·m with m in [sqrt(1/2), sqrt(2)), ln m = 2·atanh(s),
//    s = (m-1)/(m+1), by the odd series s + s^3/3 + ... + s^9/9
//    (|s| <= 0.1716, truncation < 3e-9 relative).
//  * sqrt and division: IEEE correctly rounded on both sides;
//    inverse_sqrt = 1/sqrt(x) (two correctly rounded operations).
//  * No contraction: every fused multiply-add is written as fmaf; the file is
//    compiled with -ffp-contract=off (CUDA side: -fmad=false).
#pragma once
#include <cmath>
#include <cstdint>
#include <cstring>

namespace sfo {

inline uint32_t f2u(float f) { uint32_t u; std::memcpy(&u, &f, 4); return u; }
inline float u2f(uint32_t u) { float f; std::memcpy(&f, &u, 4); return f; }

inline float expf_c(float x) {
    if (x != x) return x;
    if (x < -103.0f) return 0.0f;
    if (x > 88.8f) return INFINITY;
    const float kf = std::rint(x * 1.44269502f);
    float r = std::fma(kf, -0.693145751953125f, x);
    r = std::fma(kf, -1.42860677e-06f, r);
    float p = 1.98412701e-04f;                 // 1/7!
    p = std::fma(p, r, 1.38888892e-03f);       // 1/6!
    p = std::fma(p, r, 8.33333377e-03f);       // 1/5!
    p = std::fma(p, r, 4.16666679e-02f);       // 1/4!
    p = std::fma(p, r, 1.66666672e-01f);       // 1/3!
    p = std::fma(p, r, 0.5f);
    p = std::fma(p, r, 1.0f);
    p = std::fma(p, r, 1.0f);
    const int k = (int)kf;
    const int k1 = k / 2;
    const int k2 = k - k1;
    const float s1 = u2f((uint32_t)(k1 + 127) << 23);
    const float s2 = u2f((uint32_t)(k2 + 127) << 23);
    return (p * s1) * s2;
}

inline float logf_c(float x) {
    if (x != x || x < 0.0f) return NAN;
    if (x == 0.0f) return -INFINITY;
    if (x == INFINITY) return x;
    int e = 0;
    if (x < 1.17549435e-38f) { x = x * 8388608.0f; e = -23; }
    const uint32_t bits = f2u(x);
    e += (int)((bits >> 23) & 0xffu) - 127;
    float m = u2f((bits & 0x007fffffu) | 0x3f800000u);
    if (m > 1.41421354f) { m = m * 0.5f; e += 1; }
    const float f = m - 1.0f;
    const float s = f / (2.0f + f);
    const float s2 = s * s;
    float p = std::fma(s2, 0.111111112f, 0.142857149f);   // 1/9, 1/7
    p = std::fma(p, s2, 0.2f);
    p = std::fma(p, s2, 0.333333343f);
    const float two_s = s + s;
    const float lnm = std::fma(two_s * s2, p, two_s);
    const float ef = (float)e;
    return std::fma(ef, 0.693145751953125f, std::fma(ef, 1.42860677e-06f, lnm));
}

inline float sigmoid(float x) { return 1.0f / (1.0f + expf_c(-x)); }

// Rust `f32 as u32`: saturating, NaN -> 0 (the reference casts clamped floats).
inline uint32_t sat_u32(float v) {
    if (!(v > 0.0f)) return 0u;
    if (v >= 4294967296.0f) return 0xffffffffu;
    return (uint32_t)v;
}

// Rust f32::clamp: NaN passes through.
inline float clampf(float v, float lo, float hi) {
    if (v < lo) v = lo;
    if (v > hi) v = hi;
    return v;
}

// Rust f32::min / f32::max (IEEE minNum/maxNum, same as fminf/fmaxf).
inline float minf(float a, float b) { return std::fmin(a, b); }
inline float maxf(float a, float b) { return std::fmax(a, b); }

}  // namespace sfo
