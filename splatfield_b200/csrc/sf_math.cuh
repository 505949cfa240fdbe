// Scalar arithmetic of the splat path, shared by every kernel.
//
// The reference leaves exp/ln/sqrt/inverse_sqrt/recip rounding to each GPU
// driver's WGSL builtins (src/project.rs:264-318, src/raster.rs:187), so this
// path fixes one definition and keeps it on host and device alike:
//  * exp: Cody–Waite reduction x = k*ln2 + r (ln2 as a 16-bit head plus a
//    tail; Cody & Waite, "Software Manual for the Elementary Functions",
//    1980), degree-7 Taylor polynomial of e^r on |r| <= ln2/2 in Horner form,
//    scaling by 2^k in two exact multiplies so subnormal results round once;
//  * log: x = 2^e*m, m in [sqrt(1/2), sqrt(2)); ln m = 2*atanh(s),
//    s = (m-1)/(m+1), odd series through s^9/9;
//  * division and sqrt correctly rounded (nvcc -prec-div/-prec-sqrt defaults),
//    inverse_sqrt = 1/sqrt(x);
//  * no implicit contraction: translation units are built with -fmad=false
//    and every fused multiply-add is an explicit fmaf.
// The CPU oracle states the same methods independently; parity tests hold
// the two bit-equal.
#pragma once
#include <cstdint>
#include <cmath>

#ifdef __CUDACC__
#define SF_HD __host__ __device__ __forceinline__
#else
#define SF_HD inline
#endif

namespace sfm {

SF_HD uint32_t f2u(float f) {
#ifdef __CUDA_ARCH__
    return __float_as_uint(f);
#else
    uint32_t u;
    __builtin_memcpy(&u, &f, 4);
    return u;
#endif
}

SF_HD float u2f(uint32_t u) {
#ifdef __CUDA_ARCH__
    return __uint_as_float(u);
#else
    float f;
    __builtin_memcpy(&f, &u, 4);
    return f;
#endif
}

SF_HD float fma_(float a, float b, float c) {
#ifdef __CUDA_ARCH__
    return __fmaf_rn(a, b, c);
#else
    return std::fma(a, b, c);
#endif
}

SF_HD float rint_(float x) {
#ifdef __CUDA_ARCH__
    return rintf(x);
#else
    return std::rint(x);
#endif
}

SF_HD float exp_(float x) {
    if (x != x) return x;
    if (x < -103.0f) return 0.0f;
    if (x > 88.8f) return INFINITY;
    const float kf = rint_(x * 1.44269502f);
    float r = fma_(kf, -0.693145751953125f, x);
    r = fma_(kf, -1.42860677e-06f, r);
    float p = 1.98412701e-04f;
    p = fma_(p, r, 1.38888892e-03f);
    p = fma_(p, r, 8.33333377e-03f);
    p = fma_(p, r, 4.16666679e-02f);
    p = fma_(p, r, 1.66666672e-01f);
    p = fma_(p, r, 0.5f);
    p = fma_(p, r, 1.0f);
    p = fma_(p, r, 1.0f);
    const int k = (int)kf;
    const int k1 = k / 2;
    const int k2 = k - k1;
    return (p * u2f((uint32_t)(k1 + 127) << 23)) * u2f((uint32_t)(k2 + 127) << 23);
}

// exp for arguments known to lie in [-86, 0] (the raster's -power, which the
// power_max test bounds far tighter): the value of exp_ bit for bit, in fewer
// instructions.
//  * k = rint(x*log2e) by the round-to-integer shift: t + 1.5*2^23 rounds t
//    to an integer with ties to even (the rounding rint uses) for
//    |t| < 2^22, and that sum's low mantissa bits hold k in two's complement.
//  * The two-step 2^k scale equals one add of k to p's exponent field: for
//    k >= -125 and p in [0.7, 1.42] every step is exact and p*2^k is normal.
SF_HD float exp_neg_(float x) {
    const float kr = x * 1.44269502f + 12582912.0f;
    const float kf = kr - 12582912.0f;
    float r = fma_(kf, -0.693145751953125f, x);
    r = fma_(kf, -1.42860677e-06f, r);
    float p = 1.98412701e-04f;
    p = fma_(p, r, 1.38888892e-03f);
    p = fma_(p, r, 8.33333377e-03f);
    p = fma_(p, r, 4.16666679e-02f);
    p = fma_(p, r, 1.66666672e-01f);
    p = fma_(p, r, 0.5f);
    p = fma_(p, r, 1.0f);
    p = fma_(p, r, 1.0f);
    return u2f(f2u(p) + (f2u(kr) << 23));
}

SF_HD float log_(float x) {
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
    float p = fma_(s2, 0.111111112f, 0.142857149f);
    p = fma_(p, s2, 0.2f);
    p = fma_(p, s2, 0.333333343f);
    const float two_s = s + s;
    const float lnm = fma_(two_s * s2, p, two_s);
    const float ef = (float)e;
    return fma_(ef, 0.693145751953125f, fma_(ef, 1.42860677e-06f, lnm));
}

SF_HD float sigmoid_(float x) { return 1.0f / (1.0f + exp_(-x)); }

// Rust `f32 as u32`: saturating, NaN -> 0. On the device one truncating
// conversion (cvt.rzi.u32.f32 clamps to the destination range and gives 0
// for NaN), the same value as the host's rule for every one of the 2^32
// float patterns (checked exhaustively on a B200).
SF_HD uint32_t sat_u32(float v) {
#ifdef __CUDA_ARCH__
    return __float2uint_rz(v);
#else
    if (!(v > 0.0f)) return 0u;
    if (v >= 4294967296.0f) return 0xffffffffu;
    return (uint32_t)v;
#endif
}

// Rust f32::clamp (NaN passes through).
SF_HD float clamp_(float v, float lo, float hi) {
    if (v < lo) v = lo;
    if (v > hi) v = hi;
    return v;
}

SF_HD float min_(float a, float b) { return fminf(a, b); }
SF_HD float max_(float a, float b) { return fmaxf(a, b); }

}  // namespace sfm
