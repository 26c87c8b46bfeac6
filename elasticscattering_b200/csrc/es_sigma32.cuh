// es_sigma32.cuh - GetSigma (src/sim/es/util.h:34-46) in FP32 for one orbit:
// the Boltzmann kernel of the split-precision paths (the per-pass FP32
// integration in es_integrate.cu and the batched kernel in es_batch.cu).
#pragma once

#include "es_internal.h"

namespace es {

// sin and cos of an FP64 angle, evaluated in FP32. The quadrant reduction
// x = q pi/2 + r, |r| <= pi/4, is done in FP64 (exact enough for any |x| the
// kernel meets, a few thousand radians at most); sin r and cos r are their
// Taylor polynomials (degree 9 and 10: truncation below 2e-9 on |r| <= pi/4),
// evaluated by Horner's rule in FP32 with explicit fused multiply-adds (the
// translation units that include this header are compiled without automatic
// contraction, for their FP64 paths). Measured against FP64 sin/cos over
// [-50, 50] and down to |x| = 1e-12: at most 1.5 ulp. The code is short and
// branch-free, which matters in a kernel limited by instruction issue.
__device__ __forceinline__ void sincos_reduced(double x, float& s_out, float& c_out)
{
    constexpr double kTwoOverPi = 0.636619772367581343076;
    constexpr double kHalfPi = 1.570796326794896619231;
    const double q = rint(x * kTwoOverPi);
    const float r = (float)fma(-q, kHalfPi, x);
    const float r2 = r * r;
    const float s =
        fmaf(r * r2, fmaf(r2, fmaf(r2, fmaf(r2, 1.0f / 362880.0f, -1.0f / 5040.0f), 1.0f / 120.0f), -1.0f / 6.0f), r);
    const float c = fmaf(
        r2, fmaf(r2, fmaf(r2, fmaf(r2, fmaf(r2, -1.0f / 3628800.0f, 1.0f / 40320.0f), -1.0f / 720.0f), 1.0f / 24.0f),
                 -0.5f),
        1.0f);
    const int n = ((int)(long long)q) & 3;
    s_out = (n == 0) ? s : (n == 1) ? c : (n == 2) ? -s : -c;
    c_out = (n == 0) ? c : (n == 1) ? -s : (n == 2) ? -c : s;
}

// sincos_reduced with the quadrant taken by the round-to-integer constant
// 1.5 * 2^52 instead of rint and an FP64-to-integer conversion: fma(x, 2/pi,
// 1.5 * 2^52) holds round(x * 2/pi) in its low mantissa bits (|x| * 2/pi
// below 2^51), read with a register move. The polynomials are sincos_reduced's.
__device__ __forceinline__ void sincos_reduced_fast(double x, float& s_out, float& c_out)
{
    constexpr double kTwoOverPi = 0.636619772367581343076;
    constexpr double kHalfPi = 1.570796326794896619231;
    constexpr double kRound = 6755399441055744.0;  // 1.5 * 2^52
    const double t = fma(x, kTwoOverPi, kRound);
    const double q = t - kRound;
    const float r = (float)fma(-q, kHalfPi, x);
    const float r2 = r * r;
    const float s =
        fmaf(r * r2, fmaf(r2, fmaf(r2, fmaf(r2, 1.0f / 362880.0f, -1.0f / 5040.0f), 1.0f / 120.0f), -1.0f / 6.0f), r);
    const float c = fmaf(
        r2, fmaf(r2, fmaf(r2, fmaf(r2, fmaf(r2, -1.0f / 3628800.0f, 1.0f / 40320.0f), -1.0f / 720.0f), 1.0f / 24.0f),
                 -0.5f),
        1.0f);
    const int n = __double2loint(t) & 3;
    s_out = (n == 0) ? s : (n == 1) ? c : (n == 2) ? -s : -c;
    c_out = (n == 0) ? c : (n == 1) ? -s : (n == 2) ? -c : s;
}

// 1 - exp(-x) for x >= 0 in FP32: the Taylor series (degree 8, nested) below
// 0.5, where 1 - exp(-x) would cancel; 1 - expf(-x) above. Relative error
// below 2e-7 on [1e-10, 15].
__device__ __forceinline__ float one_minus_exp_neg(float x)
{
    if (x < 0.5f) {
        // x (1 - x/2 (1 - x/3 (1 - x/4 (1 - x/5 (1 - x/6 (1 - x/7 (1 - x/8)))))))
        float t = fmaf(-x, 0.125f, 1.0f);
        t = fmaf(-x * (1.0f / 7.0f), t, 1.0f);
        t = fmaf(-x * (1.0f / 6.0f), t, 1.0f);
        t = fmaf(-x * 0.2f, t, 1.0f);
        t = fmaf(-x * 0.25f, t, 1.0f);
        t = fmaf(-x * (1.0f / 3.0f), t, 1.0f);
        t = fmaf(-x * 0.5f, t, 1.0f);
        return x * t;
    }
    return 1.0f - expf(-x);
}

// GetSigma for a lifetime lt (already truncated at 15 tau by the caller), FP32.
// With z = exp(-t/tau), e1 = 1 - z, h = w t / 2:
//   cos(phi) - z cos(phi + 2h)       = cos(phi) e1 + 2 z sin(h) sin(phi + h)
//   w tau (z sin(phi + 2h) - sin(phi)) = w tau (2 z sin(h) cos(phi + h) - e1 sin(phi))
// Both right-hand sides are sums of products of well-conditioned factors, so
// each orbit's value keeps FP32 relative accuracy even for t << tau, where
// the left-hand sides cancel (there FP32 loses up to 1e-5 of sigma_xy). The
// angles h and phi + h are formed and reduced in FP64 (sigma_angles); they
// depend on lt only, so temperatures whose 15 tau does not truncate share them.
struct SigmaAngles {
    float sh, ch, sp, cp;  // sin h, cos h, sin(phi + h), cos(phi + h)
};

__device__ __forceinline__ SigmaAngles sigma_angles(double lt, double w_signed, const PhaseSigma& ph)
{
    const double h = 0.5 * w_signed * lt;
    SigmaAngles a;
    sincos_reduced(h, a.sh, a.ch);
    sincos_reduced(ph.phi + h, a.sp, a.cp);
    return a;
}

__device__ __forceinline__ void sigma_fp32_at(const SigmaAngles& a, double lt, double inv_tau, double wtau,
                                              const PhaseSigma& ph, float& r_xx, float& r_xy)
{
    const float c = (float)ph.cos_phi, s = (float)ph.sin_phi;
    const float e1 = one_minus_exp_neg((float)(lt * inv_tau));
    const float z = 1.0f - e1;
    const float zs = 2.0f * z * a.sh;
    const float wt = (float)wtau;
    const float r = fmaf(wt, fmaf(zs, a.cp, -e1 * s), fmaf(c, e1, zs * a.sp));
    r_xx = r * c;
    r_xy = r * s;
}

// GetSigma of the lifetime `raw` truncated at max_lt (GetTruncatedLifetimes).
__device__ __forceinline__ void sigma_fp32(double raw, double max_lt, double inv_tau, double w_signed, double wtau,
                                           const PhaseSigma& ph, float& r_xx, float& r_xy)
{
    const double lt = raw < max_lt ? raw : max_lt;
    sigma_fp32_at(sigma_angles(lt, w_signed, ph), lt, inv_tau, wtau, ph, r_xx, r_xy);
}

}  // namespace es
