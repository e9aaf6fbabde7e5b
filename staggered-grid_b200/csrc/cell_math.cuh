// cell_math.cuh — per-cell arithmetic of the staggered-grid update, shared by
// every kernel family so that all of them round identically.
//
// Operation order is fixed and every fused multiply-add is explicit
// (__fmaf_rn); the library is compiled with -fmad=false so nothing else is
// contracted.  The CPU oracle performs the same operations, which makes the
// FP32 GPU path and the FP32 oracle agree bit for bit.
//
// Reference mapping (3DGPUwithPML_1DArraySingleGPU_optimization/):
//   forward/backward staggered differences   ElasticWaveEquation.cu:244-276, 541-591
//   interior velocity / stress updates       ElasticWaveEquation.cu:253,265,277, 550-592
//   PML damping (REFGPU profile)             ElasticMacro.h:26-27, ElasticWaveEquation.cu:282-288
//   split-field updates                      ElasticMacro.h:409-531
#pragma once

#include <type_traits>

#include "sgfd_internal.h"

namespace sgfd {

// sum_i c_i (g(1+i) - g(-i)): the difference centred half a cell ahead.
template <class G>
__device__ __forceinline__ float dfwd(const float (&c)[5], G g) {
    float d = 0.0f;
#pragma unroll
    for (int i = 0; i < 5; ++i) d = __fmaf_rn(c[i], g(1 + i) - g(-i), d);
    return d;
}

// sum_i c_i (g(i) - g(-1-i)): the difference centred half a cell behind.
template <class G>
__device__ __forceinline__ float dbwd(const float (&c)[5], G g) {
    float d = 0.0f;
#pragma unroll
    for (int i = 0; i < 5; ++i) d = __fmaf_rn(c[i], g(i) - g(-1 - i), d);
    return d;
}

#ifndef SGFD_REFDIV
#define SGFD_REFDIV 2
#endif

// a / d correctly rounded (IEEE round to nearest), for d = the cell size
// along `axis`, the divisor of every REF staggered difference.  The divisor is
// known in advance, so no division instruction is needed:
//   * double-precision reciprocal: q = RN32(RN64(a * RN64(1/d))).  The
//     computed double is within 2^-52 (relative) of a/d, while a quotient of
//     two binary32 numbers is never a binary32 midpoint and stays more than
//     2^-50 (relative) away from every one (a - m d is a nonzero multiple of
//     2^(e_a - 26) for a midpoint m, and |a| < 2^(e_a + 24)), so the final
//     rounding lands on RN32(a/d): the double-rounding argument of
//     S. A. Figueroa, "When is double rounding innocuous?", SIGNUM Newsl.
//     30(3), 1995, for a product with a reciprocal accurate to 2^-53.
//     Subnormal results included; zeros keep their sign.
//   * single-precision correction step: q0 = RN(a y), y = RN(1/d);
//     t = RN(q0 d - a) (exact); q = RN(q0 - t y) — P. Markstein's correction
//     (IBM J. Res. Dev. 34(1), 1990) in the known-divisor form of Brisebarre,
//     Muller and Raina (IEEE Trans. Computers 53(8), 2004).  Whether it is
//     exact for every a depends on d; the host checks every significand of
//     one binade (ph.mdiv), which covers all |a| in [2^-100, 2^100] by
//     scaling, and tiny nonzero |a|, where t would lose bits, divide.
__device__ __forceinline__ float div_cell(const Physics &ph, int axis, float a) {
    const float d = axis == 0 ? ph.dx : axis == 1 ? ph.dy : ph.dz;
#if SGFD_REFDIV == 2
    (void)d;
    return __double2float_rn(__dmul_rn((double)a, ph.rd64[axis]));
#elif SGFD_REFDIV == 1
    if (!((ph.mdiv >> axis) & 1)) return __fdiv_rn(a, d);
    const float y = ph.rd[axis];
    const float q0 = __fmul_rn(a, y);
    const float t = __fmaf_rn(q0, d, -a);
    float q = __fmaf_rn(-t, y, q0);
    const float aa = fabsf(a);
    if (!(aa >= 0x1p-100f && aa <= 0x1p100f) && aa != 0.0f) q = __fdiv_rn(a, d);
    return q;
#else
    return __fdiv_rn(a, d);
#endif
}

// A difference sum divided by the cell size of `axis` (REF), or as it is
// (FAST sums are formed with the pre-divided coefficients).
template <bool FAST>
__device__ __forceinline__ float by_cell(const Physics &ph, int axis, float sum) {
    return FAST ? sum : div_cell(ph, axis, sum);
}

// Staggered difference along AXIS (0, 1, 2 = x, y, z) divided by the cell
// size: REF divides the sum (reference expression), FAST uses the
// pre-divided coefficients c_i / d.
template <bool FAST, int AXIS, class G>
__device__ __forceinline__ float dF(const Physics &ph, G g) {
    if (FAST) return dfwd(ph.cs[AXIS], g);
    return div_cell(ph, AXIS, dfwd(ph.c, g));
}
template <bool FAST, int AXIS, class G>
__device__ __forceinline__ float dB(const Physics &ph, G g) {
    if (FAST) return dbwd(ph.cs[AXIS], g);
    return div_cell(ph, AXIS, dbwd(ph.c, g));
}

// Two staggered differences at once on packed FP32x2 (sm_100 fma.rn.f32x2):
// lane 0 of every operand belongs to the first difference, lane 1 to the
// second; plus(i) and minus(i) give term i's taps of both (forward g(1+i),
// g(-i); backward g(i), g(-1-i)) and c their coefficients.  Each lane does
// exactly what dfwd / dbwd do: the tap difference a - b is computed as
// fma(b, -1, a), which rounds to the same value.
template <class P, class M>
__device__ __forceinline__ float2 dpair(const float2 (&c)[5], P plus, M minus) {
    const float2 neg1 = make_float2(-1.0f, -1.0f);
    float2 d = make_float2(0.0f, 0.0f);
#pragma unroll
    for (int i = 0; i < 5; ++i) d = __ffma2_rn(c[i], __ffma2_rn(minus(i), neg1, plus(i)), d);
    return d;
}

// The same differences for two vertically adjacent cells (rows r and r+1)
// that share one 11-value window, g(o) being the value o rows from row r:
// forward windows span rows r-4 .. r+6, backward windows r-5 .. r+5.  Each
// cell's sum is rounded exactly as dF / dB round it.
template <bool FAST, int AXIS, class G>
__device__ __forceinline__ void dF2(const Physics &ph, G g, float &d0, float &d1) {
    float v[11];
#pragma unroll
    for (int j = 0; j < 11; ++j) v[j] = g(j - 4);
    d0 = dF<FAST, AXIS>(ph, [&](int o) { return v[o + 4]; });
    d1 = dF<FAST, AXIS>(ph, [&](int o) { return v[o + 5]; });
}
template <bool FAST, int AXIS, class G>
__device__ __forceinline__ void dB2(const Physics &ph, G g, float &d0, float &d1) {
    float v[11];
#pragma unroll
    for (int j = 0; j < 11; ++j) v[j] = g(j - 5);
    d0 = dB<FAST, AXIS>(ph, [&](int o) { return v[o + 5]; });
    d1 = dB<FAST, AXIS>(ph, [&](int o) { return v[o + 6]; });
}

// Harmonic mean 4 / (r0 + r1 + r2 + r3) of four reciprocals of mu
// (ElasticMacro.h:111-112).  FAST computes 4 * RN(1/s), equal to RN(4/s)
// because scaling by 4 is exact.
template <bool FAST>
__device__ __forceinline__ float hmean(float r0, float r1, float r2, float r3) {
    const float s = ((r0 + r1) + r2) + r3;
    return FAST ? 4.0f * __frcp_rn(s) : 4.0f / s;
}

// Wave speed the damping profile scales with, computed once per cell:
// REFGPU the local shear speed sqrt(mu*b) (OPT/ElasticWaveEquation.cu:282),
// LOGR the local P speed sqrt((lambda+2mu)*b), REFCPU unused.
__device__ __forceinline__ float damp_speed(const Physics &ph, float mu, float b, float lam) {
    if (ph.damping == 0) return sqrtf(mu * b);
    if (ph.damping == 1) return sqrtf(__fmaf_rn(2.0f, mu, lam) * b);
    return 0.0f;
}

// The divisor of a damped split update as the updates take it: FAST the
// correctly rounded reciprocal RN(1/p) (the update multiplies by it); REF a
// 64-bit reciprocal of p within 2^-52 (relative), so that RN32(num * r) is
// the correctly rounded num / p (recip64).
template <bool FAST>
using PDiv = typename std::conditional<FAST, float, double>::type;

// 1/p in double precision within 2^-52 (relative): a single-precision
// approximation refined by two Newton steps r += r (1 - p r), each squaring
// the error (2^-21 -> 2^-42 -> below the steps' own rounding).  Then
// RN32(num * r) = RN32(num / p) for every binary32 num, by the argument of
// div_cell: the product lies within 2^-52 of num/p, every binary32 midpoint
// more than 2^-50 away from it.  Divisors outside [2^-100, 2^100] (never a
// damping divisor, which is at least 1) take a correctly rounded double
// division instead.
__device__ __forceinline__ double recip64(float p) {
    const float ap = fabsf(p);
    if (!(ap >= 0x1p-100f && ap <= 0x1p100f)) return __drcp_rn((double)p);
    float y;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(p));
    const double pd = (double)p;
    double r = (double)y;
    double e = __fma_rn(-pd, r, 1.0);
    r = __fma_rn(r, e, r);
    e = __fma_rn(-pd, r, 1.0);
    return __fma_rn(r, e, r);
}

// Damping factors of one damped axis at band distance k (1..pml):
// m = 1 - q r^2 and p = 1 + q r^2 (ElasticMacro.h:26-27 inside
// 1 -/+ 0.5*dt*DAMPING), p in the form of PDiv.  d_axis is dx, dy or dz; v
// is damp_speed() of the cell.
template <bool FAST>
__device__ __forceinline__ void damp_factors(const Physics &ph, int axis, float d_axis, int k, int pml, float v,
                                             float &m, PDiv<FAST> &p) {
    float q;
    (void)d_axis;
    if (ph.damping == 0) {                    // SGFD_DAMP_REFGPU
        q = FAST ? v * ph.qf[axis] : div_cell(ph, axis, ph.q_refgpu * v) * ph.poly;
    } else if (ph.damping == 1) {             // SGFD_DAMP_LOGR
        q = FAST ? v * ph.qf[axis] : div_cell(ph, axis, ph.q_logr * v);
    } else {                                  // SGFD_DAMP_REFCPU: constant velocity
        q = ph.q_refcpu[axis];
    }
    float pw;
    if (k < kPwTable) {
        pw = ph.pw[k];
    } else {
        const float r = (float)k / (float)pml;
        pw = r * r;
    }
    m = __fmaf_rn(-q, pw, 1.0f);
    const float pf = __fmaf_rn(q, pw, 1.0f);
    if constexpr (FAST) p = __frcp_rn(pf);
    else p = recip64(pf);
}

// One split-field update: (m*s + A*B)/p on a damped axis (FAST: times RN(1/p);
// REF: the correctly rounded quotient through the 64-bit reciprocal), s + A*B
// otherwise.
template <bool FAST>
__device__ __forceinline__ float split_update(float s, float A, float B, bool damped, float m, PDiv<FAST> p) {
    if (!damped) return __fmaf_rn(A, B, s);
    const float num = __fmaf_rn(m, s, A * B);
    if constexpr (FAST) return num * p;
    else return __double2float_rn(__dmul_rn((double)num, p));
}

}  // namespace sgfd
