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

// Damping factors m = 1 - q r^2, p = 1 + q r^2 of one damped axis at band
// distance k (1..pml).  d_axis is dx, dy or dz.
__device__ __forceinline__ void damp_factors(const Physics &ph, int axis, float d_axis, int k,
                                             int pml, float mu, float b, float lam,
                                             float &m, float &p) {
    float q;
    if (ph.damping == 0) {                    // SGFD_DAMP_REFGPU: Vs = sqrt(mu*b)
        const float vs = sqrtf(mu * b);
        q = ((ph.q_refgpu * vs) / d_axis) * ph.poly;
    } else if (ph.damping == 1) {             // SGFD_DAMP_LOGR: Vp = sqrt((lambda+2mu)*b)
        const float vp = sqrtf(__fmaf_rn(2.0f, mu, lam) * b);
        q = (ph.q_logr * vp) / d_axis;
    } else {                                  // SGFD_DAMP_REFCPU: constant velocity
        q = ph.q_refcpu[axis];
    }
    const float r = (float)k / (float)pml;
    const float pw = r * r;
    m = __fmaf_rn(-q, pw, 1.0f);
    p = __fmaf_rn(q, pw, 1.0f);
}

// One split-field update: (m*s + A*B)/p on a damped axis, s + A*B otherwise.
__device__ __forceinline__ float split_update(float s, float A, float B, bool damped, float m, float p) {
    return damped ? __fmaf_rn(m, s, A * B) / p : __fmaf_rn(A, B, s);
}

}  // namespace sgfd
