// store16.cuh — 16-bit wavefield storage as the z-marching kernels see it
// (kernels_zmarch.cu, kernels_zpair.cu): value h of field g reads back as
// float(h) * 2^e_g, and v is stored as RN16(v * 2^-e_g), binary16 saturating
// at +-65504 — the roundings of kernels_half.cu and of the oracle.
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <cstdint>

#include "../../include/sgfd.h"
#include "sgfd_internal.h"

namespace sgfd {

template <int ST>
struct H16 {
    __device__ __forceinline__ static float h2f(uint32_t h) {
        if (ST == SGFD_STORE_BF16) return __uint_as_float(h << 16);
        return __half2float(__ushort_as_half((unsigned short)h));
    }
    __device__ __forceinline__ static uint32_t f2h(float w) {
        if (ST == SGFD_STORE_BF16) return __bfloat16_as_ushort(__float2bfloat16_rn(w));
        return __half_as_ushort(__float2half_rn(fminf(fmaxf(w, -65504.0f), 65504.0f)));
    }
};

// Largest |v| of the warp's active lanes into field g's running maximum (the
// rescale steps of 16-bit storage, as kernels_half.cu notes them).
__device__ __forceinline__ void note_max16(const HalfState &hs, int g, float v) {
    const unsigned mask = __activemask();
    const unsigned bits = __reduce_max_sync(mask, __float_as_uint(fabsf(v)));
    if ((threadIdx.x & 31) == __ffs(mask) - 1) atomicMax(hs.amax + g, bits);
}

// The same into a CTA's shared running maxima (smax[g], unsigned float
// bits); the CTA adds them to the global ones once (flush_max16).
__device__ __forceinline__ void note_max16s(unsigned *smax, int g, float v) {
    const unsigned mask = __activemask();
    const unsigned bits = __reduce_max_sync(mask, __float_as_uint(fabsf(v)));
    if ((threadIdx.x & 31) == __ffs(mask) - 1) atomicMax(smax + g, bits);
}
// After a barrier: threads 0..8 add the CTA's maxima to the global ones.
__device__ __forceinline__ void flush_max16(const HalfState &hs, const unsigned *smax) {
    if (threadIdx.x < 9 && smax[threadIdx.x] != 0u) atomicMax(hs.amax + threadIdx.x, smax[threadIdx.x]);
}

}  // namespace sgfd
