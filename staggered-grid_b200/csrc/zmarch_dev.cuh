// zmarch_dev.cuh — device helpers shared by the z-marching kernel families
// (kernels_zmarch.cu, kernels_zpair.cu): mbarrier waits with an iteration
// cap, TMA tiled loads (no multicast), shared-memory alignment and the
// bounded grid barrier of the persistent batch kernel.
#pragma once

#include <cuda.h>

#include <cstdint>

#include "sgfd_internal.h"

namespace sgfd {
namespace zdev {

constexpr uint32_t kWaitCap = 2000;
constexpr uint32_t kSuspendNs = 1000000;

__device__ __forceinline__ uint32_t sptr(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(sptr(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(sptr(bar)), "r"(bytes) : "memory");
}
// One poll of the phase; the thread may sleep in the poll for up to
// kSuspendNs (it wakes as soon as the phase completes).
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok) : "r"(sptr(bar)), "r"(parity), "n"(kSuspendNs) : "memory");
    return ok != 0;
}
// Bounded wait: false after kWaitCap polls (about kWaitCap * kSuspendNs at most).
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity) {
    for (uint32_t i = 0; i < kWaitCap; ++i)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}
__device__ __forceinline__ void fence_barrier_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void tma3(void *dst, const CUtensorMap *map, int x, int y, int z, uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];"
        ::"r"(sptr(dst)), "l"(map), "r"(x), "r"(y), "r"(z), "r"(sptr(bar))
        : "memory");
}

// 4-D tiled load: box at (x, y, z, w) of the map into dst.
__device__ __forceinline__ void tma4(void *dst, const CUtensorMap *map, int x, int y, int z, int w, uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], [%6];"
        ::"r"(sptr(dst)), "l"(map), "r"(x), "r"(y), "r"(z), "r"(w), "r"(sptr(bar))
        : "memory");
}

// Bring [p, p + bytes) into L2 (p 16-byte aligned, bytes a multiple of 16).
// A hint: it returns no data and completes on no barrier.
__device__ __forceinline__ void l2_prefetch(const void *p, uint32_t bytes) {
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p), "r"(bytes) : "memory");
}

// Warp-wide, all lanes: for the lanes whose cell is a PML cell (pml) with
// compact index idx, bring rows [k0, k1) of every split block those cells
// lie in into L2 (one bulk prefetch per block, from lanes 0, 1, ...).
// Returns whether any lane's cell is a PML cell.
template <class T>
__device__ __forceinline__ bool prefetch_split_rows(const T *split, bool pml, uint32_t idx, int k0, int k1,
                                                    int lane) {
    const uint32_t lo = __reduce_min_sync(0xffffffffu, pml ? idx : 0xffffffffu);
    if (lo == 0xffffffffu) return false;
    const uint32_t hi = __reduce_max_sync(0xffffffffu, pml ? idx : 0u);
    const uint32_t b0 = lo / kSplitBlock;
    if ((uint32_t)lane <= hi / kSplitBlock - b0)
        l2_prefetch(split + (size_t)(b0 + lane) * (kNumSplit * kSplitBlock) + k0 * kSplitBlock,
                    (uint32_t)((k1 - k0) * kSplitBlock * sizeof(T)));
    return true;
}

// Wait (bounded) for the stages still in flight before an early exit:
// planes [from, issued_end) of a ring of S stages started at plane zs.
template <int S>
__device__ void drain(uint64_t *bar, int issued_end, int from, int zs) {
    for (int j = from; j < issued_end; ++j) mbar_wait(&bar[(j - zs) % S], (uint32_t)(((j - zs) / S) & 1));
}

// The same for a ring whose barriers carry their phase parities in pbits
// (bit s: the parity the next wait on stage s expects); planes [from,
// issued_end) are pending, at most one per stage.
template <int S>
__device__ void drain_bits(uint64_t *bar, int issued_end, int from, int zs, uint32_t pbits) {
    for (int j = from; j < issued_end; ++j) {
        const int s = (j - zs) % S;
        mbar_wait(&bar[s], (pbits >> s) & 1u);
    }
}

constexpr uint32_t kGridWaitCap = 1u << 20;   // polls of about 1 us: a grid barrier gives up after ~1 s

__device__ __forceinline__ unsigned ld_acquire(const unsigned *p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// All CTAs of a cooperative launch meet here: arrivals are counted in
// *arrive, and the barrier completes when `target` arrivals have been
// counted.  Bounded: false (and *status = fail_code) when the count does not
// arrive.  The fences make the other CTAs' stores of the finished phase
// visible to this CTA's later loads, TMA (async proxy) included.
__device__ __forceinline__ bool grid_sync(unsigned *arrive, unsigned target, int *status, int fail_code,
                                          int *ok_sh) {
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        atomicAdd(arrive, 1u);
        bool ok = true;
        for (uint32_t n = 0; ld_acquire(arrive) < target; ++n) {
            if (n >= kGridWaitCap) { ok = false; break; }
            __nanosleep(1000);
        }
        __threadfence();
        asm volatile("fence.proxy.async.global;" ::: "memory");
        if (!ok) atomicExch(status, fail_code);
        *ok_sh = ok;
    }
    __syncthreads();
    return *ok_sh != 0;
}

// 128-byte aligned start inside the dynamic shared array.  The offset is
// computed on the shared-window address so the result stays a pointer into
// __shared__ memory (the compiler then emits shared loads for every box read).
__device__ __forceinline__ unsigned char *align_smem(unsigned char *p) {
    return p + ((128u - (sptr(p) & 127u)) & 127u);
}

}  // namespace zdev
}  // namespace sgfd
