// kernels_audit.cu — FP64 energy audit of the wavefield: kinetic and strain
// energy summed over the computed cells of a region (all computed cells, the
// interior, or the PML shell).
//
// Not part of the reference's time loop; it is the measurement behind the
// absorbing-boundary checks (energy left in the interior once the direct wave
// has left measures what the boundary reflected).  Per cell, with the nine
// fields and the medium taken at the same array index:
//   kinetic = 1/2 * rho * |v|^2,  rho = 1/b
//   strain  = (s:s - lambda / (3 lambda + 2 mu) * tr(s)^2) / (4 mu)
//             (s:s = sxx^2 + syy^2 + szz^2 + 2 (sxy^2 + sxz^2 + syz^2));
//             for mu = 0, tr(s)^2 / (18 lambda)
// both times the cell volume dx*dy*dz.  Sums run in FP64: one partial per
// block, then one block adds the partials in a fixed order, so the result is
// deterministic for a given launch shape.  The per-step form
// (launch_energy_step) runs after the stress update of every step and
// records steps 0, every, 2*every, ... into a history buffer.
#include "../../include/sgfd.h"
#include "sgfd_internal.h"

namespace sgfd {

namespace {

constexpr int kAuditThreads = 256;

__device__ __forceinline__ double warp_sum(double v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Block-wide sum of (a, b); the result is valid in thread 0.
__device__ __forceinline__ void block_sum2(double &a, double &b) {
    __shared__ double sa[kAuditThreads / 32], sb[kAuditThreads / 32];
    a = warp_sum(a);
    b = warp_sum(b);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) { sa[w] = a; sb[w] = b; }
    __syncthreads();
    if (w == 0) {
        a = l < kAuditThreads / 32 ? sa[l] : 0.0;
        b = l < kAuditThreads / 32 ? sb[l] : 0.0;
        a = warp_sum(a);
        b = warp_sum(b);
    }
}

// Step index of a gated (per-step) audit launch, or -1 when this step is not
// sampled.
__device__ __forceinline__ int audit_sample(const AuditGate &gt) {
    const int it = gt.it_dev ? gt.it_arg + *gt.it_dev : gt.it_arg;
    if (it < 0 || it % gt.every != 0 || it / gt.every >= gt.count) return -1;
    return it / gt.every;
}

// One warp per (y, z) row of computed cells, lanes across x.  GATED: a
// per-step audit launch that returns at once on steps it does not sample.
template <bool GATED>
__global__ void __launch_bounds__(kAuditThreads) k_energy_partial(Model m, int region, double *partials,
                                                                 AuditGate gt) {
    if (GATED && audit_sample(gt) < 0) return;
    double ek = 0.0, es = 0.0;
    const int lane = threadIdx.x & 31;
    const int warps = gridDim.x * (kAuditThreads / 32);
    const int rows = m.nyc * m.nzc;
    for (int r = blockIdx.x * (kAuditThreads / 32) + (threadIdx.x >> 5); r < rows; r += warps) {
        const int cz = r / m.nyc, cy = r - cz * m.nyc;
        const int y = cy + kHalo, z = cz + kHalo;
        const bool yz_pml = band(y, m.ny, m.pml) != 0 || bandz(m, z) != 0;
        for (int cx = lane; cx < m.nxc; cx += 32) {
            const int x = cx + kHalo;
            const bool in_pml = yz_pml || band(x, m.nx, m.pml) != 0;
            if ((region == SGFD_REGION_INTERIOR && in_pml) || (region == SGFD_REGION_PML && !in_pml)) continue;
            const int64_t c = pidx(m, x, y, z);
            const double vx = m.f[0][c], vy = m.f[1][c], vz = m.f[2][c];
            const double sxx = m.f[3][c], syy = m.f[4][c], szz = m.f[5][c];
            const double sxy = m.f[6][c], sxz = m.f[7][c], syz = m.f[8][c];
            const double b = m.b[c], lam = m.lam[c], mu = m.mu[c];
            if (b > 0.0) ek += 0.5 * (vx * vx + vy * vy + vz * vz) / b;
            const double tr = sxx + syy + szz;
            const double ss = sxx * sxx + syy * syy + szz * szz + 2.0 * (sxy * sxy + sxz * sxz + syz * syz);
            if (mu > 0.0) es += (ss - lam / (3.0 * lam + 2.0 * mu) * tr * tr) / (4.0 * mu);
            else if (lam > 0.0) es += tr * tr / (18.0 * lam);
        }
    }
    block_sum2(ek, es);
    if (threadIdx.x == 0) {
        partials[2 * blockIdx.x] = ek;
        partials[2 * blockIdx.x + 1] = es;
    }
}

template <bool GATED>
__global__ void __launch_bounds__(kAuditThreads) k_energy_final(const double *partials, int nblocks, double volume,
                                                               double *out, AuditGate gt) {
    int sample = 0;
    if (GATED) {
        sample = audit_sample(gt);
        if (sample < 0) return;
        out = gt.hist + 2 * (size_t)sample;
    }
    double ek = 0.0, es = 0.0;
    for (int i = threadIdx.x; i < nblocks; i += kAuditThreads) {
        ek += partials[2 * i];
        es += partials[2 * i + 1];
    }
    block_sum2(ek, es);
    if (threadIdx.x == 0) {
        out[0] = ek * volume;
        out[1] = es * volume;
    }
}

}  // namespace

int energy_blocks(int num_sms) { return 8 * num_sms; }

cudaError_t launch_energy(const Model &m, const Physics &ph, int region, double *partials, int nblocks,
                          double *out, cudaStream_t s) {
    const AuditGate none{};
    k_energy_partial<false><<<nblocks, kAuditThreads, 0, s>>>(m, region, partials, none);
    const double volume = (double)ph.dx * (double)ph.dy * (double)ph.dz;
    k_energy_final<false><<<1, kAuditThreads, 0, s>>>(partials, nblocks, volume, out, none);
    return cudaGetLastError();
}

cudaError_t launch_energy_step(const Model &m, const Physics &ph, int region, double *partials, int nblocks,
                               const AuditGate &gt, cudaStream_t s) {
    k_energy_partial<true><<<nblocks, kAuditThreads, 0, s>>>(m, region, partials, gt);
    const double volume = (double)ph.dx * (double)ph.dy * (double)ph.dz;
    k_energy_final<true><<<1, kAuditThreads, 0, s>>>(partials, nblocks, volume, nullptr, gt);
    return cudaGetLastError();
}

}  // namespace sgfd
