// kernels_half.cu — 16-bit wavefield storage (sgfd_config.storage BF16 or
// F16) for the per-cell kernel family.
//
// Every wavefield and its PML splits are stored as 16-bit values h with a
// per-field power-of-two scale 2^e: a value v is stored as RN16(v * 2^-e)
// (binary16 saturating at +-65504) and read back as float(h) * 2^e, both
// scalings exact.  All arithmetic is the FP32 arithmetic of cell_math.cuh on
// the read-back values, so the update of one cell is the FP32 update of
// kernels_simple.cu followed by the rounding of what it stores.  The reference
// has no such mode; it halves the wavefield bytes.
//
// Scales are re-chosen after step it when it + 1 is a power of two up to
// kRescaleEvery and then every kRescaleEvery steps: the updates (and the
// source injection) of such a step note, per field, the largest magnitude
// they wrote before rounding; afterwards each field's exponent is set so that
// this maximum lands in [2^(kScaleHead-1), 2^kScaleHead) and every stored
// value is re-rounded to it.  The CPU oracle emulates the same steps.
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include "../../include/sgfd.h"
#include "cell_math.cuh"

namespace sgfd {

namespace {

constexpr int kBX = 32, kBY = 8;

template <int ST>
__device__ __forceinline__ float h2f(uint16_t h) {
    if (ST == SGFD_STORE_BF16) return __uint_as_float((uint32_t)h << 16);
    return __half2float(__ushort_as_half(h));
}
template <int ST>
__device__ __forceinline__ uint16_t f2h(float w) {
    if (ST == SGFD_STORE_BF16) return __bfloat16_as_ushort(__float2bfloat16_rn(w));
    return __half_as_ushort(__float2half_rn(fminf(fmaxf(w, -65504.0f), 65504.0f)));
}

__device__ __forceinline__ bool rescale_step(int it) {
    const int n = it + 1;
    if (n <= 0) return false;
    return (n <= kRescaleEvery && (n & (n - 1)) == 0) || n % kRescaleEvery == 0;
}

// Scale group of each split (the field it sums into).
__device__ __forceinline__ int split_group(int k) {
    return k < kNumVelSplit ? k / 3 : (k < S_XYX ? 3 + (k - S_XXX) / 3 : 6 + (k - S_XYX) / 2);
}

// Largest |v| of the warp's active lanes into the field's running maximum
// (non-negative floats order like their bit patterns); the lowest active lane
// does the atomic, since lanes of one warp may sit on different branches.
__device__ __forceinline__ void note_max(const HalfState &hs, int g, float v) {
    const unsigned mask = __activemask();
    const unsigned bits = __reduce_max_sync(mask, __float_as_uint(fabsf(v)));
    const int lane = (threadIdx.x + threadIdx.y * blockDim.x) & 31;
    if (lane == __ffs(mask) - 1) atomicMax(hs.amax + g, bits);
}

template <int ST>
struct Store16 {
    const HalfState &hs;
    __device__ float get(int g, int64_t i) const { return h2f<ST>(hs.f[g][i]) * hs.sc[g]; }
    __device__ float tap(int g, const uint16_t *p, int64_t o) const { return h2f<ST>(__ldg(p + o)) * hs.sc[g]; }
    __device__ void put(int g, int64_t i, float v) const { hs.f[g][i] = f2h<ST>(v * hs.inv[g]); }
    __device__ float sget(int k, int64_t i) const { return h2f<ST>(hs.split[i]) * hs.sc[split_group(k)]; }
    __device__ void sput(int k, int64_t i, float v) const { hs.split[i] = f2h<ST>(v * hs.inv[split_group(k)]); }
};

// txx, tyy, tzz at the source += dt*dt*s(it), stored rounded.
template <int ST>
__global__ void k_inject16(Model m, Physics ph, SourceRec sr, HalfState hs, int it_arg, float value, int use_wavelet) {
    if (threadIdx.x != 0 || sr.src < 0) return;
    const int it = step_index(sr, it_arg);
    const float v = ph.inj_dt2 * (use_wavelet ? sr.wavelet[it] : value);
    const bool track = rescale_step(it);
    const Store16<ST> S{hs};
    for (int g = 3; g <= 5; ++g) {
        const float w = S.get(g, sr.src) + v;
        if (track) atomicMax(hs.amax + g, __float_as_uint(fabsf(w)));
        S.put(g, sr.src, w);
    }
}

// Velocity update of one cell: kernels_simple.cu's k_velocity on read-back values.
template <bool FAST, int ST>
__global__ void __launch_bounds__(kBX * kBY) k_velocity16(Model m, Physics ph, SourceRec sr, HalfState hs, int it_arg) {
    const int cx = blockIdx.x * kBX + threadIdx.x;
    const int cy = blockIdx.y * kBY + threadIdx.y;
    const int cz = blockIdx.z;
    const bool track = rescale_step(step_index(sr, it_arg));
    if (cx >= m.nxc || cy >= m.nyc) return;
    const Store16<ST> S{hs};
    const int x = cx + kHalo, y = cy + kHalo, z = cz + kHalo;
    const int64_t ci = pidx(m, x, y, z);
    const int64_t SY = m.px, SZ = m.plane;
    const uint16_t *sxx = hs.f[3] + ci, *syy = hs.f[4] + ci, *szz = hs.f[5] + ci;
    const uint16_t *sxy = hs.f[6] + ci, *sxz = hs.f[7] + ci, *syz = hs.f[8] + ci;
    const float *bb = m.b + ci;

    const float bx = (bb[0] + bb[1]) / 2.0f;
    const float by = (bb[0] + bb[SY]) / 2.0f;
    const float bz = (bb[0] + bb[SZ]) / 2.0f;
    const float xX = dF<FAST, 0>(ph, [&](int o) { return S.tap(3, sxx, o); });
    const float xY = dB<FAST, 1>(ph, [&](int o) { return S.tap(6, sxy, o * SY); });
    const float xZ = dB<FAST, 2>(ph, [&](int o) { return S.tap(7, sxz, o * SZ); });
    const float yX = dB<FAST, 0>(ph, [&](int o) { return S.tap(6, sxy, o); });
    const float yY = dF<FAST, 1>(ph, [&](int o) { return S.tap(4, syy, o * SY); });
    const float yZ = dB<FAST, 2>(ph, [&](int o) { return S.tap(8, syz, o * SZ); });
    const float zX = dB<FAST, 0>(ph, [&](int o) { return S.tap(7, sxz, o); });
    const float zY = dB<FAST, 1>(ph, [&](int o) { return S.tap(8, syz, o * SY); });
    const float zZ = dF<FAST, 2>(ph, [&](int o) { return S.tap(5, szz, o * SZ); });

    const int kx = band(x, m.nx, m.pml), ky = band(y, m.ny, m.pml), kz = bandz(m, z);
    float vn[3];
    if (!(kx | ky | kz)) {
        vn[0] = __fmaf_rn(ph.dt * bx, (xX + xY) + xZ, S.get(0, ci));
        vn[1] = __fmaf_rn(ph.dt * by, (yX + yY) + yZ, S.get(1, ci));
        vn[2] = __fmaf_rn(ph.dt * bz, (zX + zY) + zZ, S.get(2, ci));
        if (track)
            for (int g = 0; g < 3; ++g) note_max(hs, g, vn[g]);
    } else {
        float mx = 1.f, my = 1.f, mz = 1.f;
        PDiv<FAST> px = 1, py = 1, pz = 1;
        {
            const float v = damp_speed(ph, m.mu[ci], bb[0], m.lam[ci]);
            if (kx) damp_factors<FAST>(ph, 0, ph.dx, kx, m.pml, v, mx, px);
            if (ky) damp_factors<FAST>(ph, 1, ph.dy, ky, m.pml, v, my, py);
            if (kz) damp_factors<FAST>(ph, 2, ph.dz, kz, m.pml, v, mz, pz);
        }
        const bool ref = ph.quirks == 0;
        const float a[3] = {ph.dt * bx, ph.dt * (ref ? bx : by), ph.dt * (ref ? bx : bz)};
        const float d[3][3] = {{xX, xY, xZ}, {yX, yY, yZ}, {zX, zY, zZ}};
        const int kk[3] = {kx, ky, kz};
        const float mm[3] = {mx, my, mz};
        const PDiv<FAST> pp[3] = {px, py, pz};
        const int64_t pi = split_base(pml_index(m, cx, cy, cz)), N = kSplitBlock;
        for (int q = 0; q < 3; ++q) {
            float part[3];
            for (int ax = 0; ax < 3; ++ax) {
                const int k = 3 * q + ax;
                part[ax] = split_update<FAST>(S.sget(k, k * N + pi), a[q], d[q][ax], kk[ax], mm[ax], pp[ax]);
                if (track) note_max(hs, q, part[ax]);
                S.sput(k, k * N + pi, part[ax]);
            }
            vn[q] = (part[0] + part[1]) + part[2];
        }
        if (track)
            for (int g = 0; g < 3; ++g) note_max(hs, g, vn[g]);
    }
    for (int g = 0; g < 3; ++g) S.put(g, ci, vn[g]);
}

// Stress update of one cell: kernels_simple.cu's k_stress on read-back values.
template <bool FAST, int ST>
__global__ void __launch_bounds__(kBX * kBY) k_stress16(Model m, Physics ph, SourceRec sr, HalfState hs, int it_arg) {
    const int cx = blockIdx.x * kBX + threadIdx.x;
    const int cy = blockIdx.y * kBY + threadIdx.y;
    const int cz = blockIdx.z;
    const bool track = rescale_step(step_index(sr, it_arg));
    if (cx >= m.nxc || cy >= m.nyc) return;
    const Store16<ST> S{hs};
    const int x = cx + kHalo, y = cy + kHalo, z = cz + kHalo;
    const int64_t ci = pidx(m, x, y, z);
    const int64_t SY = m.px, SZ = m.plane;
    const uint16_t *vx = hs.f[0] + ci, *vy = hs.f[1] + ci, *vz = hs.f[2] + ci;

    const float dXx = dB<FAST, 0>(ph, [&](int o) { return S.tap(0, vx, o); });
    const float dYy = dB<FAST, 1>(ph, [&](int o) { return S.tap(1, vy, o * SY); });
    const float dZz = dB<FAST, 2>(ph, [&](int o) { return S.tap(2, vz, o * SZ); });
    const float xyY = dF<FAST, 1>(ph, [&](int o) { return S.tap(0, vx, o * SY); });
    const float xyX = dF<FAST, 0>(ph, [&](int o) { return S.tap(1, vy, o); });
    const float xzZ = dF<FAST, 2>(ph, [&](int o) { return S.tap(0, vx, o * SZ); });
    const float xzX = dF<FAST, 0>(ph, [&](int o) { return S.tap(2, vz, o); });
    const float yzZ = dF<FAST, 2>(ph, [&](int o) { return S.tap(1, vy, o * SZ); });
    const float yzY = dF<FAST, 1>(ph, [&](int o) { return S.tap(2, vz, o * SY); });

    const float l = m.lam[ci];
    const float l2m = __fmaf_rn(2.0f, m.mu[ci], l);
    const float mxy = m.mxy[ci], mxz = m.mxz[ci], myz = m.myz[ci];

    const int kx = band(x, m.nx, m.pml), ky = band(y, m.ny, m.pml), kz = bandz(m, z);
    float sn[6];
    if (!(kx | ky | kz)) {
        sn[0] = __fmaf_rn(ph.dt, __fmaf_rn(l2m, dXx, l * (dYy + dZz)), S.get(3, ci));
        sn[1] = __fmaf_rn(ph.dt, __fmaf_rn(l2m, dYy, l * (dXx + dZz)), S.get(4, ci));
        sn[2] = __fmaf_rn(ph.dt, __fmaf_rn(l2m, dZz, l * (dXx + dYy)), S.get(5, ci));
        sn[3] = __fmaf_rn(ph.dt * mxy, xyY + xyX, S.get(6, ci));
        sn[4] = __fmaf_rn(ph.dt * mxz, xzZ + xzX, S.get(7, ci));
        sn[5] = __fmaf_rn(ph.dt * myz, yzZ + yzY, S.get(8, ci));
    } else {
        float mx = 1.f, my = 1.f, mz = 1.f;
        PDiv<FAST> px = 1, py = 1, pz = 1;
        {
            const float v = damp_speed(ph, m.mu[ci], m.b[ci], l);
            if (kx) damp_factors<FAST>(ph, 0, ph.dx, kx, m.pml, v, mx, px);
            if (ky) damp_factors<FAST>(ph, 1, ph.dy, ky, m.pml, v, my, py);
            if (kz) damp_factors<FAST>(ph, 2, ph.dz, kz, m.pml, v, mz, pz);
        }
        const int64_t pi = split_base(pml_index(m, cx, cy, cz)), N = kSplitBlock;
        const float dl = ph.dt * l2m, dt = ph.dt;
        auto upd = [&](int k, float A, float B, int kd, float mf, PDiv<FAST> pf) {
            const float r = split_update<FAST>(S.sget(k, k * N + pi), A, B, kd, mf, pf);
            if (track) note_max(hs, split_group(k), r);
            S.sput(k, k * N + pi, r);
            return r;
        };
        float a0, a1, a2;
        a0 = upd(S_XXX, dl, dXx, kx, mx, px);
        a1 = upd(S_XXY, dt, l * dYy, ky, my, py);
        a2 = upd(S_XXZ, dt, l * dZz, kz, mz, pz);
        sn[0] = (a0 + a1) + a2;
        a0 = upd(S_YYX, dt, l * dXx, kx, mx, px);
        a1 = upd(S_YYY, dl, dYy, ky, my, py);
        a2 = upd(S_YYZ, dt, l * dZz, kz, mz, pz);
        sn[1] = (a0 + a1) + a2;
        a0 = upd(S_ZZX, dt, l * dXx, kx, mx, px);
        a1 = upd(S_ZZY, dt, l * dYy, ky, my, py);
        a2 = upd(S_ZZZ, dl, dZz, kz, mz, pz);
        sn[2] = (a0 + a1) + a2;
        const float axy = dt * mxy, axz = dt * mxz, ayz = dt * myz;
        a0 = upd(S_XYX, axy, xyX, kx, mx, px);
        a1 = upd(S_XYY, axy, xyY, ky, my, py);
        sn[3] = a0 + a1;
        a0 = upd(S_XZX, axz, xzX, kx, mx, px);
        a1 = upd(S_XZZ, axz, xzZ, kz, mz, pz);
        sn[4] = a0 + a1;
        a0 = upd(S_YZY, ayz, yzY, ky, my, py);
        a1 = upd(S_YZZ, ayz, yzZ, kz, mz, pz);
        sn[5] = a0 + a1;
    }
    if (track)
        for (int q = 0; q < 6; ++q) note_max(hs, 3 + q, sn[q]);
    for (int q = 0; q < 6; ++q) S.put(3 + q, ci, sn[q]);
}

// Receivers of one phase sample their (read-back) component.
template <int ST>
__global__ void k_record16(Model m, SourceRec sr, HalfState hs, int it_arg, int velocity_phase) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    const int it = step_index(sr, it_arg);
    if (r >= sr.nrec || it < 0 || it >= sr.nt) return;
    const int4 q = sr.rec[r];
    if ((q.w <= 2) != (velocity_phase != 0)) return;
    sr.traces[(int64_t)it * sr.nrec + r] = Store16<ST>{hs}.get(q.w, pidx(m, q.x, q.y, q.z));
}

// New exponents from the noted maxima (one thread); fields that noted zero
// (or a non-finite value) keep theirs.
__global__ void k_rescale_choose(SourceRec sr, HalfState hs, int it_arg) {
    if (threadIdx.x != 0 || !rescale_step(step_index(sr, it_arg))) return;
    for (int g = 0; g < 9; ++g) {
        const float mx = __uint_as_float(hs.amax[g]);
        int e = hs.e[g];
        if (mx > 0.0f && isfinite(mx)) e = min(100, max(-100, ilogbf(mx) + 1 - kScaleHead));
        hs.e_new[g] = e;
    }
}

// Re-round every stored value of a field whose exponent changes.
template <int ST>
__global__ void k_rescale_apply(Model m, SourceRec sr, HalfState hs, int it_arg, int64_t n_grid) {
    if (!rescale_step(step_index(sr, it_arg))) return;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x, t0 = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    // every stored value h of p[0, n) becomes RN16(float(h) * f): eight at a
    // time through 16-byte accesses, the unaligned head and the tail one by one
    auto rescale = [&](uint16_t *p, int64_t n, float f) {
        const int64_t head = ((16 - (int64_t)(reinterpret_cast<uintptr_t>(p) & 15)) & 15) / 2;
        const int64_t h = head < n ? head : n;
        const int64_t n8 = (n - h) / 8;
        for (int64_t i = t0; i < h; i += stride) p[i] = f2h<ST>(h2f<ST>(p[i]) * f);
        uint4 *q = reinterpret_cast<uint4 *>(p + h);
        for (int64_t i = t0; i < n8; i += stride) {
            uint4 v = q[i];
            uint32_t w[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const uint32_t lo = f2h<ST>(h2f<ST>(w[j] & 0xffffu) * f);
                const uint32_t hi = f2h<ST>(h2f<ST>(w[j] >> 16) * f);
                w[j] = lo | (hi << 16);
            }
            q[i] = make_uint4(w[0], w[1], w[2], w[3]);
        }
        for (int64_t i = h + 8 * n8 + t0; i < n; i += stride) p[i] = f2h<ST>(h2f<ST>(p[i]) * f);
    };
    for (int g = 0; g < 9; ++g) {
        if (hs.e_new[g] == hs.e[g]) continue;
        rescale(hs.f[g] - kXOff, n_grid, ldexpf(1.0f, hs.e[g] - hs.e_new[g]));   // the whole padded array
    }
    // the blocked splits: eight values of one split per 16-byte access
    {
        const int64_t n8 = split_elems(m.npml) / 8;
        uint4 *q = reinterpret_cast<uint4 *>(hs.split);
        for (int64_t i = t0; i < n8; i += stride) {
            const int g = split_group(split_of(8 * i));
            if (hs.e_new[g] == hs.e[g]) continue;
            const float f = ldexpf(1.0f, hs.e[g] - hs.e_new[g]);
            uint4 v = q[i];
            uint32_t w[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const uint32_t lo = f2h<ST>(h2f<ST>(w[j] & 0xffffu) * f);
                const uint32_t hi = f2h<ST>(h2f<ST>(w[j] >> 16) * f);
                w[j] = lo | (hi << 16);
            }
            q[i] = make_uint4(w[0], w[1], w[2], w[3]);
        }
    }
}

// Adopt the new exponents and clear the maxima for the next rescale step.
__global__ void k_rescale_commit(SourceRec sr, HalfState hs, int it_arg) {
    if (threadIdx.x >= 9 || !rescale_step(step_index(sr, it_arg))) return;
    const int g = threadIdx.x;
    hs.e[g] = hs.e_new[g];
    hs.sc[g] = ldexpf(1.0f, hs.e[g]);
    hs.inv[g] = ldexpf(1.0f, -hs.e[g]);
    hs.amax[g] = 0u;
}

// FP32 copies of the stored fields and splits (the arrays the read-out paths use).
template <int ST>
__global__ void k_to_views(Model m, HalfState hs, int64_t n_grid) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x, t0 = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    for (int g = 0; g < 9; ++g) {
        const uint16_t *p = hs.f[g] - kXOff;
        float *q = m.f[g] - kXOff;
        const float sc = hs.sc[g];
        for (int64_t i = t0; i < n_grid; i += stride) q[i] = h2f<ST>(p[i]) * sc;
    }
    const int64_t ns = split_elems(m.npml);
    for (int64_t j = t0; j < ns; j += stride) m.split[j] = h2f<ST>(hs.split[j]) * hs.sc[split_group(split_of(j))];
}

// Stored values from the FP32 copies (after a checkpoint load).
template <int ST>
__global__ void k_from_views(Model m, HalfState hs, int64_t n_grid) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x, t0 = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    for (int g = 0; g < 9; ++g) {
        uint16_t *p = hs.f[g] - kXOff;
        const float *q = m.f[g] - kXOff;
        const float inv = hs.inv[g];
        for (int64_t i = t0; i < n_grid; i += stride) p[i] = f2h<ST>(q[i] * inv);
    }
    const int64_t ns = split_elems(m.npml);
    for (int64_t j = t0; j < ns; j += stride) hs.split[j] = f2h<ST>(m.split[j] * hs.inv[split_group(split_of(j))]);
}

template <int ST>
cudaError_t step16(const Model &m, const Physics &ph, const SourceRec &sr, const HalfState &hs, int it,
                   float src_value, bool use_wavelet, cudaStream_t s, cudaEvent_t *ev) {
    if (sr.src >= 0) k_inject16<ST><<<1, 32, 0, s>>>(m, ph, sr, hs, it, src_value, use_wavelet ? 1 : 0);
    const dim3 block(kBX, kBY);
    const dim3 grid((m.nxc + kBX - 1) / kBX, (m.nyc + kBY - 1) / kBY, m.nzc);
    if (ev) cudaEventRecord(ev[0], s);
    if (ph.fast) k_velocity16<true, ST><<<grid, block, 0, s>>>(m, ph, sr, hs, it);
    else k_velocity16<false, ST><<<grid, block, 0, s>>>(m, ph, sr, hs, it);
    if (ev) cudaEventRecord(ev[1], s);
    if (sr.nrec > 0) k_record16<ST><<<(sr.nrec + 127) / 128, 128, 0, s>>>(m, sr, hs, it, 1);
    if (ev) cudaEventRecord(ev[2], s);
    if (ph.fast) k_stress16<true, ST><<<grid, block, 0, s>>>(m, ph, sr, hs, it);
    else k_stress16<false, ST><<<grid, block, 0, s>>>(m, ph, sr, hs, it);
    if (ev) cudaEventRecord(ev[3], s);
    if (sr.nrec > 0) k_record16<ST><<<(sr.nrec + 127) / 128, 128, 0, s>>>(m, sr, hs, it, 0);
    k_rescale_choose<<<1, 32, 0, s>>>(sr, hs, it);
    k_rescale_apply<ST><<<1184, 256, 0, s>>>(m, sr, hs, it, m.plane * m.nz);
    k_rescale_commit<<<1, 32, 0, s>>>(sr, hs, it);
    return cudaGetLastError();
}

template <int ST>
cudaError_t phases16(const Model &m, const Physics &ph, const SourceRec &sr, const HalfState &hs, int it,
                     float src_value, bool use_wavelet, cudaStream_t s, int phase) {
    if (phase == 0) {
        if (sr.src >= 0) k_inject16<ST><<<1, 32, 0, s>>>(m, ph, sr, hs, it, src_value, use_wavelet ? 1 : 0);
    } else if (phase == 1) {
        if (sr.nrec > 0) k_record16<ST><<<(sr.nrec + 127) / 128, 128, 0, s>>>(m, sr, hs, it, 1);
    } else {
        if (sr.nrec > 0) k_record16<ST><<<(sr.nrec + 127) / 128, 128, 0, s>>>(m, sr, hs, it, 0);
        k_rescale_choose<<<1, 32, 0, s>>>(sr, hs, it);
        k_rescale_apply<ST><<<1184, 256, 0, s>>>(m, sr, hs, it, m.plane * m.nz);
        k_rescale_commit<<<1, 32, 0, s>>>(sr, hs, it);
    }
    return cudaGetLastError();
}

}  // namespace

cudaError_t half_phase(const Model &m, const Physics &ph, const SourceRec &sr, const HalfState &hs, int it,
                       float src_value, bool use_wavelet, cudaStream_t s, int phase) {
    return hs.storage == SGFD_STORE_BF16 ? phases16<SGFD_STORE_BF16>(m, ph, sr, hs, it, src_value, use_wavelet, s, phase)
                                         : phases16<SGFD_STORE_F16>(m, ph, sr, hs, it, src_value, use_wavelet, s, phase);
}

cudaError_t half_step(const Model &m, const Physics &ph, const SourceRec &sr, const HalfState &hs, int it,
                      float src_value, bool use_wavelet, cudaStream_t s, cudaEvent_t *ev) {
    return hs.storage == SGFD_STORE_BF16 ? step16<SGFD_STORE_BF16>(m, ph, sr, hs, it, src_value, use_wavelet, s, ev)
                                         : step16<SGFD_STORE_F16>(m, ph, sr, hs, it, src_value, use_wavelet, s, ev);
}

int half_launches_per_step(const SourceRec &sr) {
    return 2 + (sr.src >= 0 ? 1 : 0) + (sr.nrec > 0 ? 2 : 0) + 3;
}

cudaError_t half_to_views(const Model &m, const HalfState &hs, cudaStream_t s) {
    const int64_t n = m.plane * m.nz;
    if (hs.storage == SGFD_STORE_BF16) k_to_views<SGFD_STORE_BF16><<<1184, 256, 0, s>>>(m, hs, n);
    else k_to_views<SGFD_STORE_F16><<<1184, 256, 0, s>>>(m, hs, n);
    return cudaGetLastError();
}

cudaError_t half_from_views(const Model &m, const HalfState &hs, cudaStream_t s) {
    const int64_t n = m.plane * m.nz;
    if (hs.storage == SGFD_STORE_BF16) k_from_views<SGFD_STORE_BF16><<<1184, 256, 0, s>>>(m, hs, n);
    else k_from_views<SGFD_STORE_F16><<<1184, 256, 0, s>>>(m, hs, n);
    return cudaGetLastError();
}

}  // namespace sgfd
