// kernels_simple.cu — the "simple" kernel family: one thread per computed
// cell, neighbours read straight from global memory (L1/L2 cached).
//
// It is the plain restatement of the reference's per-cell kernels
// (3DGPUwithPML_1DArraySingleGPU_optimization/ElasticWaveEquation.cu:206-841)
// with the 26-way region `else if` chain replaced by a per-axis band test and
// the 26 region split arrays replaced by the compact PML array.  It serves as
// the correctness baseline for the z-marching family and as the fallback for
// grids the z-marching kernels do not tile.
#include "cell_math.cuh"

namespace sgfd {

namespace {

constexpr int kBX = 32, kBY = 8;

// txx, tyy, tzz at the source cell += dt*dt*s(it)   (ElasticWaveEquation.cu:206-221)
__global__ void k_inject(Model m, Physics ph, SourceRec sr, int it_arg, float value, int use_wavelet) {
    if (threadIdx.x != 0 || sr.src < 0) return;
    const int it = step_index(sr, it_arg);
    const float s = use_wavelet ? sr.wavelet[it] : value;
    const float v = ph.inj_dt2 * s;
    m.f[3][sr.src] = m.f[3][sr.src] + v;
    m.f[4][sr.src] = m.f[4][sr.src] + v;
    m.f[5][sr.src] = m.f[5][sr.src] + v;
}

// Velocity update of one cell (ElasticWaveEquation.cu:234-526, ElasticMacro.h:409-458).
template <bool FAST>
__global__ void __launch_bounds__(kBX * kBY) k_velocity(Model m, Physics ph, int z0) {
    const int cx = blockIdx.x * kBX + threadIdx.x;
    const int cy = blockIdx.y * kBY + threadIdx.y;
    const int cz = blockIdx.z + z0;   // computed planes [z0, z0 + gridDim.z)
    if (cx >= m.nxc || cy >= m.nyc) return;
    const int x = cx + kHalo, y = cy + kHalo, z = cz + kHalo;
    const int64_t ci = pidx(m, x, y, z);
    const int64_t SY = m.px, SZ = m.plane;
    const float *sxx = m.f[3] + ci, *syy = m.f[4] + ci, *szz = m.f[5] + ci;
    const float *sxy = m.f[6] + ci, *sxz = m.f[7] + ci, *syz = m.f[8] + ci;
    const float *bb = m.b + ci;

    const float bx = (bb[0] + bb[1]) / 2.0f;
    const float by = (bb[0] + bb[SY]) / 2.0f;
    const float bz = (bb[0] + bb[SZ]) / 2.0f;
    const float xX = dF<FAST, 0>(ph, [&](int o) { return __ldg(sxx + o); });
    const float xY = dB<FAST, 1>(ph, [&](int o) { return __ldg(sxy + o * SY); });
    const float xZ = dB<FAST, 2>(ph, [&](int o) { return __ldg(sxz + o * SZ); });
    const float yX = dB<FAST, 0>(ph, [&](int o) { return __ldg(sxy + o); });
    const float yY = dF<FAST, 1>(ph, [&](int o) { return __ldg(syy + o * SY); });
    const float yZ = dB<FAST, 2>(ph, [&](int o) { return __ldg(syz + o * SZ); });
    const float zX = dB<FAST, 0>(ph, [&](int o) { return __ldg(sxz + o); });
    const float zY = dB<FAST, 1>(ph, [&](int o) { return __ldg(syz + o * SY); });
    const float zZ = dF<FAST, 2>(ph, [&](int o) { return __ldg(szz + o * SZ); });

    const int kx = band(x, m.nx, m.pml), ky = band(y, m.ny, m.pml), kz = bandz(m, z);
    if (!(kx | ky | kz)) {
        m.f[0][ci] = __fmaf_rn(ph.dt * bx, (xX + xY) + xZ, m.f[0][ci]);
        m.f[1][ci] = __fmaf_rn(ph.dt * by, (yX + yY) + yZ, m.f[1][ci]);
        m.f[2][ci] = __fmaf_rn(ph.dt * bz, (zX + zY) + zZ, m.f[2][ci]);
        return;
    }
    float mx = 1.f, my = 1.f, mz = 1.f;
        PDiv<FAST> px = 1, py = 1, pz = 1;
    {
        const float v = damp_speed(ph, m.mu[ci], bb[0], m.lam[ci]);
        if (kx) damp_factors<FAST>(ph, 0, ph.dx, kx, m.pml, v, mx, px);
        if (ky) damp_factors<FAST>(ph, 1, ph.dy, ky, m.pml, v, my, py);
        if (kz) damp_factors<FAST>(ph, 2, ph.dz, kz, m.pml, v, mz, pz);
    }
    const bool ref = ph.quirks == 0;   // REF: x-averaged buoyancy for all components
    const float ax = ph.dt * bx, ay = ph.dt * (ref ? bx : by), az = ph.dt * (ref ? bx : bz);
    const int64_t pi = pml_index(m, cx, cy, cz);
    float *sp = m.split + split_base(pi);
    const int64_t N = kSplitBlock;   // split k at sp[k * N]
    float a0, a1, a2;
    a0 = sp[S_VXX * N] = split_update<FAST>(sp[S_VXX * N], ax, xX, kx, mx, px);
    a1 = sp[S_VXY * N] = split_update<FAST>(sp[S_VXY * N], ax, xY, ky, my, py);
    a2 = sp[S_VXZ * N] = split_update<FAST>(sp[S_VXZ * N], ax, xZ, kz, mz, pz);
    m.f[0][ci] = (a0 + a1) + a2;
    a0 = sp[S_VYX * N] = split_update<FAST>(sp[S_VYX * N], ay, yX, kx, mx, px);
    a1 = sp[S_VYY * N] = split_update<FAST>(sp[S_VYY * N], ay, yY, ky, my, py);
    a2 = sp[S_VYZ * N] = split_update<FAST>(sp[S_VYZ * N], ay, yZ, kz, mz, pz);
    m.f[1][ci] = (a0 + a1) + a2;
    a0 = sp[S_VZX * N] = split_update<FAST>(sp[S_VZX * N], az, zX, kx, mx, px);
    a1 = sp[S_VZY * N] = split_update<FAST>(sp[S_VZY * N], az, zY, ky, my, py);
    a2 = sp[S_VZZ * N] = split_update<FAST>(sp[S_VZZ * N], az, zZ, kz, mz, pz);
    m.f[2][ci] = (a0 + a1) + a2;
}

// Stress update of one cell (ElasticWaveEquation.cu:528-841, ElasticMacro.h:460-531).
template <bool FAST>
__global__ void __launch_bounds__(kBX * kBY) k_stress(Model m, Physics ph, int z0) {
    const int cx = blockIdx.x * kBX + threadIdx.x;
    const int cy = blockIdx.y * kBY + threadIdx.y;
    const int cz = blockIdx.z + z0;   // computed planes [z0, z0 + gridDim.z)
    if (cx >= m.nxc || cy >= m.nyc) return;
    const int x = cx + kHalo, y = cy + kHalo, z = cz + kHalo;
    const int64_t ci = pidx(m, x, y, z);
    const int64_t SY = m.px, SZ = m.plane;
    const float *vx = m.f[0] + ci, *vy = m.f[1] + ci, *vz = m.f[2] + ci;
    const float *r = m.rmu + ci;

    const float dXx = dB<FAST, 0>(ph, [&](int o) { return __ldg(vx + o); });
    const float dYy = dB<FAST, 1>(ph, [&](int o) { return __ldg(vy + o * SY); });
    const float dZz = dB<FAST, 2>(ph, [&](int o) { return __ldg(vz + o * SZ); });
    const float xyY = dF<FAST, 1>(ph, [&](int o) { return __ldg(vx + o * SY); });
    const float xyX = dF<FAST, 0>(ph, [&](int o) { return __ldg(vy + o); });
    const float xzZ = dF<FAST, 2>(ph, [&](int o) { return __ldg(vx + o * SZ); });
    const float xzX = dF<FAST, 0>(ph, [&](int o) { return __ldg(vz + o); });
    const float yzZ = dF<FAST, 2>(ph, [&](int o) { return __ldg(vy + o * SZ); });
    const float yzY = dF<FAST, 1>(ph, [&](int o) { return __ldg(vz + o * SY); });

    const float l = m.lam[ci];
    const float mu0 = m.mu[ci];
    const float l2m = __fmaf_rn(2.0f, mu0, l);
    const bool ref = ph.quirks == 0;   // REF: fourth txz point is mu[x+1, y+1, z]
    const float mxy = hmean<FAST>(r[0], r[1], r[SY], r[1 + SY]);
    const float mxz = hmean<FAST>(r[0], r[1], r[SZ], ref ? r[1 + SY] : r[1 + SZ]);
    const float myz = hmean<FAST>(r[0], r[SY], r[SZ], r[SY + SZ]);

    const int kx = band(x, m.nx, m.pml), ky = band(y, m.ny, m.pml), kz = bandz(m, z);
    if (!(kx | ky | kz)) {
        m.f[3][ci] = __fmaf_rn(ph.dt, __fmaf_rn(l2m, dXx, l * (dYy + dZz)), m.f[3][ci]);
        m.f[4][ci] = __fmaf_rn(ph.dt, __fmaf_rn(l2m, dYy, l * (dXx + dZz)), m.f[4][ci]);
        m.f[5][ci] = __fmaf_rn(ph.dt, __fmaf_rn(l2m, dZz, l * (dXx + dYy)), m.f[5][ci]);
        m.f[6][ci] = __fmaf_rn(ph.dt * mxy, xyY + xyX, m.f[6][ci]);
        m.f[7][ci] = __fmaf_rn(ph.dt * mxz, xzZ + xzX, m.f[7][ci]);
        m.f[8][ci] = __fmaf_rn(ph.dt * myz, yzZ + yzY, m.f[8][ci]);
        return;
    }
    float mx = 1.f, my = 1.f, mz = 1.f;
        PDiv<FAST> px = 1, py = 1, pz = 1;
    {
        const float v = damp_speed(ph, mu0, m.b[ci], l);
        if (kx) damp_factors<FAST>(ph, 0, ph.dx, kx, m.pml, v, mx, px);
        if (ky) damp_factors<FAST>(ph, 1, ph.dy, ky, m.pml, v, my, py);
        if (kz) damp_factors<FAST>(ph, 2, ph.dz, kz, m.pml, v, mz, pz);
    }
    const int64_t pi = pml_index(m, cx, cy, cz);
    float *sp = m.split + split_base(pi);
    const int64_t N = kSplitBlock;   // split k at sp[k * N]
    const float dl = ph.dt * l2m, dt = ph.dt;
    float a0, a1, a2;
    a0 = sp[S_XXX * N] = split_update<FAST>(sp[S_XXX * N], dl, dXx, kx, mx, px);
    a1 = sp[S_XXY * N] = split_update<FAST>(sp[S_XXY * N], dt, l * dYy, ky, my, py);
    a2 = sp[S_XXZ * N] = split_update<FAST>(sp[S_XXZ * N], dt, l * dZz, kz, mz, pz);
    m.f[3][ci] = (a0 + a1) + a2;
    a0 = sp[S_YYX * N] = split_update<FAST>(sp[S_YYX * N], dt, l * dXx, kx, mx, px);
    a1 = sp[S_YYY * N] = split_update<FAST>(sp[S_YYY * N], dl, dYy, ky, my, py);
    a2 = sp[S_YYZ * N] = split_update<FAST>(sp[S_YYZ * N], dt, l * dZz, kz, mz, pz);
    m.f[4][ci] = (a0 + a1) + a2;
    a0 = sp[S_ZZX * N] = split_update<FAST>(sp[S_ZZX * N], dt, l * dXx, kx, mx, px);
    a1 = sp[S_ZZY * N] = split_update<FAST>(sp[S_ZZY * N], dt, l * dYy, ky, my, py);
    a2 = sp[S_ZZZ * N] = split_update<FAST>(sp[S_ZZZ * N], dl, dZz, kz, mz, pz);
    m.f[5][ci] = (a0 + a1) + a2;
    const float axy = dt * mxy, axz = dt * mxz, ayz = dt * myz;
    a0 = sp[S_XYX * N] = split_update<FAST>(sp[S_XYX * N], axy, xyX, kx, mx, px);
    a1 = sp[S_XYY * N] = split_update<FAST>(sp[S_XYY * N], axy, xyY, ky, my, py);
    m.f[6][ci] = a0 + a1;
    a0 = sp[S_XZX * N] = split_update<FAST>(sp[S_XZX * N], axz, xzX, kx, mx, px);
    a1 = sp[S_XZZ * N] = split_update<FAST>(sp[S_XZZ * N], axz, xzZ, kz, mz, pz);
    m.f[7][ci] = a0 + a1;
    a0 = sp[S_YZY * N] = split_update<FAST>(sp[S_YZY * N], ayz, yzY, ky, my, py);
    a1 = sp[S_YZZ * N] = split_update<FAST>(sp[S_YZZ * N], ayz, yzZ, kz, mz, pz);
    m.f[8][ci] = a0 + a1;
}

// Receivers of one phase sample their component (ElasticWaveEquation.cu:223-232).
__global__ void k_record(Model m, SourceRec sr, int it_arg, int velocity_phase) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    const int it = step_index(sr, it_arg);
    if (r >= sr.nrec || it < 0 || it >= sr.nt) return;
    const int4 q = sr.rec[r];
    if ((q.w <= 2) != (velocity_phase != 0)) return;
    sr.traces[(int64_t)it * sr.nrec + r] = m.f[q.w][pidx(m, q.x, q.y, q.z)];
}

// Staggered shear moduli of one computed cell from the reciprocals rmu = 1/mu,
// in the operand order of the stress update (ElasticMacro.h:110-119):
// mxy over (x,y), (x+1,y), (x,y+1), (x+1,y+1) at z; myz over (x,y), (x,y+1)
// at z and z+1; mxz over (x,y,z), (x+1,y,z), (x,y,z+1) and, with the
// reference's index quirk, (x+1,y+1,z) instead of (x+1,y,z+1).
template <bool FAST>
__global__ void k_shear_means(Model m, int quirks, float *mxy, float *mxz, float *myz) {
    const int cx = blockIdx.x * kBX + threadIdx.x;
    const int cy = blockIdx.y * kBY + threadIdx.y;
    const int cz = blockIdx.z;
    if (cx >= m.nxc || cy >= m.nyc) return;
    const int64_t c = pidx(m, cx + kHalo, cy + kHalo, cz + kHalo);
    const int64_t X = 1, Y = m.px, Z = m.plane;
    const float *r = m.rmu;
    mxy[c] = hmean<FAST>(r[c], r[c + X], r[c + Y], r[c + X + Y]);
    mxz[c] = hmean<FAST>(r[c], r[c + X], r[c + Z], quirks == 0 ? r[c + X + Y] : r[c + X + Z]);
    myz[c] = hmean<FAST>(r[c], r[c + Y], r[c + Z], r[c + Y + Z]);
}

// Device step counter of a replayed CUDA graph: set before the first replay,
// advanced by the last node of each replay.
__global__ void k_counter(int *ctr, int value, int add) {
    if (threadIdx.x == 0) *ctr = add ? *ctr + value : value;
}

__global__ void k_reciprocal(float *rmu, const float *mu, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        rmu[i] = __frcp_rn(mu[i]);   // 1 / mu, IEEE round-to-nearest (ElasticMacro.h:112)
}

// Packed rows (nx floats each, as a host array is laid out) into the padded
// device layout (row pitch px): one block per row at a time.
__global__ void k_pitch_rows(float *dst, int64_t px, const float *src, int nx, int64_t nrows) {
    for (int64_t r = blockIdx.x; r < nrows; r += gridDim.x)
        for (int x = threadIdx.x; x < nx; x += blockDim.x) dst[r * px + x] = src[r * (int64_t)nx + x];
}

}  // namespace

int simple_launches_per_step(const SourceRec &sr) {
    int n = 2;
    if (sr.src >= 0) n += 1;
    if (sr.nrec > 0) n += 2;
    return n;
}

cudaError_t simple_step(const Model &m, const Physics &ph, const SourceRec &sr,
                        int it, float src_value, bool use_wavelet, cudaStream_t s, cudaEvent_t *ev, int phases,
                        int parts) {
    const dim3 block(kBX, kBY);
    // plane ranges of the selected parts: inner [5, nzc - 5), outer the planes below and above it
    int range[3][2];
    const int nr = part_ranges(m.nzc, 1, m.nzc, parts, range);
    auto each = [&](auto fn) {
        for (int r = 0; r < nr; ++r)
            if (range[r][1] > range[r][0])
                fn(dim3((m.nxc + kBX - 1) / kBX, (m.nyc + kBY - 1) / kBY, range[r][1] - range[r][0]), range[r][0]);
    };
    if (phases & 1) {
        if ((parts & kPartInner) && sr.src >= 0) k_inject<<<1, 32, 0, s>>>(m, ph, sr, it, src_value, use_wavelet ? 1 : 0);
        if (ev) cudaEventRecord(ev[0], s);
        each([&](dim3 grid, int z0) {
            if (ph.fast) k_velocity<true><<<grid, block, 0, s>>>(m, ph, z0);
            else k_velocity<false><<<grid, block, 0, s>>>(m, ph, z0);
        });
        if (ev) cudaEventRecord(ev[1], s);
        if ((parts & kPartOuter) && sr.nrec > 0) k_record<<<(sr.nrec + 127) / 128, 128, 0, s>>>(m, sr, it, 1);
    }
    if (phases & 2) {
        if (ev) cudaEventRecord(ev[2], s);
        each([&](dim3 grid, int z0) {
            if (ph.fast) k_stress<true><<<grid, block, 0, s>>>(m, ph, z0);
            else k_stress<false><<<grid, block, 0, s>>>(m, ph, z0);
        });
        if (ev) cudaEventRecord(ev[3], s);
        if ((parts & kPartOuter) && sr.nrec > 0) k_record<<<(sr.nrec + 127) / 128, 128, 0, s>>>(m, sr, it, 0);
    }
    return cudaGetLastError();
}

cudaError_t launch_shear_means(const Model &m, const Physics &ph, float *mxy, float *mxz, float *myz,
                               cudaStream_t s) {
    const dim3 block(kBX, kBY);
    const dim3 grid((m.nxc + kBX - 1) / kBX, (m.nyc + kBY - 1) / kBY, m.nzc);
    if (ph.fast) k_shear_means<true><<<grid, block, 0, s>>>(m, ph.quirks, mxy, mxz, myz);
    else k_shear_means<false><<<grid, block, 0, s>>>(m, ph.quirks, mxy, mxz, myz);
    return cudaGetLastError();
}

cudaError_t launch_counter(int *ctr, int value, bool add, cudaStream_t s) {
    k_counter<<<1, 32, 0, s>>>(ctr, value, add ? 1 : 0);
    return cudaGetLastError();
}

cudaError_t launch_pitch_rows(float *dst, int64_t px, const float *src, int nx, int64_t nrows, cudaStream_t s) {
    k_pitch_rows<<<1184, 128, 0, s>>>(dst, px, src, nx, nrows);
    return cudaGetLastError();
}

cudaError_t launch_reciprocal(float *rmu, const float *mu, int64_t n, cudaStream_t s) {
    k_reciprocal<<<1184, 256, 0, s>>>(rmu, mu, n);
    return cudaGetLastError();
}

}  // namespace sgfd
