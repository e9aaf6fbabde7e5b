// sgfd_internal.h — device data layout and launch parameters shared by the
// host API (sgfd_api.cu) and the kernel families (kernels_*.cu).
//
// HBM layout of one model
//   * 9 wavefields + buoyancy, lambda, mu: one array each, x fastest, the
//     reference GRID (5-cell frame included), rows padded to a pitch `px`
//     that is a multiple of 32 floats so every row starts on a 128-byte
//     boundary (coalescing, and the 16-byte rule of TMA tensor maps).  Each
//     row is shifted right by kXOff floats inside its pitch so that the
//     computed cells of every 32-wide tile start on a 128-byte boundary.
//     Model::f[k] etc. point at GRID (0,0,0); the allocation starts kXOff
//     floats earlier.  index(ix, iy, iz) = ix + iy*px + iz*px*ny.
//   * PML split fields: a compact array of the PML cells only.  PML cells
//     are enumerated plane by plane (z slowest), and within a plane row by
//     row, x fastest (pml_index()); blocks of 32 consecutive cells hold their
//     24 splits as 24 rows of 32 values, split k of cell c at
//     split[split_base(c) + 32*k] (split_base()).  A warp reading consecutive
//     x reads one 128-byte row per split, and a cell's 24 splits sit at fixed
//     offsets from one address.  The reference keeps 26 region arrays of
//     (len+1)^3 each (OPT/ElasticWaveEquation.cu:34-41).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace sgfd {

constexpr int kHalo = 5;            // reference `order` (OPT/ElasticMacro.h:24)
// Device arrays store GRID x at offset kXOff so that the first computed cell
// (x = 5) sits at a 32-float (128-byte) boundary: 5 + 27 = 32.
constexpr int kXOff = 27;
constexpr int kNumSplit = 24;
constexpr int kNumVelSplit = 9;     // velocity splits come first
constexpr float kTau = 4.3f;        // reference `tau` (OPT/ElasticMacro.h:21)
constexpr int kPwTable = 129;       // damping-profile table covers pml <= 128

// Split ids (velocity q,axis then stress), same order as the oracle.
enum SplitId {
    S_VXX, S_VXY, S_VXZ, S_VYX, S_VYY, S_VYZ, S_VZX, S_VZY, S_VZZ,
    S_XXX, S_XXY, S_XXZ, S_YYX, S_YYY, S_YYZ, S_ZZX, S_ZZY, S_ZZZ,
    S_XYX, S_XYY, S_XZX, S_XZZ, S_YZY, S_YZZ
};

// Per-step physics constants (all FP32, computed once on the host).
struct Physics {
    float c[5];          // staggered coefficients
    float cs[3][5];      // c_i / dx, c_i / dy, c_i / dz (FAST arithmetic)
    float2 cp[4][5];     // FAST pairs for FP32x2: (cs_x, cs_x), (cs_y, cs_y), (cs_z, cs_z), (cs_x, cs_y)
    int fast;            // sgfd_arith == FAST
    float dt, dx, dy, dz;
    float inj_dt2;       // dt*dt (source scale, OPT/ElasticWaveEquation.cu:213)
    int damping;         // sgfd_damping
    int quirks;          // sgfd_quirks
    float q_refgpu;      // (0.5*dt)*tau
    float poly;          // 8/15 - 0.03 p + p^2/1500
    float q_logr;        // 0.5*dt*3*ln(1/R)/(2p)
    float q_refcpu[3];   // 0.5*dt*log10(1/R)*3.4*V/(p*d)
    float qf[3];         // FAST: ((0.5*dt*tau)/d)*poly (REFGPU) or (0.5*dt*3*ln(1/R)/(2p))/d (LOGR)
    float pw[kPwTable];  // (k/pml)^2 for k = 0..kPwTable-1 (rounded as (k/p)*(k/p))
    // REF arithmetic: the reference's divisions by the cell sizes, correctly
    // rounded without a division instruction (cell_math.cuh, div_cell)
    float2 cr[5];        // (c_i, c_i): REF sums of two differences on FP32x2
    float rd[3];         // RN(1/dx), RN(1/dy), RN(1/dz)
    int mdiv;            // bit a: the single-precision correction step is exact for axis a
    double rd64[3];      // RN64(1/dx), RN64(1/dy), RN64(1/dz)
};

// Geometry and device pointers of one model.
struct Model {
    int nx, ny, nz;      // GRID (frame included)
    int px;              // row pitch in floats
    int pml;
    int nxc, nyc, nzc;   // computed extents (n - 10)
    int64_t plane;       // px * ny
    int64_t npml;        // number of PML cells
    float *f[9];         // vx vy vz txx tyy tzz txy txz tyz
    const float *b, *lam, *mu, *rmu;   // rmu = 1/mu
    // staggered shear moduli of the txy, txz, tyz updates: harmonic means of
    // four mu (ElasticMacro.h:110-119), computed once per medium upload
    const float *mxy, *mxz, *myz;
    float *split;        // split_elems(npml) values, blocked (split_base)
    // z-slab of a larger model (sgfd_config.nz_total != 0): the whole model's
    // computed planes below this slab, the whole model's computed z extent,
    // and the whole model's compact index of the slab's first PML cell.  The
    // PML bands and the compact PML order are the whole model's.  A model on
    // its own: 0, nzc, 0.
    int zoff, nzcg;
    int64_t pbase;
};

// 16-bit wavefield storage (kernels_half.cu): fields and splits as 16-bit
// values with per-field power-of-two scales; scale state in device memory so
// that replayed graphs see its updates.
constexpr int kRescaleEvery = 50;   // scales re-chosen every 50 steps (after steps 0, 1, 3, 7, ... first)
constexpr int kScaleHead = 8;       // largest stored magnitude put in [2^7, 2^8)
struct HalfState {
    uint16_t *f[9];      // same layout (pitch, offset) as Model::f
    uint16_t *split;     // split_elems(npml) values, blocked as Model::split
    int *e, *e_new;      // scale exponents (9 each)
    float *sc, *inv;     // 2^e, 2^-e
    unsigned *amax;      // largest |value| written on a rescale step (float bits)
    int storage;         // SGFD_STORE_BF16 or SGFD_STORE_F16
};

// Source (one explosive point) and receivers.
struct SourceRec {
    int64_t src;         // padded index of the source cell, -1 if none
    const float *wavelet;// device wavelet (sgfd_run) or nullptr
    int nrec;
    const int4 *rec;     // x, y, z, comp
    float *traces;       // time-major: traces[it * nrec + r]
    int nt;
    const int *it_dev;   // graph replay: step index = *it_dev + the launch's offset; nullptr otherwise
};

#ifdef __CUDACC__
// Step index a kernel works on: the launch argument, plus the device step
// counter when the launch belongs to a replayed CUDA graph.
__device__ __forceinline__ int step_index(const SourceRec &sr, int it_arg) {
    return sr.it_dev ? it_arg + *sr.it_dev : it_arg;
}
// 16-bit storage: the steps after which the scales are re-chosen (it + 1 a
// power of two up to kRescaleEvery, then every kRescaleEvery steps); their
// updates note each field's largest written magnitude.
__device__ __forceinline__ bool rescale_step16(int it) {
    const int n = it + 1;
    if (n <= 0) return false;
    return (n <= kRescaleEvery && (n & (n - 1)) == 0) || n % kRescaleEvery == 0;
}
#endif

__host__ __device__ inline int64_t pidx(const Model &m, int x, int y, int z) {
    return (int64_t)x + (int64_t)y * m.px + (int64_t)z * m.plane;
}

// Band distance along one axis: 0 outside the PML band, else 1..pml counted
// from the inner edge (OPT/ElasticWaveEquation.cu:283-285 `end - i`,
// :297 `i - start + 1`).
__host__ __device__ inline int band(int i, int n, int pml) {
    if (i < kHalo + pml) return kHalo + pml - i;
    if (i >= n - kHalo - pml) return i - (n - kHalo - pml) + 1;
    return 0;
}

// Band distance along z of GRID plane gz, counted in the whole model's planes
// (a z-slab's PML is the whole model's).
__host__ __device__ inline int bandz(const Model &m, int gz) {
    return band(gz + m.zoff, m.nzcg + 2 * kHalo, m.pml);
}

// Compact index of a PML cell given computed coordinates (cx, cy, cz), in
// the model's own split array (a z-slab's part of the whole model's order).
__host__ __device__ inline int64_t pml_index(const Model &m, int cx, int cy, int cz) {
    const int p = m.pml;
    const int64_t full = (int64_t)m.nxc * m.nyc;
    const int64_t ring = (int64_t)2 * p * m.nxc + (int64_t)(m.nyc - 2 * p) * 2 * p;
    const int z = cz + m.zoff;
    int64_t base;
    bool full_plane;
    if (z < p) { base = z * full; full_plane = true; }
    else if (z < m.nzcg - p) { base = p * full + (int64_t)(z - p) * ring; full_plane = false; }
    else { base = p * full + (int64_t)(m.nzcg - 2 * p) * ring + (int64_t)(z - (m.nzcg - p)) * full; full_plane = true; }
    base -= m.pbase;
    if (full_plane) return base + (int64_t)cy * m.nxc + cx;
    if (cy < p) return base + (int64_t)cy * m.nxc + cx;
    if (cy < m.nyc - p) {
        const int off = cx < p ? cx : cx - (m.nxc - 2 * p);
        return base + (int64_t)p * m.nxc + (int64_t)(cy - p) * 2 * p + off;
    }
    return base + (int64_t)p * m.nxc + (int64_t)(m.nyc - 2 * p) * 2 * p + (int64_t)(cy - (m.nyc - p)) * m.nxc + cx;
}

// Split storage: blocks of kSplitBlock PML cells (consecutive compact
// indices), each block kNumSplit rows of kSplitBlock values; split k of PML
// cell c at split_base(c) + k * kSplitBlock.
constexpr int kSplitBlock = 32;
__host__ __device__ inline int64_t split_base(int64_t c) {
    return (c / kSplitBlock) * (int64_t)(kNumSplit * kSplitBlock) + c % kSplitBlock;
}
__host__ __device__ inline uint32_t split_base32(uint32_t c) {
    return (c / kSplitBlock) * (uint32_t)(kNumSplit * kSplitBlock) + c % kSplitBlock;
}
// Values the split array holds (the last block padded), and the split of value j.
__host__ __device__ inline int64_t split_elems(int64_t npml) {
    return (npml + kSplitBlock - 1) / kSplitBlock * (int64_t)(kNumSplit * kSplitBlock);
}
__host__ __device__ inline int split_of(int64_t j) { return (int)((j / kSplitBlock) % kNumSplit); }

// pml_index() split in two for kernels that march along z: a per-column
// offset (in full PML planes and in ring planes) and a per-plane base.  32-bit
// arithmetic: the z-marching family requires npml < 2^31.
struct PmlColumn {
    uint32_t full_off;   // offset inside a full PML plane
    uint32_t ring_off;   // offset inside a ring plane (valid for x/y-band columns)
};
__host__ __device__ inline PmlColumn pml_column(const Model &m, int cx, int cy) {
    const int p = m.pml;
    PmlColumn c;
    c.full_off = (uint32_t)(cy * m.nxc + cx);
    if (cy < p) c.ring_off = (uint32_t)(cy * m.nxc + cx);
    else if (cy < m.nyc - p)
        c.ring_off = (uint32_t)(p * m.nxc + (cy - p) * 2 * p + (cx < p ? cx : cx - (m.nxc - 2 * p)));
    else c.ring_off = (uint32_t)(p * m.nxc + (m.nyc - 2 * p) * 2 * p + (cy - (m.nyc - p)) * m.nxc + cx);
    return c;
}
// Index of the PML cell of column c in computed plane cz.  Modulo 2^32: a
// z-slab's whole-model index may wrap, its difference with pbase (the
// slab's own index, below 2^32) does not.
__host__ __device__ inline uint32_t pml_plane_index(const Model &m, const PmlColumn &c, int cz) {
    const uint32_t p = (uint32_t)m.pml;
    const uint32_t full = (uint32_t)m.nxc * (uint32_t)m.nyc;
    const uint32_t ring = 2u * p * (uint32_t)m.nxc + (uint32_t)(m.nyc - 2 * m.pml) * 2u * p;
    const int zi = cz + m.zoff;
    const uint32_t z = (uint32_t)zi, pb = (uint32_t)m.pbase;
    if (zi < m.pml) return z * full + c.full_off - pb;
    if (zi < m.nzcg - m.pml) return p * full + (z - p) * ring + c.ring_off - pb;
    return p * full + (uint32_t)(m.nzcg - 2 * m.pml) * ring + (z - (uint32_t)(m.nzcg - m.pml)) * full + c.full_off -
           pb;
}

__host__ inline int64_t pml_count(int nxc, int nyc, int nzc, int p) {
    const int64_t full = (int64_t)nxc * nyc;
    const int64_t ring = (int64_t)2 * p * nxc + (int64_t)(nyc - 2 * p) * 2 * p;
    return 2 * p * full + (int64_t)(nzc - 2 * p) * ring;
}
// PML cells in computed planes [0, z) of a model of nzc computed planes
// (where a z-slab starting at plane z starts in the compact order).
__host__ inline int64_t pml_before(int nxc, int nyc, int nzc, int p, int z) {
    const int64_t full = (int64_t)nxc * nyc;
    const int64_t ring = (int64_t)2 * p * nxc + (int64_t)(nyc - 2 * p) * 2 * p;
    const int lo = z < p ? z : p;
    const int mid = z - p < 0 ? 0 : (z - p < nzc - 2 * p ? z - p : nzc - 2 * p);
    const int hi = z - (nzc - p) < 0 ? 0 : z - (nzc - p);
    return (int64_t)(lo + hi) * full + (int64_t)mid * ring;
}

// Parts of a half step, so that a z-slab can overlap its halo exchange with
// its own work: kPartInner the planes whose updates read no frame plane
// (5 or more computed planes from both ends of the model's planes),
// kPartOuter the others.  Run inner before outer (the simple family injects
// the source with the inner part and records receivers with the outer one).
constexpr int kPartInner = 1, kPartOuter = 2;

// The units a part covers, for a model of nzc computed planes cut into n
// units of `size` planes (z chunks; planes: size 1): up to three ranges
// [r[i][0], r[i][1]), possibly empty, in z order; returns their count.  A
// unit is inner when its planes lie 5 or more planes from both ends; the
// whole half step (both parts) is one range.
__host__ __device__ inline int part_ranges(int nzc, int size, int n, int parts, int (*r)[2]) {
    if (parts == (kPartInner | kPartOuter)) {
        r[0][0] = 0; r[0][1] = n;
        return 1;
    }
    const int a = (kHalo + size - 1) / size, i0 = a < n ? a : n;   // first inner unit
    const int b = nzc >= kHalo ? (nzc - kHalo) / size : 0, i1 = b > i0 ? b : i0;   // end of the inner units
    int k = 0;
    if (parts & kPartOuter) { r[k][0] = 0; r[k][1] = i0; ++k; }
    if (parts & kPartInner) { r[k][0] = i0; r[k][1] = i1; ++k; }
    if (parts & kPartOuter) { r[k][0] = i1; r[k][1] = n; ++k; }
    return k;
}

// ---- kernel family entry points (host side) -------------------------------

// "simple": one thread per computed cell.
// ev (optional, 4 events): recorded before/after the velocity kernel and
// before/after the stress kernel.  phases: bit 0 the source injection, the
// velocity update and its receivers, bit 1 the stress update and its
// receivers; parts: kPartInner / kPartOuter planes (both: all).
cudaError_t simple_step(const Model &m, const Physics &ph, const SourceRec &sr,
                        int it, float src_value, bool use_wavelet, cudaStream_t s,
                        cudaEvent_t *ev = nullptr, int phases = 3, int parts = 3);
int simple_launches_per_step(const SourceRec &sr);

// medium post-processing: rmu = 1/mu over the padded arrays, then the three
// staggered shear moduli of every computed cell from rmu.
cudaError_t launch_reciprocal(float *rmu, const float *mu, int64_t n, cudaStream_t s);
// dst[r * px + x] = src[r * nx + x] for nrows rows of nx floats.
cudaError_t launch_pitch_rows(float *dst, int64_t px, const float *src, int nx, int64_t nrows, cudaStream_t s);
cudaError_t launch_shear_means(const Model &m, const Physics &ph, float *mxy, float *mxz, float *myz,
                               cudaStream_t s);
// FP64 energy audit (kernels_audit.cu): partials holds 2 doubles per block,
// out 2 doubles (kinetic, strain).
int energy_blocks(int num_sms);
cudaError_t launch_energy(const Model &m, const Physics &ph, int region, double *partials, int nblocks,
                          double *out, cudaStream_t s);
// Per-step audit: step it = it_arg (+ *it_dev under graph replay) is sampled
// when it % every == 0 and it / every < count; sample k goes to hist[2k..2k+1].
struct AuditGate {
    const int *it_dev;
    int it_arg;
    int every;
    int count;
    double *hist;
};
cudaError_t launch_energy_step(const Model &m, const Physics &ph, int region, double *partials, int nblocks,
                               const AuditGate &gt, cudaStream_t s);
// 16-bit storage: one step, launches per step, and the FP32 copies of the
// stored fields and splits (Model::f, Model::split) in both directions.
cudaError_t half_step(const Model &m, const Physics &ph, const SourceRec &sr, const HalfState &hs, int it,
                      float src_value, bool use_wavelet, cudaStream_t s, cudaEvent_t *ev = nullptr);
int half_launches_per_step(const SourceRec &sr);
// The 16-bit step's kernels around the two updates, for update kernels of
// another family: phase 0 the source injection (before the velocity update),
// 1 the velocity receivers, 2 the stress receivers and the rescale kernels.
cudaError_t half_phase(const Model &m, const Physics &ph, const SourceRec &sr, const HalfState &hs, int it,
                       float src_value, bool use_wavelet, cudaStream_t s, int phase);
cudaError_t half_to_views(const Model &m, const HalfState &hs, cudaStream_t s);
cudaError_t half_from_views(const Model &m, const HalfState &hs, cudaStream_t s);
// *ctr = value, or *ctr += value when add is set.
cudaError_t launch_counter(int *ctr, int value, bool add, cudaStream_t s);

}  // namespace sgfd
