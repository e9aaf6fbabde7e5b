// kernels_zpair.cu — the paired tiling of the z-marching family: each thread
// owns two x-adjacent cells, so that the y and z differences, the updates and
// the global stores of both run on packed FP32x2 (fma.rn.f32x2 and friends)
// and every shared-memory load of a y tap or an own-cell value brings both.
//
// Work decomposition.  A CTA of 256 threads owns a 64 x 8 tile of computed
// cells (warp w = tile row w, lane l = cells 2l and 2l+1 of that row) and
// marches along z over a chunk of planes, as the single-cell tiling of
// kernels_zmarch.cu does: per plane, TMA (cp.async.bulk.tensor.3d, no
// multicast) stages the xy boxes with the 5-cell halos each field is
// differentiated along (80 wide for x halos, 18 rows for y halos), the lead
// planes of the z register queues and the cells' own read-modify-write data
// into a ring of S stages guarded by one mbarrier each (expect-tx bytes,
// bounded parity waits); lane 0 of every warp issues a share of a stage's
// boxes; a stage is refilled with plane z + S as soon as plane z is done.
//
// Per thread and plane: x differences per cell from a 12-value window loaded
// as six 8-byte shared loads; y differences on FP32x2 from ten 8-byte column
// loads; z differences on FP32x2 from register queues of float2.  Each lane
// of a packed operation rounds exactly as the scalar operation, so results
// are bit-identical to kernels_zmarch.cu, kernels_simple.cu and the oracle.
// Tile-planes with PML cells, the source or receivers take the general path,
// which updates cell by cell; every other tile-plane updates the pair on
// FP32x2 and stores it with one 8-byte store per field.
#include <cuda.h>
#include <cudaTypedefs.h>

#include <type_traits>

#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include "../../include/sgfd.h"
#include "cell_math.cuh"
#include "store16.cuh"
#include "zmarch.h"
#include "zmarch_dev.cuh"

namespace sgfd {

namespace {

using namespace zdev;

constexpr int PX = kPairTileX;   // computed cells per tile row (two per thread)
constexpr int PY = 8;            // tile rows, one warp each
constexpr int NT = 256;
constexpr int XW = PX + 16;      // x-halo boxes start 8 cells left: TMA x stays a multiple of 4
constexpr int BW = PX + 4;       // buoyancy box: the tile and one cell to the right, width a multiple of 4
constexpr int SV = 3;            // velocity ring stages
constexpr int SS = 2;            // stress ring stages

constexpr int al128(int b) { return (b + 127) / 128 * 128; }
constexpr int OB = al128(PX * PY * 4);   // one 64 x 8 FP32 box (medium)

// Shared-memory stage of the velocity update (byte offsets, 128-aligned
// boxes); wavefield boxes hold ES-byte values (4: FP32, 2: 16-bit storage),
// the buoyancy boxes FP32.
template <int ES>
struct VelP {
    static constexpr int OBE = al128(PX * PY * ES);                // one 64 x 8 wavefield box
    static constexpr int SXX = 0;                                  // XW x PY        sigma_xx (x halo)
    static constexpr int SYY = SXX + al128(XW * PY * ES);          // PX x (PY+10)   sigma_yy (y halo)
    static constexpr int SXY = SYY + al128(PX * (PY + 10) * ES);   // XW x (PY+10)   sigma_xy (x, y halo)
    static constexpr int SXZ = SXY + al128(XW * (PY + 10) * ES);   // XW x PY        sigma_xz (x halo)
    static constexpr int SYZ = SXZ + al128(XW * PY * ES);          // PX x (PY+10)   sigma_yz (y halo)
    static constexpr int B = SYZ + al128(PX * (PY + 10) * ES);     // BW x (PY+1)    buoyancy (x+1, y+1)
    static constexpr int LXZ = B + al128(BW * (PY + 1) * 4);       // sigma_xz at z+4
    static constexpr int LYZ = LXZ + OBE;                          // sigma_yz at z+4
    static constexpr int LZZ = LYZ + OBE;                          // sigma_zz at z+5
    static constexpr int LB = LZZ + OBE;                           // buoyancy at z+1
    static constexpr int OV = LB + OB;                             // own vx, vy, vz at z
    static constexpr int STAGE = OV + 3 * OBE;
    static constexpr uint32_t TXB = ES * (2 * XW * PY + 2 * PX * (PY + 10) + XW * (PY + 10) + 6 * PX * PY) +
                                    4 * (BW * (PY + 1) + PX * PY);
};
// Shared-memory stage of the stress update.
template <int ES>
struct StrP {
    static constexpr int OBE = al128(PX * PY * ES);
    static constexpr int VX = 0;                                   // XW x (PY+10)  vx (x, y halo)
    static constexpr int VY = VX + al128(XW * (PY + 10) * ES);
    static constexpr int VZ = VY + al128(XW * (PY + 10) * ES);
    static constexpr int LX = VZ + al128(XW * (PY + 10) * ES);     // vx at z+5
    static constexpr int LY = LX + OBE;                            // vy at z+5
    static constexpr int LZ = LY + OBE;                            // vz at z+4
    static constexpr int OWN = LZ + OBE;                           // txx..tyz at z
    static constexpr int MED = OWN + 6 * OBE;                      // lambda, mu, mxy, mxz, myz at z
    static constexpr int STAGE = MED + 5 * OB;
    static constexpr uint32_t TXB = ES * (3 * XW * (PY + 10) + 9 * PX * PY) + 4 * 5 * PX * PY;
    // byte offset of own-cell box q (0..5 stresses, 6..10 medium)
    static constexpr uint32_t own(int q) { return q < 6 ? OWN + q * OBE : MED + (q - 6) * OB; }
};

struct PTile {
    int cx0, cy0;    // computed coordinates of the tile origin
    int xd;          // device x of the tile origin (128-byte aligned)
    int gx0, gy0;    // GRID coordinates of the tile origin
    int zs, ze;      // computed z range of this CTA
    bool xy_pml;     // the tile touches the x or y PML band
};

__device__ __forceinline__ PTile make_ptile(const Model &m, const ZGeom &g, int tile, int chunk) {
    PTile t;
    t.cx0 = (tile % g.ntx) * PX;
    t.cy0 = (tile / g.ntx) * PY;
    t.gx0 = t.cx0 + kHalo;
    t.gy0 = t.cy0 + kHalo;
    t.xd = t.gx0 + kXOff;
    t.zs = chunk * g.zc;
    t.ze = min(t.zs + g.zc, m.nzc);
    t.xy_pml = t.cx0 < m.pml || t.cx0 + PX > m.nxc - m.pml || t.cy0 < m.pml || t.cy0 + PY > m.nyc - m.pml;
    return t;
}

struct TmaBox {
    const CUtensorMap *map;
    uint32_t off;
    int x, y, dz;
};
constexpr int kWarps = NT / 32;
constexpr int kMaxBoxesPerWarp = 3;
constexpr int kVelBoxes = 13;
constexpr int kStrBoxes = 17;

template <int ES>
__device__ __forceinline__ TmaBox vel_box(const VelMaps &mp, const PTile &t, int q) {
    using L = VelP<ES>;
    switch (q) {
    case 0: return {&mp.sxx, L::SXX, t.xd - 8, t.gy0, 0};
    case 1: return {&mp.syy, L::SYY, t.xd, t.gy0 - 5, 0};
    case 2: return {&mp.sxy, L::SXY, t.xd - 8, t.gy0 - 5, 0};
    case 3: return {&mp.sxz, L::SXZ, t.xd - 8, t.gy0, 0};
    case 4: return {&mp.syz, L::SYZ, t.xd, t.gy0 - 5, 0};
    case 5: return {&mp.b, L::B, t.xd, t.gy0, 0};
    case 6: return {&mp.sxz_c, L::LXZ, t.xd, t.gy0, 4};
    case 7: return {&mp.syz_c, L::LYZ, t.xd, t.gy0, 4};
    case 8: return {&mp.szz_c, L::LZZ, t.xd, t.gy0, 5};
    case 9: return {&mp.b_c, L::LB, t.xd, t.gy0, 1};
    case 10: return {&mp.own[0], L::OV, t.xd, t.gy0, 0};
    case 11: return {&mp.own[1], L::OV + L::OBE, t.xd, t.gy0, 0};
    default: return {&mp.own[2], L::OV + 2 * L::OBE, t.xd, t.gy0, 0};
    }
}

template <int ES>
__device__ __forceinline__ TmaBox str_box(const StrMaps &mp, const PTile &t, int q) {
    using L = StrP<ES>;
    switch (q) {
    case 0: return {&mp.vx, L::VX, t.xd - 8, t.gy0 - 5, 0};
    case 1: return {&mp.vy, L::VY, t.xd - 8, t.gy0 - 5, 0};
    case 2: return {&mp.vz, L::VZ, t.xd - 8, t.gy0 - 5, 0};
    case 3: return {&mp.vx_c, L::LX, t.xd, t.gy0, 5};
    case 4: return {&mp.vy_c, L::LY, t.xd, t.gy0, 5};
    case 5: return {&mp.vz_c, L::LZ, t.xd, t.gy0, 4};
    default: return {&mp.own[q - 6], L::own(q - 6), t.xd, t.gy0, 0};
    }
}

// Stage the inputs of computed plane cz from this warp's boxes (lane 0 of
// every warp); warp 0 arms the stage's barrier with all of the stage's bytes.
__device__ __forceinline__ void issue(const TmaBox *b, int n, unsigned char *st, uint64_t *bar, int cz, int warp,
                                      uint32_t txb) {
    if (warp == 0) mbar_expect_tx(bar, txb);
    for (int j = 0; j < n; ++j) tma3(st + b[j].off, b[j].map, b[j].x, b[j].y, cz + kHalo + b[j].dz, bar);
}

__device__ __forceinline__ float2 ld2(const float *p) { return *reinterpret_cast<const float2 *>(p); }
__device__ __forceinline__ float2 bcast(float v) { return make_float2(v, v); }

// A pair's difference sums (FP32x2, lane = cell) divided by the cell size of
// `axis` (REF) or as they are (FAST).
template <bool FAST>
__device__ __forceinline__ float2 by_cell2(const Physics &ph, int axis, float2 s) {
    if (FAST) return s;
    return make_float2(div_cell(ph, axis, s.x), div_cell(ph, axis, s.y));
}
// Forward / backward staggered difference of a cell pair from taps g(o)
// (float2: both cells' values o cells, rows or planes away).
template <bool FAST, int AXIS, class G>
__device__ __forceinline__ float2 dF2p(const Physics &ph, G g) {
    const float2 s = dpair(FAST ? ph.cp[AXIS] : ph.cr, [&](int i) { return g(1 + i); }, [&](int i) { return g(-i); });
    return by_cell2<FAST>(ph, AXIS, s);
}
template <bool FAST, int AXIS, class G>
__device__ __forceinline__ float2 dB2p(const Physics &ph, G g) {
    const float2 s = dpair(FAST ? ph.cp[AXIS] : ph.cr, [&](int i) { return g(i); }, [&](int i) { return g(-1 - i); });
    return by_cell2<FAST>(ph, AXIS, s);
}
// x differences of both cells of a pair from one 12-value window w (w[0]
// at x offset `first` from cell 0): forward taps of cell c at offsets -4..5,
// backward at -5..4.
template <bool FAST>
__device__ __forceinline__ float2 dFx(const Physics &ph, const float (&w)[12], int first) {
    const float a = dF<FAST, 0>(ph, [&](int o) { return w[o - first]; });
    const float b = dF<FAST, 0>(ph, [&](int o) { return w[o + 1 - first]; });
    return make_float2(a, b);
}
template <bool FAST>
__device__ __forceinline__ float2 dBx(const Physics &ph, const float (&w)[12], int first) {
    const float a = dB<FAST, 0>(ph, [&](int o) { return w[o - first]; });
    const float b = dB<FAST, 0>(ph, [&](int o) { return w[o + 1 - first]; });
    return make_float2(a, b);
}
// Twelve values of one row starting at an even float index (six 8-byte loads).
__device__ __forceinline__ void window(const float *row, float (&w)[12]) {
#pragma unroll
    for (int k = 0; k < 6; ++k) {
        const float2 v = ld2(row + 2 * k);
        w[2 * k] = v.x;
        w[2 * k + 1] = v.y;
    }
}
__device__ __forceinline__ float lane_of(float2 v, int c) { return c ? v.y : v.x; }
// Element k of a six-value register array without indexing it at run time
// (which would move the array to local memory).
template <class T>
__device__ __forceinline__ T pick6(const T (&a)[6], int k) {
    return k == 0 ? a[0] : k == 1 ? a[1] : k == 2 ? a[2] : k == 3 ? a[3] : k == 4 ? a[4] : a[5];
}

__device__ __forceinline__ void st2(float *p, float2 v, bool both) {
    if (both) *reinterpret_cast<float2 *>(p) = v;
    else *p = v.x;
}

// Wavefield storage as the pair kernels see it.  FP32: the arrays as they
// are.  BF16 / F16 (the 16-bit storage of kernels_half.cu): value h of field
// g reads back as float(h) * 2^e_g and v is stored as RN16(v * 2^-e_g), F16
// saturating at +-65504; the same roundings as kernels_half.cu and the oracle.
template <int ST>
struct Sto {
    using E = float;
    static constexpr int ES = 4;
    __device__ __forceinline__ static float2 pair(const E *p, float2) { return ld2(p); }
    __device__ __forceinline__ static float one(const E *p, float) { return *p; }
    __device__ __forceinline__ static void win(const E *row, float (&w)[12], float) { window(row, w); }
    __device__ __forceinline__ static void put2(E *p, float2 v, float2, bool both) { st2(p, v, both); }
    __device__ __forceinline__ static void put1(E *p, float v, float) { *p = v; }
};
template <int ST>
struct Sto16 {
    using E = uint16_t;
    static constexpr int ES = 2;
    __device__ __forceinline__ static float h2f(uint32_t h) { return H16<ST>::h2f(h); }
    __device__ __forceinline__ static uint32_t f2h(float w) { return H16<ST>::f2h(w); }
    __device__ __forceinline__ static float2 pair(const E *p, float2 sc) {
        const uint32_t u = *reinterpret_cast<const uint32_t *>(p);
        return make_float2(h2f(u & 0xffffu) * sc.x, h2f(u >> 16) * sc.y);
    }
    __device__ __forceinline__ static float one(const E *p, float sc) { return h2f(*p) * sc; }
    __device__ __forceinline__ static void win(const E *row, float (&w)[12], float sc) {
#pragma unroll
        for (int k = 0; k < 6; ++k) {
            const float2 v = pair(row + 2 * k, make_float2(sc, sc));
            w[2 * k] = v.x;
            w[2 * k + 1] = v.y;
        }
    }
    __device__ __forceinline__ static void put2(E *p, float2 v, float2 inv, bool both) {
        const float2 q = __fmul2_rn(v, inv);
        if (both) *reinterpret_cast<uint32_t *>(p) = f2h(q.x) | (f2h(q.y) << 16);
        else *p = (E)f2h(q.x);
    }
    __device__ __forceinline__ static void put1(E *p, float v, float inv) { *p = (E)f2h(v * inv); }
};
template <> struct Sto<SGFD_STORE_BF16> : Sto16<SGFD_STORE_BF16> {};
template <> struct Sto<SGFD_STORE_F16> : Sto16<SGFD_STORE_F16> {};

// The wavefield arrays, split array and scales of either storage (read
// where used: the pointers live in the kernel parameters, the 16-bit scales
// in device memory, re-chosen between steps).
template <int ST>
struct Fields {
    using E = typename Sto<ST>::E;
    const Model &m;
    const HalfState &hs;
    const float *scl;   // 16-bit: the 9 scales 2^e then the 9 inverses, staged in shared memory
    __device__ __forceinline__ Fields(const Model &m_, const HalfState &hs_, const float *scl_)
        : m(m_), hs(hs_), scl(scl_) {}
    __device__ __forceinline__ E *f(int k) const {
        if constexpr (ST == SGFD_STORE_F32) return m.f[k];
        else return hs.f[k];
    }
    __device__ __forceinline__ E *split() const {
        if constexpr (ST == SGFD_STORE_F32) return m.split;
        else return hs.split;
    }
    __device__ __forceinline__ float sc(int k) const {
        if constexpr (ST == SGFD_STORE_F32) return 1.0f;
        else return scl[k];
    }
    __device__ __forceinline__ float inv(int k) const {
        if constexpr (ST == SGFD_STORE_F32) return 1.0f;
        else return scl[9 + k];
    }
};


// Common per-thread state of both updates.
struct PairCtx {
    int gx, gy;          // GRID coordinates of cell 0
    bool act0, act1;     // cells inside the computed region
    int kx0, kx1, ky;    // PML band distances
    uint32_t col;        // element offset of the pair at z = 0 (in bounds for inactive pairs)
    PmlColumn pc0, pc1;
};

__device__ __forceinline__ PairCtx pair_ctx(const Model &m, const PTile &t, int lx, int ly) {
    PairCtx p;
    p.gx = t.gx0 + 2 * lx;       // odd GRID x: the pair is 8-byte aligned in the device rows
    p.gy = t.gy0 + ly;
    const bool row_ok = t.cy0 + ly < m.nyc;
    p.act0 = row_ok && t.cx0 + 2 * lx < m.nxc;
    p.act1 = row_ok && t.cx0 + 2 * lx + 1 < m.nxc;
    p.kx0 = band(p.gx, m.nx, m.pml);
    p.kx1 = band(p.gx + 1, m.nx, m.pml);
    p.ky = band(p.gy, m.ny, m.pml);
    const int nxo = (m.nx - 2) | 1;   // largest odd x whose pair stays inside the row
    p.col = (uint32_t)pidx(m, min(p.gx, nxo), min(p.gy, m.ny - 1), 0);
    p.pc0 = pml_column(m, min(t.cx0 + 2 * lx, m.nxc - 1), min(t.cy0 + ly, m.nyc - 1));
    p.pc1 = pml_column(m, min(t.cx0 + 2 * lx + 1, m.nxc - 1), min(t.cy0 + ly, m.nyc - 1));
    return p;
}


// ---------------------------------------------------------------------------
// velocity update
// ---------------------------------------------------------------------------

// One work item of the vel update: tile `tile`, z chunk `chunk`.  The
// ring's barriers (bar, S of them) are initialised by the caller; pbits holds
// the parity of the next wait of each stage and carries over between the
// work items of a persistent caller.  Returns false when the block gave up
// on a wait (after waiting, bounded, for its own copies still in flight).
template <bool FAST, int ST>
__device__ __forceinline__ bool vel_pair(const VelMaps &mp, const Model &m, const Physics &ph, const ZGeom &g,
                                        const SourceRec &sr, const HalfState &hs, int it_arg, float src_value,
                                        int use_wavelet, int tile, int chunk, unsigned char *smem, uint64_t *bar,
                                        TmaBox (*boxes)[kMaxBoxesPerWarp], uint32_t &pbits) {
    using SA = Sto<ST>;
    using E = typename SA::E;
    using L = VelP<SA::ES>;
    constexpr int S = SV;
    constexpr bool H = ST != SGFD_STORE_F32;   // 16-bit storage: source and receivers run as separate kernels
    __shared__ float scl[18];   // 16-bit storage: this step's scales, read at every tap
    __shared__ unsigned smax[9];   // 16-bit storage, rescale steps: this CTA's largest written magnitudes
    if constexpr (ST != SGFD_STORE_F32) {
        if (threadIdx.x < 9) {
            scl[threadIdx.x] = hs.sc[threadIdx.x];
            scl[9 + threadIdx.x] = hs.inv[threadIdx.x];
            smax[threadIdx.x] = 0u;
        }
        __syncthreads();
    }
    const Fields<ST> F(m, hs, scl);
    const PTile t = make_ptile(m, g, tile, chunk);
    const int tid = threadIdx.x, lx = tid & 31, ly = tid >> 5, warp = ly;
    const TmaBox *mybox = boxes[warp];
    const int nbox = (kVelBoxes - warp + kWarps - 1) / kWarps;
    if (lx == 0) {
        fence_proxy_async();   // a persistent caller's previous item read these stages
        for (int j = 0; j < nbox; ++j) boxes[warp][j] = vel_box<SA::ES>(mp, t, warp + j * kWarps);
        for (int s = 0; s < S && t.zs + s < t.ze; ++s)
            issue(mybox, nbox, smem + s * L::STAGE, &bar[s], t.zs + s, warp, L::TXB);
    }
    int issued_end = min(t.zs + S, t.ze);   // planes [zs, issued_end) issued
    int stage = 0;                          // stage of plane cz

    const int it = step_index(sr, it_arg);
    const float inj = ph.inj_dt2 * ((use_wavelet && sr.wavelet) ? sr.wavelet[it] : src_value);
    const bool track = H && rescale_step16(it);
    int sx = -1, sy = -1, sz = -1;
    if (!H && sr.src >= 0) {
        const int64_t r = sr.src;
        sz = (int)(r / m.plane);
        sy = (int)((r - (int64_t)sz * m.plane) / m.px);
        sx = (int)(r - (int64_t)sz * m.plane - (int64_t)sy * m.px);
    }
    const PairCtx pc = pair_ctx(m, t, lx, ly);
    const uint32_t PL = (uint32_t)m.plane;

    // z queues (both cells), 11 deep: planes are taken two at a time, the
    // even plane of a pair reads entries 0..9, the odd one 1..10, and the
    // queues move by two after the odd plane.  qxz, qyz hold z-5..z+4 and qzz
    // z-4..z+5 of the even plane; filled 9 deep here.
    float2 qxz[11], qyz[11], qzz[11];
    const int gz0 = t.zs + kHalo;
#pragma unroll
    for (int k = 0; k < 9; ++k) {
        qxz[k] = SA::pair(F.f(7) + pc.col + (uint32_t)(gz0 - 5 + k) * PL, bcast(F.sc(7)));
        qyz[k] = SA::pair(F.f(8) + pc.col + (uint32_t)(gz0 - 5 + k) * PL, bcast(F.sc(8)));
        float2 zz = SA::pair(F.f(5) + pc.col + (uint32_t)(gz0 - 4 + k) * PL, bcast(F.sc(5)));
        if (!H && pc.gy == sy && gz0 - 4 + k == sz) {
            if (pc.gx == sx) zz.x = zz.x + inj;
            if (pc.gx + 1 == sx) zz.y = zz.y + inj;
        }
        qzz[k] = zz;
    }

    // receivers of this tile, sorted by z: skip those below the chunk
    int rp = H ? 0 : g.rec_off[tile];
    const int rend = H ? 0 : g.rec_off[tile + 1];
    while (rp < rend && g.rec_list[rp].z < gz0) ++rp;
    int rz = rp < rend ? g.rec_list[rp].z : 0x7fffffff;

    bool failed = false, abort = false;
    int cz = t.zs;
    const bool src_near = !H && sr.src >= 0 && sy >= t.gy0 - 5 && sy < t.gy0 + PY + 5 && sx >= t.gx0 - 8 &&
                          sx < t.gx0 + PX + 8;
    // One plane.  GEN selects the general path (PML cells, source, receivers);
    // every other tile-plane takes the packed interior path.  ODD: the second
    // plane of a pair (queue window one entry further).  Returns false when
    // the block votes to abort.
    auto plane = [&](auto gen_tag, auto odd_tag) -> bool {
        constexpr bool GEN = decltype(gen_tag)::value;
        constexpr int Q = decltype(odd_tag)::value ? 1 : 0;
        const int s = stage;
        unsigned char *st = smem + s * L::STAGE;
        const int gz = cz + kHalo;
        const int kz = bandz(m, gz);

        if (mbar_wait(&bar[s], (pbits >> s) & 1u)) pbits ^= 1u << s;
        else failed = true;

        // source patch of the staged copies (uniform branch)
        if constexpr (!H) if (GEN && src_near && (gz == sz || gz + 5 == sz)) {
            if (tid == 0) {
                const int ox = sx - t.gx0, oy = sy - t.gy0;
                if (gz == sz) {
                    float *sxx = reinterpret_cast<float *>(st + L::SXX);
                    float *syy = reinterpret_cast<float *>(st + L::SYY);
                    if (oy >= 0 && oy < PY && ox + 8 >= 0 && ox + 8 < XW) sxx[oy * XW + ox + 8] += inj;
                    if (oy + 5 >= 0 && oy + 5 < PY + 10 && ox >= 0 && ox < PX) syy[(oy + 5) * PX + ox] += inj;
                }
                if (gz + 5 == sz) {
                    float *szz = reinterpret_cast<float *>(st + L::LZZ);
                    if (oy >= 0 && oy < PY && ox >= 0 && ox < PX) szz[oy * PX + ox] += inj;
                }
            }
            __syncthreads();
        }

        const E *sxx = reinterpret_cast<const E *>(st + L::SXX);
        const E *syy = reinterpret_cast<const E *>(st + L::SYY);
        const E *sxy = reinterpret_cast<const E *>(st + L::SXY);
        const E *sxz = reinterpret_cast<const E *>(st + L::SXZ);
        const E *syz = reinterpret_cast<const E *>(st + L::SYZ);
        const float *bb = reinterpret_cast<const float *>(st + L::B);
        const E *ov = reinterpret_cast<const E *>(st + L::OV);
        constexpr int OVS = L::OBE / SA::ES;        // values between the own-velocity boxes
        const int e = ly * PX + 2 * lx;             // 64 x 8 box index of cell 0

        // the lead planes enter the z queues
        qxz[9 + Q] = SA::pair(reinterpret_cast<const E *>(st + L::LXZ) + e, bcast(F.sc(7)));
        qyz[9 + Q] = SA::pair(reinterpret_cast<const E *>(st + L::LYZ) + e, bcast(F.sc(8)));
        qzz[9 + Q] = SA::pair(reinterpret_cast<const E *>(st + L::LZZ) + e, bcast(F.sc(5)));

        if (pc.act0) {
            // x differences, per cell, from 12-value windows
            float w[12];
            SA::win(sxx + ly * XW + 2 * lx + 4, w, F.sc(3));     // x offsets -4 .. 7 of cell 0
            const float2 xX = dFx<FAST>(ph, w, -4);
            SA::win(sxy + (ly + 5) * XW + 2 * lx + 2, w, F.sc(6));  // -6 .. 5
            const float2 yX = dBx<FAST>(ph, w, -6);
            SA::win(sxz + ly * XW + 2 * lx + 2, w, F.sc(7));
            const float2 zX = dBx<FAST>(ph, w, -6);
            // y and z differences, both cells at once
            const E *cxy = sxy + (ly + 5) * XW + 2 * lx + 8;
            const E *cyy = syy + (ly + 5) * PX + 2 * lx;
            const E *cyz = syz + (ly + 5) * PX + 2 * lx;
            const float2 s6 = bcast(F.sc(6)), s4 = bcast(F.sc(4)), s8 = bcast(F.sc(8));
            const float2 xY = dB2p<FAST, 1>(ph, [&](int o) { return SA::pair(cxy + o * XW, s6); });
            const float2 yY = dF2p<FAST, 1>(ph, [&](int o) { return SA::pair(cyy + o * PX, s4); });
            const float2 zY = dB2p<FAST, 1>(ph, [&](int o) { return SA::pair(cyz + o * PX, s8); });
            const float2 xZ = dB2p<FAST, 2>(ph, [&](int o) { return qxz[Q + 5 + o]; });
            const float2 yZ = dB2p<FAST, 2>(ph, [&](int o) { return qyz[Q + 5 + o]; });
            const float2 zZ = dF2p<FAST, 2>(ph, [&](int o) { return qzz[Q + 4 + o]; });

            const float2 b0 = ld2(bb + ly * BW + 2 * lx);
            const float2 bxp = make_float2(b0.y, bb[ly * BW + 2 * lx + 2]);
            const float2 byp = ld2(bb + (ly + 1) * BW + 2 * lx);
            const float2 bzp = ld2(reinterpret_cast<const float *>(st + L::LB) + e);
            const float2 half = bcast(0.5f);            // (a + b) / 2 rounds as (a + b) * 0.5
            const float2 bx = __fmul2_rn(__fadd2_rn(b0, bxp), half);
            const float2 by = __fmul2_rn(__fadd2_rn(b0, byp), half);
            const float2 bz = __fmul2_rn(__fadd2_rn(b0, bzp), half);
            const float2 dt2 = bcast(ph.dt);
            const uint32_t ci = pc.col + (uint32_t)gz * PL;   // cell 0

            const bool pml0 = (pc.kx0 | pc.ky | kz) != 0, pml1 = (pc.kx1 | pc.ky | kz) != 0;
            if (!(GEN && (t.xy_pml || kz != 0) && (pml0 || (pc.act1 && pml1)))) {
                const float2 v0 = __ffma2_rn(__fmul2_rn(dt2, bx), __fadd2_rn(__fadd2_rn(xX, xY), xZ),
                                             SA::pair(ov + e, bcast(F.sc(0))));
                const float2 v1 = __ffma2_rn(__fmul2_rn(dt2, by), __fadd2_rn(__fadd2_rn(yX, yY), yZ),
                                             SA::pair(ov + OVS + e, bcast(F.sc(1))));
                const float2 v2 = __ffma2_rn(__fmul2_rn(dt2, bz), __fadd2_rn(__fadd2_rn(zX, zY), zZ),
                                             SA::pair(ov + 2 * OVS + e, bcast(F.sc(2))));
                SA::put2(F.f(0) + ci, v0, bcast(F.inv(0)), pc.act1);
                SA::put2(F.f(1) + ci, v1, bcast(F.inv(1)), pc.act1);
                SA::put2(F.f(2) + ci, v2, bcast(F.inv(2)), pc.act1);
                if (track) {
                    note_max16s(smax, 0, fmaxf(fabsf(v0.x), pc.act1 ? fabsf(v0.y) : 0.0f));
                    note_max16s(smax, 1, fmaxf(fabsf(v1.x), pc.act1 ? fabsf(v1.y) : 0.0f));
                    note_max16s(smax, 2, fmaxf(fabsf(v2.x), pc.act1 ? fabsf(v2.y) : 0.0f));
                }
                if (!H && GEN && gz == rz && it >= 0 && it < sr.nt) {
                    for (int r = rp; r < rend && g.rec_list[r].z == gz; ++r) {
                        const int4 q = g.rec_list[r];
                        if (q.y == pc.gy && q.w <= 2 && (q.x == pc.gx || (pc.act1 && q.x == pc.gx + 1))) {
                            const int c = q.x - pc.gx;
                            sr.traces[(int64_t)it * sr.nrec + g.rec_idx[r]] =
                                q.w == 0 ? lane_of(v0, c) : q.w == 1 ? lane_of(v1, c) : lane_of(v2, c);
                        }
                    }
                }
            } else {
                // general path, cell by cell; PML cells through their split fields
#pragma unroll
                for (int c = 0; c < 2; ++c) {
                    if (c == 1 && !pc.act1) break;
                    const int kx = c ? pc.kx1 : pc.kx0, ky = pc.ky;
                    const uint32_t cc = ci + c;
                    float vnew[3];
                    if (!(kx | ky | kz)) {
                        vnew[0] = __fmaf_rn(ph.dt * lane_of(bx, c), (lane_of(xX, c) + lane_of(xY, c)) + lane_of(xZ, c),
                                            SA::one(ov + e + c, F.sc(0)));
                        vnew[1] = __fmaf_rn(ph.dt * lane_of(by, c), (lane_of(yX, c) + lane_of(yY, c)) + lane_of(yZ, c),
                                            SA::one(ov + OVS + e + c, F.sc(1)));
                        vnew[2] = __fmaf_rn(ph.dt * lane_of(bz, c), (lane_of(zX, c) + lane_of(zY, c)) + lane_of(zZ, c),
                                            SA::one(ov + 2 * OVS + e + c, F.sc(2)));
                    } else {
                        // every global load of the cell first: the split stores below could
                        // alias them as far as the compiler knows, so loads after a store wait
                        E *sp = F.split() + split_base32(pml_plane_index(m, c ? pc.pc1 : pc.pc0, cz));
                        const uint32_t N = kSplitBlock;   // split k at sp[k * N]
                        float o[9];
#pragma unroll
                        for (int k = 0; k < 9; ++k) o[k] = SA::one(sp + k * N, F.sc(k / 3));
                        const float mu_c = m.mu[cc], lam_c = ph.damping == 1 ? m.lam[cc] : 0.f;
                        float mx = 1.f, my = 1.f, mz = 1.f;
        PDiv<FAST> px = 1, py = 1, pz = 1;
                        {
                            const float v = damp_speed(ph, mu_c, lane_of(b0, c), lam_c);
                            if (kx) damp_factors<FAST>(ph, 0, ph.dx, kx, m.pml, v, mx, px);
                            if (ky) damp_factors<FAST>(ph, 1, ph.dy, ky, m.pml, v, my, py);
                            if (kz) damp_factors<FAST>(ph, 2, ph.dz, kz, m.pml, v, mz, pz);
                        }
                        const bool ref = ph.quirks == 0;
                        const float bxc = lane_of(bx, c);
                        const float ax = ph.dt * bxc, ay = ph.dt * (ref ? bxc : lane_of(by, c)),
                                    az = ph.dt * (ref ? bxc : lane_of(bz, c));
                        const float dxyz[3][3] = {{lane_of(xX, c), lane_of(xY, c), lane_of(xZ, c)},
                                                  {lane_of(yX, c), lane_of(yY, c), lane_of(yZ, c)},
                                                  {lane_of(zX, c), lane_of(zY, c), lane_of(zZ, c)}};
                        const float aq[3] = {ax, ay, az};
                        const int kk[3] = {kx, ky, kz};
                        const float mm[3] = {mx, my, mz};
        const PDiv<FAST> pp[3] = {px, py, pz};
#pragma unroll
                        for (int q = 0; q < 3; ++q) {
                            float part[3];
#pragma unroll
                            for (int a = 0; a < 3; ++a) {
                                // split S_VXX + 3q + a, in the scale of field q
                                part[a] = split_update<FAST>(o[3 * q + a], aq[q], dxyz[q][a], kk[a], mm[a], pp[a]);
                                if (track) note_max16s(smax, q, part[a]);
                                SA::put1(sp + (3 * q + a) * N, part[a], F.inv(q));
                            }
                            vnew[q] = (part[0] + part[1]) + part[2];
                        }
                    }
#pragma unroll
                    for (int q = 0; q < 3; ++q) {
                        if (track) note_max16s(smax, q, vnew[q]);
                        SA::put1(F.f(q) + cc, vnew[q], F.inv(q));
                    }
                    if (!H && gz == rz && it >= 0 && it < sr.nt) {
                        for (int r = rp; r < rend && g.rec_list[r].z == gz; ++r) {
                            const int4 q = g.rec_list[r];
                            if (q.x == pc.gx + c && q.y == pc.gy && q.w <= 2)
                                sr.traces[(int64_t)it * sr.nrec + g.rec_idx[r]] =
                                    q.w == 0 ? vnew[0] : q.w == 1 ? vnew[1] : vnew[2];
                        }
                    }
                }
            }
        }
        if (GEN && gz == rz) {
            while (rp < rend && g.rec_list[rp].z == gz) ++rp;
            rz = rp < rend ? g.rec_list[rp].z : 0x7fffffff;
        }
        if constexpr (Q == 1) {   // after a pair of planes the queues move by two
#pragma unroll
            for (int j = 0; j < 9; ++j) {
                qxz[j] = qxz[j + 2];
                qyz[j] = qyz[j + 2];
                qzz[j] = qzz[j + 2];
            }
        }

        // every thread is done with this stage: vote on aborts, then refill it
        if (__syncthreads_or(failed)) return false;
        if (cz + S < t.ze) {
            if (lx == 0) {
                fence_proxy_async();
                issue(mybox, nbox, st, &bar[s], cz + S, warp, L::TXB);
            }
            issued_end = cz + S + 1;
        }
        if (++stage == S) stage = 0;
        return true;
    };
    using T1 = std::true_type;
    using T0 = std::false_type;
    for (; cz < t.ze; ++cz) {
        const int gzp = cz + kHalo;
        const bool gen = t.xy_pml || bandz(m, gzp) != 0 || (src_near && (gzp == sz || gzp + 5 == sz)) ||
                         gzp == rz;
        const bool odd = ((cz - t.zs) & 1) != 0;
        const bool ok = odd ? (gen ? plane(T1{}, T1{}) : plane(T0{}, T1{})) : (gen ? plane(T1{}, T0{}) : plane(T0{}, T0{}));
        if (!ok) {
            abort = true;
            break;
        }
    }
    if (abort && tid == 0) {
        atomicExch(g.err, 1);
        // planes still in flight: [cz, issued_end), less plane cz when this
        // thread's own wait for it completed
        for (int j = failed ? cz : cz + 1; j < issued_end; ++j) {
            const int q = (j - t.zs) % S;
            mbar_wait(&bar[q], (pbits >> q) & 1u);
            pbits ^= 1u << q;
        }
    }
    if constexpr (H) {
        if (track) {
            __syncthreads();
            flush_max16(hs, smax);
        }
    }
    return !abort;
}

// ---------------------------------------------------------------------------
// stress update
// ---------------------------------------------------------------------------

// One work item of the str update: tile `tile`, z chunk `chunk`.  The
// ring's barriers (bar, S of them) are initialised by the caller; pbits holds
// the parity of the next wait of each stage and carries over between the
// work items of a persistent caller.  Returns false when the block gave up
// on a wait (after waiting, bounded, for its own copies still in flight).
template <bool FAST, int ST>
__device__ __forceinline__ bool str_pair(const StrMaps &mp, const Model &m, const Physics &ph, const ZGeom &g,
                                        const SourceRec &sr, const HalfState &hs, int it_arg, float src_value,
                                        int use_wavelet, int tile, int chunk, unsigned char *smem, uint64_t *bar,
                                        TmaBox (*boxes)[kMaxBoxesPerWarp], uint32_t &pbits) {
    using SA = Sto<ST>;
    using E = typename SA::E;
    using L = StrP<SA::ES>;
    constexpr int S = SS;
    constexpr bool H = ST != SGFD_STORE_F32;   // 16-bit storage: source and receivers run as separate kernels
    __shared__ float scl[18];   // 16-bit storage: this step's scales, read at every tap
    __shared__ unsigned smax[9];   // 16-bit storage, rescale steps: this CTA's largest written magnitudes
    if constexpr (ST != SGFD_STORE_F32) {
        if (threadIdx.x < 9) {
            scl[threadIdx.x] = hs.sc[threadIdx.x];
            scl[9 + threadIdx.x] = hs.inv[threadIdx.x];
            smax[threadIdx.x] = 0u;
        }
        __syncthreads();
    }
    const Fields<ST> F(m, hs, scl);
    const PTile t = make_ptile(m, g, tile, chunk);
    const int tid = threadIdx.x, lx = tid & 31, ly = tid >> 5, warp = ly;
    const TmaBox *mybox = boxes[warp];
    const int nbox = (kStrBoxes - warp + kWarps - 1) / kWarps;
    if (lx == 0) {
        fence_proxy_async();
        for (int j = 0; j < nbox; ++j) boxes[warp][j] = str_box<SA::ES>(mp, t, warp + j * kWarps);
        for (int s = 0; s < S && t.zs + s < t.ze; ++s)
            issue(mybox, nbox, smem + s * L::STAGE, &bar[s], t.zs + s, warp, L::TXB);
    }
    int issued_end = min(t.zs + S, t.ze);
    int stage = 0;                          // stage of plane cz

    const int it = step_index(sr, it_arg);
    const float inj = ph.inj_dt2 * ((use_wavelet && sr.wavelet) ? sr.wavelet[it] : src_value);
    const int64_t src = H ? -1 : sr.src;
    const bool track = H && rescale_step16(it);
    const PairCtx pc = pair_ctx(m, t, lx, ly);
    const uint32_t PL = (uint32_t)m.plane;

    // z queues (both cells), 11 deep and taken two planes at a time as in
    // the velocity update: qx, qy hold z-4..z+5 (vx, vy), qz holds z-5..z+4
    // (vz) of the even plane
    float2 qx[11], qy[11], qz[11];
    const int gz0 = t.zs + kHalo;
#pragma unroll
    for (int k = 0; k < 9; ++k) {
        qx[k] = SA::pair(F.f(0) + pc.col + (uint32_t)(gz0 - 4 + k) * PL, bcast(F.sc(0)));
        qy[k] = SA::pair(F.f(1) + pc.col + (uint32_t)(gz0 - 4 + k) * PL, bcast(F.sc(1)));
        qz[k] = SA::pair(F.f(2) + pc.col + (uint32_t)(gz0 - 5 + k) * PL, bcast(F.sc(2)));
    }

    int rp = H ? 0 : g.rec_off[tile];
    const int rend = H ? 0 : g.rec_off[tile + 1];
    while (rp < rend && g.rec_list[rp].z < gz0) ++rp;
    int rz = rp < rend ? g.rec_list[rp].z : 0x7fffffff;

    bool failed = false, abort = false;
    int cz = t.zs;
    const int sz = src >= 0 ? (int)(src / m.plane) : -1;
    auto plane = [&](auto gen_tag, auto odd_tag) -> bool {
        constexpr bool GEN = decltype(gen_tag)::value;
        constexpr int Q = decltype(odd_tag)::value ? 1 : 0;
        const int s = stage;
        unsigned char *st = smem + s * L::STAGE;
        const int gz = cz + kHalo;
        const int kz = bandz(m, gz);

        if (mbar_wait(&bar[s], (pbits >> s) & 1u)) pbits ^= 1u << s;
        else failed = true;

        const E *svx = reinterpret_cast<const E *>(st + L::VX);
        const E *svy = reinterpret_cast<const E *>(st + L::VY);
        const E *svz = reinterpret_cast<const E *>(st + L::VZ);
        // own-cell boxes: txx..tyz (wavefield values), then lambda, mu and the
        // three shear moduli (FP32)
        const E *own = reinterpret_cast<const E *>(st + L::OWN);
        const float *med = reinterpret_cast<const float *>(st + L::MED);
        constexpr int OS = L::OBE / SA::ES, MS = OB / 4;
        const int e = ly * PX + 2 * lx;

        qx[9 + Q] = SA::pair(reinterpret_cast<const E *>(st + L::LX) + e, bcast(F.sc(0)));
        qy[9 + Q] = SA::pair(reinterpret_cast<const E *>(st + L::LY) + e, bcast(F.sc(1)));
        qz[9 + Q] = SA::pair(reinterpret_cast<const E *>(st + L::LZ) + e, bcast(F.sc(2)));

        if (pc.act0) {
            float w[12];
            SA::win(svx + (ly + 5) * XW + 2 * lx + 2, w, F.sc(0));  // x offsets -6 .. 5 of cell 0
            const float2 dXx = dBx<FAST>(ph, w, -6);
            SA::win(svy + (ly + 5) * XW + 2 * lx + 4, w, F.sc(1));  // -4 .. 7
            const float2 xyX = dFx<FAST>(ph, w, -4);
            SA::win(svz + (ly + 5) * XW + 2 * lx + 4, w, F.sc(2));
            const float2 xzX = dFx<FAST>(ph, w, -4);
            const E *cx_ = svx + (ly + 5) * XW + 2 * lx + 8;
            const E *cy_ = svy + (ly + 5) * XW + 2 * lx + 8;
            const E *cz_ = svz + (ly + 5) * XW + 2 * lx + 8;
            const float2 s0 = bcast(F.sc(0)), s1 = bcast(F.sc(1)), s2 = bcast(F.sc(2));
            const float2 dYy = dB2p<FAST, 1>(ph, [&](int o) { return SA::pair(cy_ + o * XW, s1); });
            const float2 xyY = dF2p<FAST, 1>(ph, [&](int o) { return SA::pair(cx_ + o * XW, s0); });
            const float2 yzY = dF2p<FAST, 1>(ph, [&](int o) { return SA::pair(cz_ + o * XW, s2); });
            const float2 xzZ = dF2p<FAST, 2>(ph, [&](int o) { return qx[Q + 4 + o]; });
            const float2 yzZ = dF2p<FAST, 2>(ph, [&](int o) { return qy[Q + 4 + o]; });
            const float2 dZz = dB2p<FAST, 2>(ph, [&](int o) { return qz[Q + 5 + o]; });

            const float2 l = ld2(med + e), mu2 = ld2(med + MS + e);
            const float2 l2m = __ffma2_rn(bcast(2.0f), mu2, l);
            const float2 mxy = ld2(med + 2 * MS + e), mxz = ld2(med + 3 * MS + e), myz = ld2(med + 4 * MS + e);
            const uint32_t ci = pc.col + (uint32_t)gz * PL;
            const float2 dt2 = bcast(ph.dt);

            const bool pml0 = (pc.kx0 | pc.ky | kz) != 0, pml1 = (pc.kx1 | pc.ky | kz) != 0;
            if (!(GEN && (t.xy_pml || kz != 0) && (pml0 || (pc.act1 && pml1)))) {
                float2 o0 = SA::pair(own + e, bcast(F.sc(3))), o1 = SA::pair(own + OS + e, bcast(F.sc(4))),
                       o2 = SA::pair(own + 2 * OS + e, bcast(F.sc(5)));
                if (GEN && (int64_t)ci == src) { o0.x = o0.x + inj; o1.x = o1.x + inj; o2.x = o2.x + inj; }
                if (GEN && (int64_t)ci + 1 == src) { o0.y = o0.y + inj; o1.y = o1.y + inj; o2.y = o2.y + inj; }
                float2 sn[6];
                sn[0] = __ffma2_rn(dt2, __ffma2_rn(l2m, dXx, __fmul2_rn(l, __fadd2_rn(dYy, dZz))), o0);
                sn[1] = __ffma2_rn(dt2, __ffma2_rn(l2m, dYy, __fmul2_rn(l, __fadd2_rn(dXx, dZz))), o1);
                sn[2] = __ffma2_rn(dt2, __ffma2_rn(l2m, dZz, __fmul2_rn(l, __fadd2_rn(dXx, dYy))), o2);
                sn[3] = __ffma2_rn(__fmul2_rn(dt2, mxy), __fadd2_rn(xyY, xyX), SA::pair(own + 3 * OS + e, bcast(F.sc(6))));
                sn[4] = __ffma2_rn(__fmul2_rn(dt2, mxz), __fadd2_rn(xzZ, xzX), SA::pair(own + 4 * OS + e, bcast(F.sc(7))));
                sn[5] = __ffma2_rn(__fmul2_rn(dt2, myz), __fadd2_rn(yzZ, yzY), SA::pair(own + 5 * OS + e, bcast(F.sc(8))));
#pragma unroll
                for (int q = 0; q < 6; ++q) {
                    SA::put2(F.f(3 + q) + ci, sn[q], bcast(F.inv(3 + q)), pc.act1);
                    if (track) note_max16s(smax, 3 + q, fmaxf(fabsf(sn[q].x), pc.act1 ? fabsf(sn[q].y) : 0.0f));
                }
                if (!H && GEN && gz == rz && it >= 0 && it < sr.nt) {
                    for (int r = rp; r < rend && g.rec_list[r].z == gz; ++r) {
                        const int4 q = g.rec_list[r];
                        if (q.y == pc.gy && q.w >= 3 && (q.x == pc.gx || (pc.act1 && q.x == pc.gx + 1)))
                            sr.traces[(int64_t)it * sr.nrec + g.rec_idx[r]] = lane_of(pick6(sn, q.w - 3), q.x - pc.gx);
                    }
                }
            } else {
#pragma unroll
                for (int c = 0; c < 2; ++c) {
                    if (c == 1 && !pc.act1) break;
                    const int kx = c ? pc.kx1 : pc.kx0, ky = pc.ky;
                    const uint32_t cc = ci + c;
                    const float lc = lane_of(l, c), mu_c = lane_of(mu2, c), l2mc = lane_of(l2m, c);
                    const float dXxc = lane_of(dXx, c), dYyc = lane_of(dYy, c), dZzc = lane_of(dZz, c);
                    float snew[6];
                    if (!(kx | ky | kz)) {
                        float o0 = SA::one(own + e + c, F.sc(3)), o1 = SA::one(own + OS + e + c, F.sc(4)),
                              o2 = SA::one(own + 2 * OS + e + c, F.sc(5));
                        if ((int64_t)cc == src) { o0 = o0 + inj; o1 = o1 + inj; o2 = o2 + inj; }
                        snew[0] = __fmaf_rn(ph.dt, __fmaf_rn(l2mc, dXxc, lc * (dYyc + dZzc)), o0);
                        snew[1] = __fmaf_rn(ph.dt, __fmaf_rn(l2mc, dYyc, lc * (dXxc + dZzc)), o1);
                        snew[2] = __fmaf_rn(ph.dt, __fmaf_rn(l2mc, dZzc, lc * (dXxc + dYyc)), o2);
                        snew[3] = __fmaf_rn(ph.dt * lane_of(mxy, c), lane_of(xyY, c) + lane_of(xyX, c),
                                            SA::one(own + 3 * OS + e + c, F.sc(6)));
                        snew[4] = __fmaf_rn(ph.dt * lane_of(mxz, c), lane_of(xzZ, c) + lane_of(xzX, c),
                                            SA::one(own + 4 * OS + e + c, F.sc(7)));
                        snew[5] = __fmaf_rn(ph.dt * lane_of(myz, c), lane_of(yzZ, c) + lane_of(yzY, c),
                                            SA::one(own + 5 * OS + e + c, F.sc(8)));
                    } else {
                        E *sp = F.split() + split_base32(pml_plane_index(m, c ? pc.pc1 : pc.pc0, cz));
                        const uint32_t N = kSplitBlock;   // split k at sp[k * N]
                        // split k, in its field's scale (S_XXX.. -> txx.., two per shear stress)
                        auto grp = [](int k) { return k < S_XYX ? 3 + (k - S_XXX) / 3 : 6 + (k - S_XYX) / 2; };
                        // every global load of the cell first (the split stores could alias them)
                        float o[15];
#pragma unroll
                        for (int k = 0; k < 15; ++k) o[k] = SA::one(sp + (S_XXX + k) * N, F.sc(grp(S_XXX + k)));
                        const float b_c = m.b[cc];
                        auto rd = [&](int k) { return o[k - S_XXX]; };
                        auto wr = [&](int k, float v) {
                            if (track) note_max16s(smax, grp(k), v);
                            SA::put1(sp + k * N, v, F.inv(grp(k)));
                        };
                        float mx = 1.f, my = 1.f, mz = 1.f;
        PDiv<FAST> px = 1, py = 1, pz = 1;
                        {
                            const float v = damp_speed(ph, mu_c, b_c, lc);
                            if (kx) damp_factors<FAST>(ph, 0, ph.dx, kx, m.pml, v, mx, px);
                            if (ky) damp_factors<FAST>(ph, 1, ph.dy, ky, m.pml, v, my, py);
                            if (kz) damp_factors<FAST>(ph, 2, ph.dz, kz, m.pml, v, mz, pz);
                        }
                        const float dl = ph.dt * l2mc, dt = ph.dt;
                        float a0, a1, a2;
                        a0 = split_update<FAST>(rd(S_XXX), dl, dXxc, kx, mx, px);
                        a1 = split_update<FAST>(rd(S_XXY), dt, lc * dYyc, ky, my, py);
                        a2 = split_update<FAST>(rd(S_XXZ), dt, lc * dZzc, kz, mz, pz);
                        wr(S_XXX, a0); wr(S_XXY, a1); wr(S_XXZ, a2);
                        snew[0] = (a0 + a1) + a2;
                        a0 = split_update<FAST>(rd(S_YYX), dt, lc * dXxc, kx, mx, px);
                        a1 = split_update<FAST>(rd(S_YYY), dl, dYyc, ky, my, py);
                        a2 = split_update<FAST>(rd(S_YYZ), dt, lc * dZzc, kz, mz, pz);
                        wr(S_YYX, a0); wr(S_YYY, a1); wr(S_YYZ, a2);
                        snew[1] = (a0 + a1) + a2;
                        a0 = split_update<FAST>(rd(S_ZZX), dt, lc * dXxc, kx, mx, px);
                        a1 = split_update<FAST>(rd(S_ZZY), dt, lc * dYyc, ky, my, py);
                        a2 = split_update<FAST>(rd(S_ZZZ), dl, dZzc, kz, mz, pz);
                        wr(S_ZZX, a0); wr(S_ZZY, a1); wr(S_ZZZ, a2);
                        snew[2] = (a0 + a1) + a2;
                        const float axy = dt * lane_of(mxy, c), axz = dt * lane_of(mxz, c),
                                    ayz = dt * lane_of(myz, c);
                        a0 = split_update<FAST>(rd(S_XYX), axy, lane_of(xyX, c), kx, mx, px);
                        a1 = split_update<FAST>(rd(S_XYY), axy, lane_of(xyY, c), ky, my, py);
                        wr(S_XYX, a0); wr(S_XYY, a1);
                        snew[3] = a0 + a1;
                        a0 = split_update<FAST>(rd(S_XZX), axz, lane_of(xzX, c), kx, mx, px);
                        a1 = split_update<FAST>(rd(S_XZZ), axz, lane_of(xzZ, c), kz, mz, pz);
                        wr(S_XZX, a0); wr(S_XZZ, a1);
                        snew[4] = a0 + a1;
                        a0 = split_update<FAST>(rd(S_YZY), ayz, lane_of(yzY, c), ky, my, py);
                        a1 = split_update<FAST>(rd(S_YZZ), ayz, lane_of(yzZ, c), kz, mz, pz);
                        wr(S_YZY, a0); wr(S_YZZ, a1);
                        snew[5] = a0 + a1;
                    }
#pragma unroll
                    for (int q = 0; q < 6; ++q) {
                        if (track) note_max16s(smax, 3 + q, snew[q]);
                        SA::put1(F.f(3 + q) + cc, snew[q], F.inv(3 + q));
                    }
                    if (!H && gz == rz && it >= 0 && it < sr.nt) {
                        for (int r = rp; r < rend && g.rec_list[r].z == gz; ++r) {
                            const int4 q = g.rec_list[r];
                            if (q.x == pc.gx + c && q.y == pc.gy && q.w >= 3)
                                sr.traces[(int64_t)it * sr.nrec + g.rec_idx[r]] = pick6(snew, q.w - 3);
                        }
                    }
                }
            }
        }
        if (GEN && gz == rz) {
            while (rp < rend && g.rec_list[rp].z == gz) ++rp;
            rz = rp < rend ? g.rec_list[rp].z : 0x7fffffff;
        }
        if constexpr (Q == 1) {
#pragma unroll
            for (int j = 0; j < 9; ++j) {
                qx[j] = qx[j + 2];
                qy[j] = qy[j + 2];
                qz[j] = qz[j + 2];
            }
        }

        if (__syncthreads_or(failed)) return false;
        if (cz + S < t.ze) {
            if (lx == 0) {
                fence_proxy_async();
                issue(mybox, nbox, st, &bar[s], cz + S, warp, L::TXB);
            }
            issued_end = cz + S + 1;
        }
        if (++stage == S) stage = 0;
        return true;
    };
    using T1 = std::true_type;
    using T0 = std::false_type;
    for (; cz < t.ze; ++cz) {
        const int gzp = cz + kHalo;
        const bool gen = t.xy_pml || bandz(m, gzp) != 0 || gzp == sz || gzp == rz;
        const bool odd = ((cz - t.zs) & 1) != 0;
        const bool ok = odd ? (gen ? plane(T1{}, T1{}) : plane(T0{}, T1{})) : (gen ? plane(T1{}, T0{}) : plane(T0{}, T0{}));
        if (!ok) {
            abort = true;
            break;
        }
    }
    if (abort && tid == 0) {
        atomicExch(g.err, 1);
        // planes still in flight: [cz, issued_end), less plane cz when this
        // thread's own wait for it completed
        for (int j = failed ? cz : cz + 1; j < issued_end; ++j) {
            const int q = (j - t.zs) % S;
            mbar_wait(&bar[q], (pbits >> q) & 1u);
            pbits ^= 1u << q;
        }
    }
    if constexpr (H) {
        if (track) {
            __syncthreads();
            flush_max16(hs, smax);
        }
    }
    return !abort;
}

// One launch per update: one CTA per (tile, z chunk).
template <bool FAST, int ST>
__global__ void __launch_bounds__(NT, 2)
k_velocity_zpair(const __grid_constant__ VelMaps mp, const __grid_constant__ Model m, const __grid_constant__ Physics ph,
                 const __grid_constant__ ZGeom g, const __grid_constant__ SourceRec sr,
                 const __grid_constant__ HalfState hs, int it_arg, float src_value, int use_wavelet) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    __shared__ __align__(8) uint64_t bar[SV];
    __shared__ TmaBox boxes[kWarps][kMaxBoxesPerWarp];
    if (threadIdx.x == 0) {
        for (int s = 0; s < SV; ++s) mbar_init(&bar[s], 1);
        fence_barrier_init();
    }
    __syncthreads();
    uint32_t pbits = 0;
    vel_pair<FAST, ST>(mp, m, ph, g, sr, hs, it_arg, src_value, use_wavelet, blockIdx.x, blockIdx.y + g.c0,
                       align_smem(smem_raw), bar, boxes, pbits);
}

template <bool FAST, int ST>
__global__ void __launch_bounds__(NT, 2)
k_stress_zpair(const __grid_constant__ StrMaps mp, const __grid_constant__ Model m, const __grid_constant__ Physics ph,
               const __grid_constant__ ZGeom g, const __grid_constant__ SourceRec sr,
               const __grid_constant__ HalfState hs, int it_arg, float src_value, int use_wavelet) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    __shared__ __align__(8) uint64_t bar[SS];
    __shared__ TmaBox boxes[kWarps][kMaxBoxesPerWarp];
    if (threadIdx.x == 0) {
        for (int s = 0; s < SS; ++s) mbar_init(&bar[s], 1);
        fence_barrier_init();
    }
    __syncthreads();
    uint32_t pbits = 0;
    str_pair<FAST, ST>(mp, m, ph, g, sr, hs, it_arg, src_value, use_wavelet, blockIdx.x, blockIdx.y + g.c0,
                       align_smem(smem_raw), bar, boxes, pbits);
}

template <int ST>
constexpr int vel_smem() { return SV * VelP<Sto<ST>::ES>::STAGE + 128; }
template <int ST>
constexpr int str_smem() { return SS * StrP<Sto<ST>::ES>::STAGE + 128; }
static_assert(vel_smem<SGFD_STORE_F32>() <= 113 * 1024 && str_smem<SGFD_STORE_F32>() <= 113 * 1024,
              "two CTAs per SM");

template <bool FAST, int ST>
cudaError_t set_attrs() {
    cudaError_t e = cudaFuncSetAttribute(k_velocity_zpair<FAST, ST>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         vel_smem<ST>());
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_stress_zpair<FAST, ST>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 str_smem<ST>());
    return e;
}

template <bool FAST, int ST>
void launch(const Model &m, const Physics &ph, const SourceRec &sr, const HalfState &hs, const ZGeom &g,
            const VelMaps &vm, const StrMaps &sm, int it, float src_value, int uw, cudaStream_t s, cudaEvent_t *ev) {
    const dim3 grid(g.ntx * g.nty, g.nchunks);
    if (ev) cudaEventRecord(ev[0], s);
    k_velocity_zpair<FAST, ST><<<grid, NT, vel_smem<ST>(), s>>>(vm, m, ph, g, sr, hs, it, src_value, uw);
    if (ev) cudaEventRecord(ev[1], s);
    if (ST != SGFD_STORE_F32) half_phase(m, ph, sr, hs, it, src_value, uw != 0, s, 1);
    if (ev) cudaEventRecord(ev[2], s);
    k_stress_zpair<FAST, ST><<<grid, NT, str_smem<ST>(), s>>>(sm, m, ph, g, sr, hs, it, src_value, uw);
    if (ev) cudaEventRecord(ev[3], s);
}

template <int ST>
cudaError_t launch_st(const Model &m, const Physics &ph, const SourceRec &sr, const HalfState &hs, const ZGeom &g,
                      const VelMaps &vm, const StrMaps &sm, int it, float src_value, bool use_wavelet, cudaStream_t s,
                      cudaEvent_t *ev) {
    const int uw = use_wavelet ? 1 : 0;
    if (ST != SGFD_STORE_F32) half_phase(m, ph, sr, hs, it, src_value, use_wavelet, s, 0);
    if (ph.fast) launch<true, ST>(m, ph, sr, hs, g, vm, sm, it, src_value, uw, s, ev);
    else launch<false, ST>(m, ph, sr, hs, g, vm, sm, it, src_value, uw, s, ev);
    if (ST != SGFD_STORE_F32) half_phase(m, ph, sr, hs, it, src_value, use_wavelet, s, 2);
    return cudaGetLastError();
}

}  // namespace

cudaError_t zpair_prepare(const Model &m, const HalfState *hs, VelMaps *vm, StrMaps *sm) {
    constexpr int ty = PY;
    bool ok = true;
    // wavefield maps: the FP32 arrays, or the 16-bit ones of the same layout
    auto fm = [&](CUtensorMap *map, int k, int bx, int by) {
        if (hs) return make_box_map16(map, hs->f[k], m, bx, by);
        return make_box_map(map, m.f[k], m, bx, by);
    };
    ok &= fm(&vm->sxx, 3, XW, ty);
    ok &= fm(&vm->syy, 4, PX, ty + 10);
    ok &= fm(&vm->sxy, 6, XW, ty + 10);
    ok &= fm(&vm->sxz, 7, XW, ty);
    ok &= fm(&vm->syz, 8, PX, ty + 10);
    ok &= make_box_map(&vm->b, m.b, m, BW, ty + 1);
    ok &= fm(&vm->sxz_c, 7, PX, ty);
    ok &= fm(&vm->syz_c, 8, PX, ty);
    ok &= fm(&vm->szz_c, 5, PX, ty);
    ok &= make_box_map(&vm->b_c, m.b, m, PX, ty);
    for (int q = 0; q < 3; ++q) ok &= fm(&vm->own[q], q, PX, ty);
    ok &= fm(&sm->vx, 0, XW, ty + 10);
    ok &= fm(&sm->vy, 1, XW, ty + 10);
    ok &= fm(&sm->vz, 2, XW, ty + 10);
    ok &= fm(&sm->vx_c, 0, PX, ty);
    ok &= fm(&sm->vy_c, 1, PX, ty);
    ok &= fm(&sm->vz_c, 2, PX, ty);
    for (int q = 0; q < 6; ++q) ok &= fm(&sm->own[q], 3 + q, PX, ty);
    const float *med[5] = {m.lam, m.mu, m.mxy, m.mxz, m.myz};
    for (int q = 0; q < 5; ++q) ok &= make_box_map(&sm->own[6 + q], med[q], m, PX, ty);
    if (!ok) return cudaErrorInvalidValue;
    if (!hs) {
        cudaError_t e = set_attrs<false, SGFD_STORE_F32>();
        return e == cudaSuccess ? set_attrs<true, SGFD_STORE_F32>() : e;
    }
    cudaError_t e = set_attrs<false, SGFD_STORE_BF16>();
    if (e == cudaSuccess) e = set_attrs<true, SGFD_STORE_BF16>();
    if (e == cudaSuccess) e = set_attrs<false, SGFD_STORE_F16>();
    if (e == cudaSuccess) e = set_attrs<true, SGFD_STORE_F16>();
    return e;
}

void zpair_tiles(const Model &m, int *ntx, int *nty) {
    *ntx = (m.nxc + PX - 1) / PX;
    *nty = (m.nyc + PY - 1) / PY;
}

cudaError_t zpair_step(const Model &m, const Physics &ph, const SourceRec &sr, const HalfState *hs, const ZGeom &g,
                       const VelMaps &vm, const StrMaps &sm, int it, float src_value, bool use_wavelet, cudaStream_t s,
                       cudaEvent_t *ev) {
    if (!hs) return launch_st<SGFD_STORE_F32>(m, ph, sr, HalfState{}, g, vm, sm, it, src_value, use_wavelet, s, ev);
    if (hs->storage == SGFD_STORE_BF16)
        return launch_st<SGFD_STORE_BF16>(m, ph, sr, *hs, g, vm, sm, it, src_value, use_wavelet, s, ev);
    return launch_st<SGFD_STORE_F16>(m, ph, sr, *hs, g, vm, sm, it, src_value, use_wavelet, s, ev);
}

}  // namespace sgfd
