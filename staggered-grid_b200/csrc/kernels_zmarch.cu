// kernels_zmarch.cu — the "zmarch" kernel family: 2.5-D z-marching velocity
// and stress updates for sm_100a, and the persistent batch kernel built from
// the same per-tile bodies.
//
// Work decomposition.  A CTA of 256 threads owns a 32 x TY tile of computed
// cells in the xy plane (TY = 8 * CELLS, each thread owning CELLS vertically
// adjacent cells, whose y differences share one window of staged values) and
// marches along z over a chunk of planes (a work item: vel_item / str_item).
//
// Data movement per plane z (all HBM traffic is TMA or coalesced 128-byte rows):
//   * TMA (cp.async.bulk.tensor.4d over the array pool, no multicast) stages
//     the xy boxes the x/y derivatives need — tile plus its 5-cell halo on the
//     sides a field is differentiated along — and the "lead" planes that feed
//     the z register queues, and the cell's own read-modify-write data, into
//     a 3-stage shared-memory ring guarded by one mbarrier per stage (expect-tx
//     bytes, parity wait with an iteration cap).  Arrays read with the same
//     box at the same plane come in one copy (the 4th map dimension walks the
//     arrays): 8 copies per velocity plane, 4 per stress plane; lane 0 of warp
//     w issues copy w.  A stage is refilled with plane z + 3 as soon as plane
//     z is done, so every load has two plane-iterations to land.
//   * Each thread keeps the z-taps of the fields it differentiates along z in
//     register queues (sigma_xz, sigma_yz, sigma_zz for the velocity update,
//     10 deep, shifted by one per plane; vx, vy, vz for the stress update, 11
//     deep, planes taken in pairs and the queues moved by two per pair).
//   * The velocity update loads the PML split fields of its cell into
//     registers before the plane's TMA wait; the stress update, which needs
//     15 of them, loads them where they are used, so that it fits the 80
//     registers per thread of three resident CTAs per SM, and brings them
//     (and the buoyancy of the damping) into L2 one plane ahead: one bulk
//     prefetch of the 15 stress rows per 32-cell split block.
//   * 16-bit wavefield storage (ST = BF16 / F16, 32 x 8 tiles): the field
//     boxes arrive as 16-bit values and are widened once per plane into an
//     FP32 work buffer (float(h) * 2^e) before the same FP32 arithmetic.
// Every row starts at a 128-byte boundary (the device arrays are shifted by
// kXOff), so x-halo boxes start 8 cells left of the tile (48 wide), centre
// boxes are exactly 32 wide, and every TMA x coordinate is a multiple of 8.
// One block barrier per plane separates the reads of a stage from its refill
// and carries the abort vote of the bounded waits.
//
// PML cells take the split-field path (cell_math.cuh), interior cells the
// plain update; a tile-plane with no PML cell never enters the PML code.
// The source (dt*dt*s(it) on txx, tyy, tzz, OPT/ElasticWaveEquation.cu:206-221)
// is applied to the staged copies the velocity update reads and to the old
// value the stress update accumulates onto, which reproduces the reference's
// store-then-read order exactly; receivers are written from registers (with
// 16-bit storage both run as the 16-bit family's own kernels).
// Arithmetic per cell is the same sequence as kernels_simple.cu and the oracle.
#include <cuda.h>
#include <cudaTypedefs.h>

#include <type_traits>

#include "cell_math.cuh"
#include "store16.cuh"
#include "zmarch.h"
#include "zmarch_dev.cuh"

namespace sgfd {

namespace {

using namespace zdev;

constexpr int TX = kZTileX, NT = 256, S = 3;
constexpr int W48 = 48, W32 = 32, W36 = 36;

constexpr int al128(int b) { return (b + 127) / 128 * 128; }

// Shared-memory stage layout of the velocity update (bytes, 128-aligned boxes).
// Wavefield boxes hold ES-byte values (4: FP32, 2: 16-bit storage), the
// buoyancy boxes FP32.  Arrays that arrive in one 4-D copy are adjacent
// (sigma_xx, sigma_xz; sigma_yy, sigma_yz; the two lead planes at z+4; vx,
// vy, vz).
template <int TY, int ES = 4>
struct VelL {
    static constexpr int SXX = 0;                                  // 48 x TY       sigma_xx (x halo)
    static constexpr int SXZ = SXX + W48 * TY * ES;                // 48 x TY       sigma_xz (x halo)
    static constexpr int SYY = SXZ + al128(W48 * TY * ES);         // 32 x (TY+10)  sigma_yy (y halo)
    static constexpr int SYZ = SYY + W32 * (TY + 10) * ES;         // 32 x (TY+10)  sigma_yz (y halo)
    static constexpr int SXY = SYZ + al128(W32 * (TY + 10) * ES);  // 48 x (TY+10)  sigma_xy (x, y halo)
    static constexpr int B = SXY + al128(W48 * (TY + 10) * ES);    // 36 x (TY+1)   buoyancy (x+1, y+1)
    static constexpr int LXZ = B + al128(W36 * (TY + 1) * 4);      // 32 x TY       sigma_xz at z+4
    static constexpr int LYZ = LXZ + al128(W32 * TY * ES);         // 32 x TY       sigma_yz at z+4
    static constexpr int LZZ = LYZ + al128(W32 * TY * ES);         // 32 x TY       sigma_zz at z+5
    static constexpr int LB = LZZ + al128(W32 * TY * ES);          // 32 x TY       buoyancy at z+1
    static constexpr int OV = LB + al128(W32 * TY * 4);            // 3 x 32 x TY   own vx, vy, vz at z
    static constexpr int STAGE = OV + 3 * al128(W32 * TY * ES);
    static constexpr uint32_t TXB = ES * (2 * W48 * TY + 2 * W32 * (TY + 10) + W48 * (TY + 10) + 6 * W32 * TY) +
                                    4 * (W36 * (TY + 1) + W32 * TY);
    static_assert(W48 * TY * ES % 128 == 0 && W32 * (TY + 10) * ES % 128 == 0 && W32 * TY * ES % 128 == 0,
                  "arrays of one copy must be contiguous and 128-byte aligned");
};
// Shared-memory stage layout of the stress update (ES as above; the medium
// boxes FP32).
template <int TY, int ES = 4>
struct StrL {
    static constexpr int VX = 0;                                   // 48 x (TY+10)  vx (x, y halo)
    static constexpr int VY = VX + W48 * (TY + 10) * ES;           // 48 x (TY+10)  vy
    static constexpr int VZ = VY + W48 * (TY + 10) * ES;           // 48 x (TY+10)  vz
    static constexpr int LX = al128(VZ + W48 * (TY + 10) * ES);    // 32 x TY       vx at z+5
    static constexpr int LY = LX + W32 * TY * ES;                  // 32 x TY       vy at z+5
    static constexpr int LZ = LY + al128(W32 * TY * ES);           // 32 x TY       vz at z+4
    // own-cell data at z, 32 x TY each: txx tyy tzz txy txz tyz, then the
    // medium: lambda, mu, the shear moduli of txy, txz, tyz
    static constexpr int OWN = LZ + al128(W32 * TY * ES);
    static constexpr int MED = OWN + 6 * W32 * TY * ES;
    static constexpr int STAGE = MED + 5 * W32 * TY * 4;
    static constexpr uint32_t TXB = ES * (3 * W48 * (TY + 10) + 9 * W32 * TY) + 4 * 5 * W32 * TY;
    static_assert(W32 * TY * ES % 128 == 0 && (ES == 2 || W48 * (TY + 10) * ES % 128 == 0),
                  "arrays of one copy must be contiguous and 128-byte aligned");
};

struct Tile {
    int cx0, cy0;    // computed coordinates of the tile origin
    int xd;          // device x of the tile origin (128-byte aligned)
    int gx0, gy0;    // GRID coordinates of the tile origin
    int zs, ze;      // computed z range of this CTA
    bool xy_pml;     // the tile touches the x or y PML band
};

template <int TY>
__device__ __forceinline__ Tile make_tile(const Model &m, const ZGeom &g, int tile, int chunk) {
    Tile t;
    t.cx0 = (tile % g.ntx) * TX;
    t.cy0 = (tile / g.ntx) * TY;
    t.gx0 = t.cx0 + kHalo;
    t.gy0 = t.cy0 + kHalo;
    t.xd = t.gx0 + kXOff;
    t.zs = chunk * g.zc;
    t.ze = min(t.zs + g.zc, m.nzc);
    t.xy_pml = t.cx0 < m.pml || t.cx0 + TX > m.nxc - m.pml || t.cy0 < m.pml || t.cy0 + TY > m.nyc - m.pml;
    return t;
}

// ---------------------------------------------------------------------------
// velocity update
// ---------------------------------------------------------------------------

constexpr int kWarps = NT / 32;

// One TMA box of a stage: 4-D tensor map (its first array at w = 0),
// destination offset in the stage, x and y of its origin and its plane
// relative to the staged plane.  Each warp's boxes are worked out once per
// CTA and kept in shared memory, so that the per-plane issue is a few loads
// and the copies themselves.
struct TmaBox {
    const CUtensorMap *map;
    uint32_t off;
    int x, y, dz;
};
constexpr int kMaxBoxesPerWarp = 3;

__device__ __forceinline__ void issue_boxes(const TmaBox *b, int n, unsigned char *st, uint64_t *bar, int gz) {
    for (int j = 0; j < n; ++j) tma4(st + b[j].off, b[j].map, b[j].x, b[j].y, gz + b[j].dz, 0, bar);
}
constexpr int kVelBoxes = 8;
constexpr int kStrBoxes = 4;      // FP32: the 11 own-cell arrays in one copy
constexpr int kStrBoxes16 = 5;    // 16-bit storage: the 6 stresses and the FP32 medium separately

// 16-bit storage: n stored values of field box `src` (stage) as FP32 values
// float(h) * sc in `dst` (the work buffer, laid out as an FP32 stage) — the
// read-back of every tap, done once per staged value.
template <int ST, int N>
__device__ __forceinline__ void widen(const unsigned char *src, unsigned char *dst, float sc) {
    static_assert(N % 2 == 0, "pairs of values");
    const uint32_t *s2 = reinterpret_cast<const uint32_t *>(src);
    float2 *d2 = reinterpret_cast<float2 *>(dst);
#pragma unroll
    for (int i = threadIdx.x; i < N / 2; i += NT) {
        const uint32_t u = s2[i];
        d2[i] = make_float2(H16<ST>::h2f(u & 0xffffu) * sc, H16<ST>::h2f(u >> 16) * sc);
    }
}

// Box q of the velocity stage (ES: bytes per stored wavefield value).
template <int TY, int ES>
__device__ __forceinline__ TmaBox vel_box(const ZMaps &mp, const Tile &t, int q) {
    using L = VelL<TY, ES>;
    switch (q) {
    case 0: return {&mp.v_sxx_sxz, L::SXX, t.xd - 8, t.gy0, 0};
    case 1: return {&mp.v_syy_syz, L::SYY, t.xd, t.gy0 - 5, 0};
    case 2: return {&mp.v_sxy, L::SXY, t.xd - 8, t.gy0 - 5, 0};
    case 3: return {&mp.v_b, L::B, t.xd, t.gy0, 0};
    case 4: return {&mp.v_lead_xz_yz, L::LXZ, t.xd, t.gy0, 4};
    case 5: return {&mp.v_lead_zz, L::LZZ, t.xd, t.gy0, 5};
    case 6: return {&mp.v_lead_b, L::LB, t.xd, t.gy0, 1};
    default: return {&mp.v_own, L::OV, t.xd, t.gy0, 0};
    }
}

// Stage the velocity inputs of computed plane cz from this warp's boxes
// (boxes w, w + 8, ... of the stage for warp w; called by lane 0 of every
// warp).  Thread 0 also arms the stage's barrier with all of the stage's
// bytes; the barrier's phase cannot complete before that arrival, whichever
// copy lands first.
template <int TY, int ES>
__device__ __forceinline__ void vel_issue(const TmaBox *b, int n, unsigned char *st, uint64_t *bar, int cz, int warp) {
    if (warp == 0) mbar_expect_tx(bar, VelL<TY, ES>::TXB);
    issue_boxes(b, n, st, bar, cz + kHalo);
}

// The velocity update of one work item: the tile `tile` (x fastest) over z
// chunk `chunk`.  smem: the stage ring; bar: its S initialised mbarriers,
// whose phase parities pbits carries from item to item (bit s: the parity
// the next wait on stage s expects); boxes: per-warp TMA box scratch.
// Returns false after a bounded wait gave up (g.err set, copies drained).
// MANY: the CTA runs several items (persistent batch); a single-item launch
// keeps one parity for the whole ring and skips the fences a previous item needs.
// ST: wavefield storage.  16-bit storage (32 x 8 tiles): the copies bring
// 16-bit field boxes, which each plane widens once into an FP32 work buffer
// after the ring (float(h) * 2^e, the read-back of kernels_half.cu and the
// oracle) for the unchanged FP32 arithmetic; stores round to 16 bits; the
// source and the receivers run as the 16-bit family's own kernels.
template <bool FAST, int CELLS, bool MANY, int ST = SGFD_STORE_F32>
__device__ __forceinline__ bool vel_item(const ZMaps &mp, const Model &m, const Physics &ph, const ZGeom &g,
                                         const SourceRec &sr, int it_arg, float src_value, int use_wavelet, int tile,
                                         int chunk, unsigned char *smem, uint64_t *bar,
                                         TmaBox (*boxes)[kMaxBoxesPerWarp], uint32_t &pbits,
                                         const HalfState &hs = HalfState{}) {
    constexpr int TY = 8 * CELLS;
    constexpr bool H = ST != SGFD_STORE_F32;
    static_assert(!H || CELLS == 1, "16-bit storage runs on 32 x 8 tiles");
    constexpr int ES = H ? 2 : 4;
    using L = VelL<TY>;          // FP32 layout: the stage itself, or the 16-bit storage's work buffer
    using LS = VelL<TY, ES>;     // the stage as the copies fill it
    __shared__ float scl[18];    // 16-bit storage: this step's scales 2^e, then 2^-e
    __shared__ unsigned smax[9]; // 16-bit storage, rescale steps: this CTA's largest written magnitudes
    if constexpr (H) {
        if (threadIdx.x < 9) {
            scl[threadIdx.x] = hs.sc[threadIdx.x];
            scl[9 + threadIdx.x] = hs.inv[threadIdx.x];
            smax[threadIdx.x] = 0u;
        }
        __syncthreads();
    }
    unsigned char *work = smem + S * LS::STAGE;   // 16-bit storage only
    // stored value k of field (or split group) g, read back as FP32
    auto ld = [&](auto *p, int g) -> float {
        if constexpr (H) return H16<ST>::h2f(*p) * scl[g];
        else return *p;
    };
    auto put = [&](auto *p, int g, float v) {
        if constexpr (H) *p = (uint16_t)H16<ST>::f2h(v * scl[9 + g]);
        else *p = v;
    };
    const Tile t = make_tile<TY>(m, g, tile, chunk);
    const int tid = threadIdx.x, lx = tid & 31, ty = tid >> 5;
    const int warp = tid >> 5;
    const TmaBox *mybox = boxes[warp];
    const int nbox = (kVelBoxes - warp + kWarps - 1) / kWarps;
    if (lx == 0) {
        for (int j = 0; j < nbox; ++j) boxes[warp][j] = vel_box<TY, ES>(mp, t, warp + j * kWarps);
        if (MANY) fence_proxy_async();   // a previous item's stages were read through the generic proxy
        for (int s = 0; s < S && t.zs + s < t.ze; ++s)
            vel_issue<TY, ES>(mybox, nbox, smem + s * LS::STAGE, &bar[s], t.zs + s, warp);
    }
    int issued_end = min(t.zs + S, t.ze);   // planes [zs, issued_end) issued
    int stage = 0;                          // stage of plane cz
    uint32_t parity = 0;                    // single item: the parity of every stage's next wait

    const int it = step_index(sr, it_arg);
    const float inj = ph.inj_dt2 * ((use_wavelet && sr.wavelet) ? sr.wavelet[it] : src_value);
    [[maybe_unused]] const bool track = H && rescale_step16(it);   // 16-bit: note the written maxima
    int sx = -1, sy = -1, sz = -1;
    if (!H && sr.src >= 0) {
        const int64_t r = sr.src;
        sz = (int)(r / m.plane);
        sy = (int)((r - (int64_t)sz * m.plane) / m.px);
        sx = (int)(r - (int64_t)sz * m.plane - (int64_t)sy * m.px);
    }
    [[maybe_unused]] auto fld = [&](int k) {
        if constexpr (H) return hs.f[k];
        else return m.f[k];
    };
    [[maybe_unused]] auto spl = [&]() {
        if constexpr (H) return hs.split;
        else return m.split;
    };

    const int gx = t.gx0 + lx;
    const int kx = band(gx, m.nx, m.pml);
    int lyc[CELLS], gyc[CELLS], kyc[CELLS];
    bool act[CELLS];
    uint32_t col[CELLS];          // element offset of the thread's column at z = 0
    PmlColumn pcol[CELLS];
    const uint32_t PL = (uint32_t)m.plane;
#pragma unroll
    for (int c = 0; c < CELLS; ++c) {
        lyc[c] = CELLS * ty + c;   // a thread's cells are vertically adjacent
        gyc[c] = t.gy0 + lyc[c];
        act[c] = (t.cx0 + lx < m.nxc) && (t.cy0 + lyc[c] < m.nyc);
        kyc[c] = band(gyc[c], m.ny, m.pml);
        // inactive threads of edge tiles address a valid cell (results discarded)
        col[c] = (uint32_t)pidx(m, min(gx, m.nx - 1), min(gyc[c], m.ny - 1), 0);
        pcol[c] = pml_column(m, min(t.cx0 + lx, m.nxc - 1), min(t.cy0 + lyc[c], m.nyc - 1));
    }

    // z queues: qxz, qyz hold z-5..z+4, qzz holds z-4..z+5 (filled 9 deep here)
    float qxz[CELLS][10], qyz[CELLS][10], qzz[CELLS][10];
    const int gz0 = t.zs + kHalo;
#pragma unroll
    for (int c = 0; c < CELLS; ++c) {
#pragma unroll
        for (int k = 0; k < 9; ++k) {
            qxz[c][k + 1] = ld(fld(7) + col[c] + (uint32_t)(gz0 - 5 + k) * PL, 7);
            qyz[c][k + 1] = ld(fld(8) + col[c] + (uint32_t)(gz0 - 5 + k) * PL, 8);
            float zz = ld(fld(5) + col[c] + (uint32_t)(gz0 - 4 + k) * PL, 5);
            if (gx == sx && gyc[c] == sy && gz0 - 4 + k == sz) zz = zz + inj;
            qzz[c][k + 1] = zz;
        }
    }

    // receivers of this tile, sorted by z: skip those below the chunk
    int rp = H ? 0 : g.rec_off[tile];
    const int rend = H ? 0 : g.rec_off[tile + 1];
    while (rp < rend && g.rec_list[rp].z < gz0) ++rp;
    int rz = rp < rend ? g.rec_list[rp].z : 0x7fffffff;   // z of the next receiver

    bool failed = false, abort = false;
    int cz = t.zs;
    const bool src_near = !H && sr.src >= 0 && sy >= t.gy0 - 5 && sy < t.gy0 + TY + 5 && sx >= t.gx0 - 8 &&
                          sx < t.gx0 + TX + 8;
    // One plane.  GEN selects the general path (PML cells, source, receivers);
    // the interior-only path is used for every other tile-plane.  Returns
    // false when the block votes to abort.
    auto plane = [&](auto gen_tag) -> bool {
        constexpr bool GEN = decltype(gen_tag)::value;
        const int s = stage;
        unsigned char *st = smem + s * LS::STAGE;
        const int gz = cz + kHalo;
        const int kz = bandz(m, gz);
        const bool plane_pml = GEN && (t.xy_pml || kz != 0);


        // PML cells: splits and the medium of the damping, loaded before the
        // stage wait so that their latency overlaps the wait and the stencil
        float opre[CELLS][9], mupre[CELLS], lampre[CELLS];
        if (plane_pml) {
#pragma unroll
            for (int c = 0; c < CELLS; ++c) {
                if (act[c] && (kx | kyc[c] | kz)) {
                    const uint32_t ci = col[c] + (uint32_t)gz * PL;
                    const auto *sp = spl() + split_base32(pml_plane_index(m, pcol[c], cz));
#pragma unroll
                    for (int q = 0; q < 9; ++q) opre[c][q] = ld(sp + q * kSplitBlock, q / 3);   // split q: field q / 3
                    mupre[c] = m.mu[ci];
                    lampre[c] = ph.damping == 1 ? m.lam[ci] : 0.f;
                }
            }
        }

        if (!mbar_wait(&bar[s], MANY ? (pbits >> s) & 1u : parity)) failed = true;
        // the FP32 view of the stage's wavefield boxes
        const unsigned char *wk = st;
        if constexpr (H) {
            widen<ST, W48 * TY>(st + LS::SXX, work + L::SXX, scl[3]);
            widen<ST, W48 * TY>(st + LS::SXZ, work + L::SXZ, scl[7]);
            widen<ST, W32 * (TY + 10)>(st + LS::SYY, work + L::SYY, scl[4]);
            widen<ST, W32 * (TY + 10)>(st + LS::SYZ, work + L::SYZ, scl[8]);
            widen<ST, W48 * (TY + 10)>(st + LS::SXY, work + L::SXY, scl[6]);
            widen<ST, W32 * TY>(st + LS::LXZ, work + L::LXZ, scl[7]);
            widen<ST, W32 * TY>(st + LS::LYZ, work + L::LYZ, scl[8]);
            widen<ST, W32 * TY>(st + LS::LZZ, work + L::LZZ, scl[5]);
#pragma unroll
            for (int q = 0; q < 3; ++q)
                widen<ST, W32 * TY>(st + LS::OV + q * al128(W32 * TY * ES), work + L::OV + q * al128(W32 * TY * 4),
                                    scl[q]);
            __syncthreads();
            wk = work;
        }

        // source patch of the staged copies (uniform branch)
        if (GEN && src_near && (gz == sz || gz + 5 == sz)) {
            if (tid == 0) {
                const int ox = sx - t.gx0, oy = sy - t.gy0;
                if (gz == sz) {
                    float *sxx = reinterpret_cast<float *>(st + L::SXX);
                    float *syy = reinterpret_cast<float *>(st + L::SYY);
                    if (oy >= 0 && oy < TY && ox + 8 >= 0 && ox + 8 < W48) sxx[oy * W48 + ox + 8] += inj;
                    if (oy + 5 >= 0 && oy + 5 < TY + 10 && ox >= 0 && ox < W32) syy[(oy + 5) * W32 + ox] += inj;
                }
                if (gz + 5 == sz) {
                    float *szz = reinterpret_cast<float *>(st + L::LZZ);
                    if (oy >= 0 && oy < TY && ox >= 0 && ox < W32) szz[oy * W32 + ox] += inj;
                }
            }
            __syncthreads();
        }

        const float *sxx = reinterpret_cast<const float *>(wk + L::SXX);
        const float *syy = reinterpret_cast<const float *>(wk + L::SYY);
        const float *sxy = reinterpret_cast<const float *>(wk + L::SXY);
        const float *sxz = reinterpret_cast<const float *>(wk + L::SXZ);
        const float *syz = reinterpret_cast<const float *>(wk + L::SYZ);
        const float *bb = reinterpret_cast<const float *>(st + LS::B);
        const float *lxz = reinterpret_cast<const float *>(wk + L::LXZ);
        const float *lyz = reinterpret_cast<const float *>(wk + L::LYZ);
        const float *lzz = reinterpret_cast<const float *>(wk + L::LZZ);
        const float *lb = reinterpret_cast<const float *>(st + LS::LB);
        const float *ov = reinterpret_cast<const float *>(wk + L::OV);
        constexpr int OVS = al128(W32 * TY * 4) / 4;   // floats between the own-velocity boxes

        // y differences of vertically adjacent cells share their windows
        [[maybe_unused]] float xY2[2] = {0.f, 0.f}, yY2[2] = {0.f, 0.f}, zY2[2] = {0.f, 0.f};
        if constexpr (CELLS == 2) {
            const float *cxy0 = sxy + (lyc[0] + 5) * W48 + lx + 8;
            const float *cyy0 = syy + (lyc[0] + 5) * W32 + lx;
            const float *cyz0 = syz + (lyc[0] + 5) * W32 + lx;
            dB2<FAST, 1>(ph, [&](int o) { return cxy0[o * W48]; }, xY2[0], xY2[1]);
            dF2<FAST, 1>(ph, [&](int o) { return cyy0[o * W32]; }, yY2[0], yY2[1]);
            dB2<FAST, 1>(ph, [&](int o) { return cyz0[o * W32]; }, zY2[0], zY2[1]);
        }
#pragma unroll
        for (int c = 0; c < CELLS; ++c) {
            const int ly = lyc[c];
            // advance the z queues
#pragma unroll
            for (int j = 0; j < 9; ++j) {
                qxz[c][j] = qxz[c][j + 1];
                qyz[c][j] = qyz[c][j + 1];
                qzz[c][j] = qzz[c][j + 1];
            }
            qxz[c][9] = lxz[ly * W32 + lx];
            qyz[c][9] = lyz[ly * W32 + lx];
            qzz[c][9] = lzz[ly * W32 + lx];
            if (!act[c]) continue;

            const float *rxx = sxx + ly * W48 + lx + 8;
            const float *cxy = sxy + (ly + 5) * W48 + lx + 8;
            const float *rxz = sxz + ly * W48 + lx + 8;
            const float *cyy = syy + (ly + 5) * W32 + lx;
            const float *cyz = syz + (ly + 5) * W32 + lx;
            float xX, xY, xZ, yX, yY, yZ, zX, zY, zZ;
            if constexpr (CELLS == 1) {
                // eight of the nine differences in pairs on FP32x2, same roundings
                // (REF: sums with the plain coefficients, then the divisions)
                const float2 yzX = dpair(FAST ? ph.cp[0] : ph.cr, [&](int i) { return make_float2(cxy[i], rxz[i]); },
                                         [&](int i) { return make_float2(cxy[-1 - i], rxz[-1 - i]); });
                const float2 xzY = dpair(FAST ? ph.cp[1] : ph.cr,
                                         [&](int i) { return make_float2(cxy[i * W48], cyz[i * W32]); },
                                         [&](int i) { return make_float2(cxy[(-1 - i) * W48], cyz[(-1 - i) * W32]); });
                const float2 xyZ = dpair(FAST ? ph.cp[2] : ph.cr,
                                         [&](int i) { return make_float2(qxz[c][5 + i], qyz[c][5 + i]); },
                                         [&](int i) { return make_float2(qxz[c][4 - i], qyz[c][4 - i]); });
                const float2 xXyY = dpair(FAST ? ph.cp[3] : ph.cr,
                                          [&](int i) { return make_float2(rxx[1 + i], cyy[(1 + i) * W32]); },
                                          [&](int i) { return make_float2(rxx[-i], cyy[-i * W32]); });
                xX = by_cell<FAST>(ph, 0, xXyY.x); yY = by_cell<FAST>(ph, 1, xXyY.y);
                yX = by_cell<FAST>(ph, 0, yzX.x); zX = by_cell<FAST>(ph, 0, yzX.y);
                xY = by_cell<FAST>(ph, 1, xzY.x); zY = by_cell<FAST>(ph, 1, xzY.y);
                xZ = by_cell<FAST>(ph, 2, xyZ.x); yZ = by_cell<FAST>(ph, 2, xyZ.y);
            } else {
                xX = dF<FAST, 0>(ph, [&](int o) { return rxx[o]; });
                xY = CELLS == 2 ? xY2[c] : dB<FAST, 1>(ph, [&](int o) { return cxy[o * W48]; });
                xZ = dB<FAST, 2>(ph, [&](int o) { return qxz[c][5 + o]; });
                yX = dB<FAST, 0>(ph, [&](int o) { return cxy[o]; });
                yY = CELLS == 2 ? yY2[c] : dF<FAST, 1>(ph, [&](int o) { return cyy[o * W32]; });
                yZ = dB<FAST, 2>(ph, [&](int o) { return qyz[c][5 + o]; });
                zX = dB<FAST, 0>(ph, [&](int o) { return rxz[o]; });
                zY = CELLS == 2 ? zY2[c] : dB<FAST, 1>(ph, [&](int o) { return cyz[o * W32]; });
            }
            zZ = dF<FAST, 2>(ph, [&](int o) { return qzz[c][4 + o]; });
            const float b0 = bb[ly * W36 + lx];
            const float bx = (b0 + bb[ly * W36 + lx + 1]) / 2.0f;
            const float by = (b0 + bb[(ly + 1) * W36 + lx]) / 2.0f;
            const float bz = (b0 + lb[ly * W32 + lx]) / 2.0f;

            const uint32_t ci = col[c] + (uint32_t)gz * PL;
            float vnew[3];
            const int ky = kyc[c];
            if (!(plane_pml && (kx | ky | kz))) {
                const int e = ly * W32 + lx;
                vnew[0] = __fmaf_rn(ph.dt * bx, (xX + xY) + xZ, ov[e]);
                vnew[1] = __fmaf_rn(ph.dt * by, (yX + yY) + yZ, ov[OVS + e]);
                vnew[2] = __fmaf_rn(ph.dt * bz, (zX + zY) + zZ, ov[2 * OVS + e]);
            } else {
                float mx = 1.f, my = 1.f, mz = 1.f;
        PDiv<FAST> px = 1, py = 1, pz = 1;
                {
                    const float v = damp_speed(ph, mupre[c], b0, lampre[c]);
                    if (kx) damp_factors<FAST>(ph, 0, ph.dx, kx, m.pml, v, mx, px);
                    if (ky) damp_factors<FAST>(ph, 1, ph.dy, ky, m.pml, v, my, py);
                    if (kz) damp_factors<FAST>(ph, 2, ph.dz, kz, m.pml, v, mz, pz);
                }
                const bool ref = ph.quirks == 0;
                const float ax = ph.dt * bx, ay = ph.dt * (ref ? bx : by), az = ph.dt * (ref ? bx : bz);
                auto *sp = spl() + split_base32(pml_plane_index(m, pcol[c], cz));
                constexpr uint32_t N = kSplitBlock;   // split k at sp[k * N]
                const float *o = opre[c];
                // split k belongs to field k / 3 (its scale with 16-bit storage)
                auto sput = [&](int k, float v) {
                    if constexpr (H) {
                        if (track) note_max16s(smax, k / 3, v);
                    }
                    put(sp + k * N, k / 3, v);
                };
                float a0, a1, a2;
                a0 = split_update<FAST>(o[S_VXX], ax, xX, kx, mx, px);
                a1 = split_update<FAST>(o[S_VXY], ax, xY, ky, my, py);
                a2 = split_update<FAST>(o[S_VXZ], ax, xZ, kz, mz, pz);
                sput(S_VXX, a0); sput(S_VXY, a1); sput(S_VXZ, a2);
                vnew[0] = (a0 + a1) + a2;
                a0 = split_update<FAST>(o[S_VYX], ay, yX, kx, mx, px);
                a1 = split_update<FAST>(o[S_VYY], ay, yY, ky, my, py);
                a2 = split_update<FAST>(o[S_VYZ], ay, yZ, kz, mz, pz);
                sput(S_VYX, a0); sput(S_VYY, a1); sput(S_VYZ, a2);
                vnew[1] = (a0 + a1) + a2;
                a0 = split_update<FAST>(o[S_VZX], az, zX, kx, mx, px);
                a1 = split_update<FAST>(o[S_VZY], az, zY, ky, my, py);
                a2 = split_update<FAST>(o[S_VZZ], az, zZ, kz, mz, pz);
                sput(S_VZX, a0); sput(S_VZY, a1); sput(S_VZZ, a2);
                vnew[2] = (a0 + a1) + a2;
            }
            if constexpr (H) {
                if (track) {
                    note_max16s(smax, 0, vnew[0]);
                    note_max16s(smax, 1, vnew[1]);
                    note_max16s(smax, 2, vnew[2]);
                }
            }
            put(fld(0) + ci, 0, vnew[0]);
            put(fld(1) + ci, 1, vnew[1]);
            put(fld(2) + ci, 2, vnew[2]);
            // receivers of velocity components at this cell (list sorted by z)
            if (GEN && !H && gz == rz && it >= 0 && it < sr.nt) {
                for (int r = rp; r < rend && g.rec_list[r].z == gz; ++r) {
                    const int4 q = g.rec_list[r];
                    if (q.x == gx && q.y == gyc[c] && q.w <= 2)
                        sr.traces[(int64_t)it * sr.nrec + g.rec_idx[r]] =
                            q.w == 0 ? vnew[0] : q.w == 1 ? vnew[1] : vnew[2];
                }
            }
        }
        if (GEN && gz == rz) {
            while (rp < rend && g.rec_list[rp].z == gz) ++rp;
            rz = rp < rend ? g.rec_list[rp].z : 0x7fffffff;
        }

        // every thread is done with this stage: vote on aborts, then refill it
        if (__syncthreads_or(failed)) return false;
        if (cz + S < t.ze) {
            if (lx == 0) {
                fence_proxy_async();
                vel_issue<TY, ES>(mybox, nbox, st, &bar[s], cz + S, warp);
            }
            issued_end = cz + S + 1;
        }
        if (MANY) pbits ^= 1u << s;
        if (++stage == S) {
            stage = 0;
            if (!MANY) parity ^= 1u;
        }
        return true;
    };
    for (; cz < t.ze; ++cz) {
        const int gzp = cz + kHalo;
        const bool gen = t.xy_pml || bandz(m, gzp) != 0 || (src_near && (gzp == sz || gzp + 5 == sz)) || gzp == rz;
        if (!(gen ? plane(std::true_type{}) : plane(std::false_type{}))) {
            abort = true;
            break;
        }
    }
    if (abort && tid == 0) {
        atomicExch(g.err, 1);
        if (MANY) drain_bits<S>(bar, issued_end, cz, t.zs, pbits);
        else drain<S>(bar, issued_end, cz, t.zs);
    }
    if constexpr (H) {
        if (track) {
            __syncthreads();
            flush_max16(hs, smax);
        }
    }
    return !abort;
}

template <bool FAST, int CELLS>
__global__ void __launch_bounds__(NT, 3)
k_velocity_zmarch(const __grid_constant__ ZMaps mp, const __grid_constant__ Model m, const __grid_constant__ Physics ph,
                  const __grid_constant__ ZGeom g, const __grid_constant__ SourceRec sr, int it_arg,
                  float src_value, int use_wavelet) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    __shared__ __align__(8) uint64_t bar[S];
    __shared__ TmaBox boxes[kWarps][kMaxBoxesPerWarp];
    if (threadIdx.x == 0) {
        for (int s = 0; s < S; ++s) mbar_init(&bar[s], 1);
        fence_barrier_init();
    }
    __syncthreads();
    uint32_t pbits = 0;
    vel_item<FAST, CELLS, false>(mp, m, ph, g, sr, it_arg, src_value, use_wavelet, blockIdx.x, blockIdx.y + g.c0,
                          align_smem(smem_raw), bar, boxes, pbits);
}

// ---------------------------------------------------------------------------
// stress update
// ---------------------------------------------------------------------------

// Box q of the stress stage (ES as vel_box; FP32: the 11 own-cell arrays
// in one copy, 16-bit: the 6 stored stresses, then the FP32 medium).
template <int TY, int ES>
__device__ __forceinline__ TmaBox str_box(const ZMaps &mp, const Tile &t, int q) {
    using L = StrL<TY, ES>;
    switch (q) {
    case 0: return {&mp.s_v, L::VX, t.xd - 8, t.gy0 - 5, 0};
    case 1: return {&mp.s_lead_xy, L::LX, t.xd, t.gy0, 5};
    case 2: return {&mp.s_lead_z, L::LZ, t.xd, t.gy0, 4};
    case 3: return {&mp.s_own, L::OWN, t.xd, t.gy0, 0};
    default: return {&mp.s_med, L::MED, t.xd, t.gy0, 0};
    }
}

// Stage the stress inputs of computed plane cz, as vel_issue.
template <int TY, int ES>
__device__ __forceinline__ void str_issue(const TmaBox *b, int n, unsigned char *st, uint64_t *bar, int cz, int warp) {
    if (warp == 0) mbar_expect_tx(bar, StrL<TY, ES>::TXB);
    issue_boxes(b, n, st, bar, cz + kHalo);
}

// The stress update of one work item, as vel_item (ST: storage, as there).
template <bool FAST, int CELLS, bool MANY, int ST = SGFD_STORE_F32>
__device__ __forceinline__ bool str_item(const ZMaps &mp, const Model &m, const Physics &ph, const ZGeom &g,
                                         const SourceRec &sr, int it_arg, float src_value, int use_wavelet, int tile,
                                         int chunk, unsigned char *smem, uint64_t *bar,
                                         TmaBox (*boxes)[kMaxBoxesPerWarp], uint32_t &pbits,
                                         const HalfState &hs = HalfState{}) {
    constexpr int TY = 8 * CELLS;
    constexpr bool H = ST != SGFD_STORE_F32;
    static_assert(!H || CELLS == 1, "16-bit storage runs on 32 x 8 tiles");
    constexpr int ES = H ? 2 : 4;
    using L = StrL<TY>;          // FP32 layout: the stage itself, or the 16-bit storage's work buffer
    using LS = StrL<TY, ES>;     // the stage as the copies fill it
    __shared__ float scl[18];    // 16-bit storage: this step's scales 2^e, then 2^-e
    __shared__ unsigned smax[9]; // 16-bit storage, rescale steps: this CTA's largest written magnitudes
    if constexpr (H) {
        if (threadIdx.x < 9) {
            scl[threadIdx.x] = hs.sc[threadIdx.x];
            scl[9 + threadIdx.x] = hs.inv[threadIdx.x];
            smax[threadIdx.x] = 0u;
        }
        __syncthreads();
    }
    unsigned char *work = smem + S * LS::STAGE;   // 16-bit storage only
    auto ld = [&](auto *p, int g) -> float {
        if constexpr (H) return H16<ST>::h2f(*p) * scl[g];
        else return *p;
    };
    auto put = [&](auto *p, int g, float v) {
        if constexpr (H) *p = (uint16_t)H16<ST>::f2h(v * scl[9 + g]);
        else *p = v;
    };
    [[maybe_unused]] auto fld = [&](int k) {
        if constexpr (H) return hs.f[k];
        else return m.f[k];
    };
    [[maybe_unused]] auto spl = [&]() {
        if constexpr (H) return hs.split;
        else return m.split;
    };
    const Tile t = make_tile<TY>(m, g, tile, chunk);
    const int tid = threadIdx.x, lx = tid & 31, ty = tid >> 5;
    const int warp = tid >> 5;
    const TmaBox *mybox = boxes[warp];
    constexpr int NB = H ? kStrBoxes16 : kStrBoxes;
    const int nbox = (NB - warp + kWarps - 1) / kWarps;
    if (lx == 0) {
        for (int j = 0; j < nbox; ++j) boxes[warp][j] = str_box<TY, ES>(mp, t, warp + j * kWarps);
        if (MANY) fence_proxy_async();   // a previous item's stages were read through the generic proxy
        for (int s = 0; s < S && t.zs + s < t.ze; ++s)
            str_issue<TY, ES>(mybox, nbox, smem + s * LS::STAGE, &bar[s], t.zs + s, warp);
    }
    int issued_end = min(t.zs + S, t.ze);   // planes [zs, issued_end) issued
    int stage = 0;                          // stage of plane cz
    uint32_t parity = 0;                    // single item: the parity of every stage's next wait

    const int it = step_index(sr, it_arg);
    const float inj = ph.inj_dt2 * ((use_wavelet && sr.wavelet) ? sr.wavelet[it] : src_value);
    [[maybe_unused]] const bool track = H && rescale_step16(it);   // 16-bit: note the written maxima
    const int64_t src = H ? -1 : sr.src;

    const int gx = t.gx0 + lx;
    const int kx = band(gx, m.nx, m.pml);
    int lyc[CELLS], gyc[CELLS], kyc[CELLS];
    bool act[CELLS];
    uint32_t col[CELLS];          // element offset of the thread's column at z = 0
    PmlColumn pcol[CELLS];
    const uint32_t PL = (uint32_t)m.plane;
#pragma unroll
    for (int c = 0; c < CELLS; ++c) {
        lyc[c] = CELLS * ty + c;   // a thread's cells are vertically adjacent
        gyc[c] = t.gy0 + lyc[c];
        act[c] = (t.cx0 + lx < m.nxc) && (t.cy0 + lyc[c] < m.nyc);
        kyc[c] = band(gyc[c], m.ny, m.pml);
        // inactive threads of edge tiles address a valid cell (results discarded)
        col[c] = (uint32_t)pidx(m, min(gx, m.nx - 1), min(gyc[c], m.ny - 1), 0);
        pcol[c] = pml_column(m, min(t.cx0 + lx, m.nxc - 1), min(t.cy0 + lyc[c], m.nyc - 1));
    }

    // z queues, 11 deep, planes in pairs as in the velocity update: before the
    // first plane of a pair at z, qx and qy (vx, vy) hold z-4..z+4 and qz (vz)
    // z-5..z+3 in slots 0..8
    float qx[CELLS][11], qy[CELLS][11], qz[CELLS][11];
    const int gz0 = t.zs + kHalo;
#pragma unroll
    for (int c = 0; c < CELLS; ++c) {
#pragma unroll
        for (int k = 0; k < 9; ++k) {
            qx[c][k] = ld(fld(0) + col[c] + (uint32_t)(gz0 - 4 + k) * PL, 0);
            qy[c][k] = ld(fld(1) + col[c] + (uint32_t)(gz0 - 4 + k) * PL, 1);
            qz[c][k] = ld(fld(2) + col[c] + (uint32_t)(gz0 - 5 + k) * PL, 2);
        }
    }

    int rp = H ? 0 : g.rec_off[tile];
    const int rend = H ? 0 : g.rec_off[tile + 1];
    while (rp < rend && g.rec_list[rp].z < gz0) ++rp;
    int rz = rp < rend ? g.rec_list[rp].z : 0x7fffffff;

    bool failed = false, abort = false;
    int cz = t.zs;
    int sz = -1;
    if (src >= 0) sz = (int)(src / m.plane);
    // The PML cells' splits and buoyancy, loaded by plain loads after the
    // stencil, are brought into L2 one plane ahead, while the plane before
    // them is computed (32 x 8 tiles: a warp's cells are one row): their
    // loads then wait on L2 rather than on HBM.  Two and three planes ahead
    // measured slower.
    auto prefetch = [&](int pz) {
        if constexpr (CELLS == 1) {
            if (pz >= t.ze) return;
            const int kzp = bandz(m, pz + kHalo);
            if (!t.xy_pml && kzp == 0) return;
            const bool p = act[0] && (kx | kyc[0] | kzp);
            if (prefetch_split_rows(spl(), p, pml_plane_index(m, pcol[0], pz), S_XXX, kNumSplit, lx) && lx == 0)
                l2_prefetch(m.b + col[0] + (uint32_t)(pz + kHalo) * PL, TX * 4);
        }
    };
    prefetch(t.zs);

    // One plane, as in the velocity update (GEN: general path; P: place in
    // the pair).  Returns false when the block votes to abort.
    auto plane = [&](auto gen_tag, auto p_tag) -> bool {
        constexpr bool GEN = decltype(gen_tag)::value;
        constexpr int P = decltype(p_tag)::value;
        const int s = stage;
        unsigned char *st = smem + s * LS::STAGE;
        const int gz = cz + kHalo;
        const int kz = bandz(m, gz);
        const bool plane_pml = GEN && (t.xy_pml || kz != 0);

        if (!mbar_wait(&bar[s], MANY ? (pbits >> s) & 1u : parity)) failed = true;
        // the FP32 view of the stage's wavefield boxes
        const unsigned char *wk = st;
        if constexpr (H) {
            widen<ST, W48 * (TY + 10)>(st + LS::VX, work + L::VX, scl[0]);
            widen<ST, W48 * (TY + 10)>(st + LS::VY, work + L::VY, scl[1]);
            widen<ST, W48 * (TY + 10)>(st + LS::VZ, work + L::VZ, scl[2]);
            widen<ST, W32 * TY>(st + LS::LX, work + L::LX, scl[0]);
            widen<ST, W32 * TY>(st + LS::LY, work + L::LY, scl[1]);
            widen<ST, W32 * TY>(st + LS::LZ, work + L::LZ, scl[2]);
#pragma unroll
            for (int q = 0; q < 6; ++q)
                widen<ST, W32 * TY>(st + LS::OWN + q * W32 * TY * ES, work + L::OWN + q * W32 * TY * 4, scl[3 + q]);
            __syncthreads();
            wk = work;
        }

        const float *svx = reinterpret_cast<const float *>(wk + L::VX);
        const float *svy = reinterpret_cast<const float *>(wk + L::VY);
        const float *svz = reinterpret_cast<const float *>(wk + L::VZ);
        const float *llx = reinterpret_cast<const float *>(wk + L::LX);
        const float *lly = reinterpret_cast<const float *>(wk + L::LY);
        const float *llz = reinterpret_cast<const float *>(wk + L::LZ);
        // own-cell boxes: txx..tyz at q = 0..5; the medium: lambda, mu, shear moduli 0..4
        const float *own = reinterpret_cast<const float *>(wk + L::OWN);
        const float *med = reinterpret_cast<const float *>(st + LS::MED);
        constexpr int OS = al128(W32 * TY * 4) / 4;

        [[maybe_unused]] float dYy2[2] = {0.f, 0.f}, xyY2[2] = {0.f, 0.f}, yzY2[2] = {0.f, 0.f};
        if constexpr (CELLS == 2) {
            const float *cx0 = svx + (lyc[0] + 5) * W48 + lx + 8;
            const float *cy0 = svy + (lyc[0] + 5) * W48 + lx + 8;
            const float *cz0 = svz + (lyc[0] + 5) * W48 + lx + 8;
            dB2<FAST, 1>(ph, [&](int o) { return cy0[o * W48]; }, dYy2[0], dYy2[1]);
            dF2<FAST, 1>(ph, [&](int o) { return cx0[o * W48]; }, xyY2[0], xyY2[1]);
            dF2<FAST, 1>(ph, [&](int o) { return cz0[o * W48]; }, yzY2[0], yzY2[1]);
        }
#pragma unroll
        for (int c = 0; c < CELLS; ++c) {
            const int ly = lyc[c];
            qx[c][9 + P] = llx[ly * W32 + lx];
            qy[c][9 + P] = lly[ly * W32 + lx];
            qz[c][9 + P] = llz[ly * W32 + lx];
            if (!act[c]) continue;

            const float *cx_ = svx + (ly + 5) * W48 + lx + 8;
            const float *cy_ = svy + (ly + 5) * W48 + lx + 8;
            const float *cz_ = svz + (ly + 5) * W48 + lx + 8;
            float dXx, dYy, dZz, xyY, xyX, xzZ, xzX, yzZ, yzY;
            if constexpr (CELLS == 1) {
                // eight of the nine differences in pairs on FP32x2, same roundings
                // (REF: sums with the plain coefficients, then the divisions)
                const float2 pX = dpair(FAST ? ph.cp[0] : ph.cr,
                                        [&](int i) { return make_float2(cy_[1 + i], cz_[1 + i]); },
                                        [&](int i) { return make_float2(cy_[-i], cz_[-i]); });
                const float2 pY = dpair(FAST ? ph.cp[1] : ph.cr,
                                        [&](int i) { return make_float2(cx_[(1 + i) * W48], cz_[(1 + i) * W48]); },
                                        [&](int i) { return make_float2(cx_[-i * W48], cz_[-i * W48]); });
                const float2 pZ = dpair(FAST ? ph.cp[2] : ph.cr,
                                        [&](int i) { return make_float2(qx[c][P + 5 + i], qy[c][P + 5 + i]); },
                                        [&](int i) { return make_float2(qx[c][P + 4 - i], qy[c][P + 4 - i]); });
                const float2 pN = dpair(FAST ? ph.cp[3] : ph.cr,
                                        [&](int i) { return make_float2(cx_[i], cy_[i * W48]); },
                                        [&](int i) { return make_float2(cx_[-1 - i], cy_[(-1 - i) * W48]); });
                xyX = by_cell<FAST>(ph, 0, pX.x); xzX = by_cell<FAST>(ph, 0, pX.y);
                xyY = by_cell<FAST>(ph, 1, pY.x); yzY = by_cell<FAST>(ph, 1, pY.y);
                xzZ = by_cell<FAST>(ph, 2, pZ.x); yzZ = by_cell<FAST>(ph, 2, pZ.y);
                dXx = by_cell<FAST>(ph, 0, pN.x); dYy = by_cell<FAST>(ph, 1, pN.y);
            } else {
                dXx = dB<FAST, 0>(ph, [&](int o) { return cx_[o]; });
                dYy = CELLS == 2 ? dYy2[c] : dB<FAST, 1>(ph, [&](int o) { return cy_[o * W48]; });
                xyY = CELLS == 2 ? xyY2[c] : dF<FAST, 1>(ph, [&](int o) { return cx_[o * W48]; });
                xyX = dF<FAST, 0>(ph, [&](int o) { return cy_[o]; });
                xzZ = dF<FAST, 2>(ph, [&](int o) { return qx[c][P + 4 + o]; });
                xzX = dF<FAST, 0>(ph, [&](int o) { return cz_[o]; });
                yzZ = dF<FAST, 2>(ph, [&](int o) { return qy[c][P + 4 + o]; });
                yzY = CELLS == 2 ? yzY2[c] : dF<FAST, 1>(ph, [&](int o) { return cz_[o * W48]; });
            }
            dZz = dB<FAST, 2>(ph, [&](int o) { return qz[c][P + 5 + o]; });

            const int e = ly * W32 + lx;
            const float l = med[e], mu_c = med[OS + e];
            const float l2m = __fmaf_rn(2.0f, mu_c, l);
            const float mxy = med[2 * OS + e], mxz = med[3 * OS + e], myz = med[4 * OS + e];

            const uint32_t ci = col[c] + (uint32_t)gz * PL;
            const int ky = kyc[c];
            float snew[6];
            if (!(plane_pml && (kx | ky | kz))) {
                float o0 = own[e], o1 = own[OS + e], o2 = own[2 * OS + e];
                if (GEN && (int64_t)ci == src) { o0 = o0 + inj; o1 = o1 + inj; o2 = o2 + inj; }
                snew[0] = __fmaf_rn(ph.dt, __fmaf_rn(l2m, dXx, l * (dYy + dZz)), o0);
                snew[1] = __fmaf_rn(ph.dt, __fmaf_rn(l2m, dYy, l * (dXx + dZz)), o1);
                snew[2] = __fmaf_rn(ph.dt, __fmaf_rn(l2m, dZz, l * (dXx + dYy)), o2);
                snew[3] = __fmaf_rn(ph.dt * mxy, xyY + xyX, own[3 * OS + e]);
                snew[4] = __fmaf_rn(ph.dt * mxz, xzZ + xzX, own[4 * OS + e]);
                snew[5] = __fmaf_rn(ph.dt * myz, yzZ + yzY, own[5 * OS + e]);
            } else {
                auto *sp = spl() + split_base32(pml_plane_index(m, pcol[c], cz));
                constexpr uint32_t N = kSplitBlock;   // split k at sp[k * N]
                // split S_XXX + k belongs to field txx..tyz (its scale with 16-bit storage)
                auto grp = [](int k) { return k < 9 ? 3 + k / 3 : 6 + (k - 9) / 2; };
                auto sput = [&](int k, float v) {
                    if constexpr (H) {
                        if (track) note_max16s(smax, grp(k - S_XXX), v);
                    }
                    put(sp + k * N, grp(k - S_XXX), v);
                };
                float o[15];
#pragma unroll
                for (int q = 0; q < 15; ++q) o[q] = ld(sp + (S_XXX + q) * N, grp(q));
                float mx = 1.f, my = 1.f, mz = 1.f;
        PDiv<FAST> px = 1, py = 1, pz = 1;
                {
                    const float v = damp_speed(ph, mu_c, m.b[ci], l);
                    if (kx) damp_factors<FAST>(ph, 0, ph.dx, kx, m.pml, v, mx, px);
                    if (ky) damp_factors<FAST>(ph, 1, ph.dy, ky, m.pml, v, my, py);
                    if (kz) damp_factors<FAST>(ph, 2, ph.dz, kz, m.pml, v, mz, pz);
                }
                const float dl = ph.dt * l2m, dt = ph.dt;
                float a0, a1, a2;
                a0 = split_update<FAST>(o[S_XXX - S_XXX], dl, dXx, kx, mx, px);
                a1 = split_update<FAST>(o[S_XXY - S_XXX], dt, l * dYy, ky, my, py);
                a2 = split_update<FAST>(o[S_XXZ - S_XXX], dt, l * dZz, kz, mz, pz);
                sput(S_XXX, a0); sput(S_XXY, a1); sput(S_XXZ, a2);
                snew[0] = (a0 + a1) + a2;
                a0 = split_update<FAST>(o[S_YYX - S_XXX], dt, l * dXx, kx, mx, px);
                a1 = split_update<FAST>(o[S_YYY - S_XXX], dl, dYy, ky, my, py);
                a2 = split_update<FAST>(o[S_YYZ - S_XXX], dt, l * dZz, kz, mz, pz);
                sput(S_YYX, a0); sput(S_YYY, a1); sput(S_YYZ, a2);
                snew[1] = (a0 + a1) + a2;
                a0 = split_update<FAST>(o[S_ZZX - S_XXX], dt, l * dXx, kx, mx, px);
                a1 = split_update<FAST>(o[S_ZZY - S_XXX], dt, l * dYy, ky, my, py);
                a2 = split_update<FAST>(o[S_ZZZ - S_XXX], dl, dZz, kz, mz, pz);
                sput(S_ZZX, a0); sput(S_ZZY, a1); sput(S_ZZZ, a2);
                snew[2] = (a0 + a1) + a2;
                const float axy = dt * mxy, axz = dt * mxz, ayz = dt * myz;
                a0 = split_update<FAST>(o[S_XYX - S_XXX], axy, xyX, kx, mx, px);
                a1 = split_update<FAST>(o[S_XYY - S_XXX], axy, xyY, ky, my, py);
                sput(S_XYX, a0); sput(S_XYY, a1);
                snew[3] = a0 + a1;
                a0 = split_update<FAST>(o[S_XZX - S_XXX], axz, xzX, kx, mx, px);
                a1 = split_update<FAST>(o[S_XZZ - S_XXX], axz, xzZ, kz, mz, pz);
                sput(S_XZX, a0); sput(S_XZZ, a1);
                snew[4] = a0 + a1;
                a0 = split_update<FAST>(o[S_YZY - S_XXX], ayz, yzY, ky, my, py);
                a1 = split_update<FAST>(o[S_YZZ - S_XXX], ayz, yzZ, kz, mz, pz);
                sput(S_YZY, a0); sput(S_YZZ, a1);
                snew[5] = a0 + a1;
            }
#pragma unroll
            for (int q = 0; q < 6; ++q) {
                if constexpr (H) {
                    if (track) note_max16s(smax, 3 + q, snew[q]);
                }
                put(fld(3 + q) + ci, 3 + q, snew[q]);
            }
            if (GEN && !H && gz == rz && it >= 0 && it < sr.nt) {
                for (int r = rp; r < rend && g.rec_list[r].z == gz; ++r) {
                    const int4 q = g.rec_list[r];
                    if (q.x == gx && q.y == gyc[c] && q.w >= 3)
                        sr.traces[(int64_t)it * sr.nrec + g.rec_idx[r]] =
                            q.w == 3 ? snew[0] : q.w == 4 ? snew[1] : q.w == 5 ? snew[2]
                          : q.w == 6 ? snew[3] : q.w == 7 ? snew[4] : snew[5];
                }
            }
        }
        if (GEN && gz == rz) {
            while (rp < rend && g.rec_list[rp].z == gz) ++rp;
            rz = rp < rend ? g.rec_list[rp].z : 0x7fffffff;
        }

        if (__syncthreads_or(failed)) return false;
        if (cz + S < t.ze) {
            if (lx == 0) {
                fence_proxy_async();
                str_issue<TY, ES>(mybox, nbox, st, &bar[s], cz + S, warp);
            }
            issued_end = cz + S + 1;
        }
        if (MANY) pbits ^= 1u << s;
        if (++stage == S) {
            stage = 0;
            if (!MANY) parity ^= 1u;
        }
        return true;
    };
    auto run = [&](auto p_tag) -> bool {
        const int gzp = cz + kHalo;
        const bool gen = t.xy_pml || bandz(m, gzp) != 0 || gzp == sz || gzp == rz;
        prefetch(cz + 1);
        return gen ? plane(std::true_type{}, p_tag) : plane(std::false_type{}, p_tag);
    };
    while (cz < t.ze) {
        if (!run(std::integral_constant<int, 0>{})) { abort = true; break; }
        if (++cz == t.ze) break;
        if (!run(std::integral_constant<int, 1>{})) { abort = true; break; }
        ++cz;
#pragma unroll
        for (int c = 0; c < CELLS; ++c) {
#pragma unroll
            for (int j = 0; j < 9; ++j) {
                qx[c][j] = qx[c][j + 2];
                qy[c][j] = qy[c][j + 2];
                qz[c][j] = qz[c][j + 2];
            }
        }
    }
    if (abort && tid == 0) {
        atomicExch(g.err, 1);
        if (MANY) drain_bits<S>(bar, issued_end, cz, t.zs, pbits);
        else drain<S>(bar, issued_end, cz, t.zs);
    }
    if constexpr (H) {
        if (track) {
            __syncthreads();
            flush_max16(hs, smax);
        }
    }
    return !abort;
}

template <bool FAST, int CELLS>
__global__ void __launch_bounds__(NT, 3)
k_stress_zmarch(const __grid_constant__ ZMaps mp, const __grid_constant__ Model m, const __grid_constant__ Physics ph,
                const __grid_constant__ ZGeom g, const __grid_constant__ SourceRec sr, int it_arg,
                float src_value, int use_wavelet) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    __shared__ __align__(8) uint64_t bar[S];
    __shared__ TmaBox boxes[kWarps][kMaxBoxesPerWarp];
    if (threadIdx.x == 0) {
        for (int s = 0; s < S; ++s) mbar_init(&bar[s], 1);
        fence_barrier_init();
    }
    __syncthreads();
    uint32_t pbits = 0;
    str_item<FAST, CELLS, false>(mp, m, ph, g, sr, it_arg, src_value, use_wavelet, blockIdx.x, blockIdx.y + g.c0,
                          align_smem(smem_raw), bar, boxes, pbits);
}

// 16-bit wavefield storage (ST = SGFD_STORE_BF16 / _F16), 32 x 8 tiles.
template <bool FAST, int ST>
__global__ void __launch_bounds__(NT, 3)
k_velocity_zmarch16(const __grid_constant__ ZMaps mp, const __grid_constant__ Model m,
                    const __grid_constant__ Physics ph, const __grid_constant__ ZGeom g,
                    const __grid_constant__ SourceRec sr, const __grid_constant__ HalfState hs, int it_arg) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    __shared__ __align__(8) uint64_t bar[S];
    __shared__ TmaBox boxes[kWarps][kMaxBoxesPerWarp];
    if (threadIdx.x == 0) {
        for (int s = 0; s < S; ++s) mbar_init(&bar[s], 1);
        fence_barrier_init();
    }
    __syncthreads();
    uint32_t pbits = 0;
    vel_item<FAST, 1, false, ST>(mp, m, ph, g, sr, it_arg, 0.0f, 0, blockIdx.x, blockIdx.y + g.c0, align_smem(smem_raw), bar,
                                 boxes, pbits, hs);
}
template <bool FAST, int ST>
__global__ void __launch_bounds__(NT, 3)
k_stress_zmarch16(const __grid_constant__ ZMaps mp, const __grid_constant__ Model m,
                  const __grid_constant__ Physics ph, const __grid_constant__ ZGeom g,
                  const __grid_constant__ SourceRec sr, const __grid_constant__ HalfState hs, int it_arg) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    __shared__ __align__(8) uint64_t bar[S];
    __shared__ TmaBox boxes[kWarps][kMaxBoxesPerWarp];
    if (threadIdx.x == 0) {
        for (int s = 0; s < S; ++s) mbar_init(&bar[s], 1);
        fence_barrier_init();
    }
    __syncthreads();
    uint32_t pbits = 0;
    str_item<FAST, 1, false, ST>(mp, m, ph, g, sr, it_arg, 0.0f, 0, blockIdx.x, blockIdx.y + g.c0, align_smem(smem_raw), bar,
                                 boxes, pbits, hs);
}

PFN_cuTensorMapEncodeTiled_v12000 get_encoder() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    if (!fn) {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    }
    return fn;
}

template <int CELLS>
int vel_smem() { return S * VelL<8 * CELLS>::STAGE + 128; }
template <int CELLS>
int str_smem() { return S * StrL<8 * CELLS>::STAGE + 128; }

template <bool FAST, int CELLS>
cudaError_t set_attrs() {
    cudaError_t e = cudaFuncSetAttribute(k_velocity_zmarch<FAST, CELLS>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, vel_smem<CELLS>());
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_stress_zmarch<FAST, CELLS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 str_smem<CELLS>());
    return e;
}

// 16-bit storage: the ring of 16-bit stages, then the FP32 work buffer.
constexpr int vel_smem16() { return S * VelL<8, 2>::STAGE + VelL<8>::STAGE + 128; }
constexpr int str_smem16() { return S * StrL<8, 2>::STAGE + StrL<8>::STAGE + 128; }
static_assert(3 * (vel_smem16() + 1024) <= 228 * 1024 && 3 * (str_smem16() + 1024) <= 228 * 1024,
              "three CTAs per SM");

template <bool FAST, int ST>
cudaError_t set_attrs16() {
    cudaError_t e = cudaFuncSetAttribute(k_velocity_zmarch16<FAST, ST>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         vel_smem16());
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_stress_zmarch16<FAST, ST>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 str_smem16());
    return e;
}

// ---------------------------------------------------------------------------
// persistent batch: every model's (tile, z chunk) work items of the 32 x 8
// tiling, the velocity phase then the stress phase of each step, a bounded
// grid barrier after each phase
// ---------------------------------------------------------------------------

constexpr int batch_smem() { return vel_smem<1>() > str_smem<1>() ? vel_smem<1>() : str_smem<1>(); }

// The two updates as called functions, so that each is register-allocated on
// its own rather than inlined side by side into the persistent loop.
template <bool FAST>
__device__ __noinline__ bool vel_item_call(const ZMaps &mp, const Model &m, const Physics &ph, const ZGeom &g,
                                           const SourceRec &sr, int it, int tile, int chunk, unsigned char *smem,
                                           uint64_t *bar, TmaBox (*boxes)[kMaxBoxesPerWarp], uint32_t &pbits) {
    return vel_item<FAST, 1, true>(mp, m, ph, g, sr, it, 0.0f, 1, tile, chunk, smem, bar, boxes, pbits);
}
template <bool FAST>
__device__ __noinline__ bool str_item_call(const ZMaps &mp, const Model &m, const Physics &ph, const ZGeom &g,
                                           const SourceRec &sr, int it, int tile, int chunk, unsigned char *smem,
                                           uint64_t *bar, TmaBox (*boxes)[kMaxBoxesPerWarp], uint32_t &pbits) {
    return str_item<FAST, 1, true>(mp, m, ph, g, sr, it, 0.0f, 1, tile, chunk, smem, bar, boxes, pbits);
}

// Two CTAs per SM: the 128 registers a thread then has keep both called
// updates nearly free of spills (at three CTAs the stress update, whose
// physics and geometry come from shared memory here, spills 0.5 KB).
template <bool FAST>
__global__ void __launch_bounds__(NT, 2)
k_batch_zmarch(const ZModel *models, int nmodels, const int *first_item, int it0, int nsteps, unsigned *ctl,
               unsigned barrier_ctas, int *status) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    __shared__ __align__(8) uint64_t bar_v[S];
    __shared__ __align__(8) uint64_t bar_s[S];
    __shared__ TmaBox boxes[kWarps][kMaxBoxesPerWarp];
    __shared__ int item_sh, ok_sh;
    // the current model's physics and geometry, read in every plane's inner
    // loops: a shared copy instead of loads from the descriptor array
    __shared__ __align__(16) Physics ph_s;
    __shared__ __align__(16) Model m_s;
    int cur = -1;
    if (threadIdx.x == 0) {
        for (int s = 0; s < S; ++s) mbar_init(&bar_v[s], 1);
        for (int s = 0; s < S; ++s) mbar_init(&bar_s[s], 1);
        fence_barrier_init();
    }
    __syncthreads();
    unsigned char *smem = align_smem(smem_raw);
    uint32_t pv = 0, ps = 0;
    const int total = first_item[nmodels];
    unsigned phases = 0;
    for (int k = 0; k < nsteps; ++k) {
        for (int p = 0; p < 2; ++p) {
            unsigned *ctr = ctl + 1 + 2 * k + p;
            for (;;) {
                if (threadIdx.x == 0) item_sh = (int)atomicAdd(ctr, 1u);
                __syncthreads();
                const int item = item_sh;
                __syncthreads();
                if (item >= total) break;
                int mi = 0;
                while (first_item[mi + 1] <= item) ++mi;
                const ZModel &d = models[mi];
                if (mi != cur) {   // every thread is past the previous item (the barriers above)
                    const uint32_t *src = reinterpret_cast<const uint32_t *>(&d.ph);
                    uint32_t *dst = reinterpret_cast<uint32_t *>(&ph_s);
                    for (int i = threadIdx.x; i < (int)(sizeof(Physics) / 4); i += NT) dst[i] = src[i];
                    src = reinterpret_cast<const uint32_t *>(&d.m);
                    dst = reinterpret_cast<uint32_t *>(&m_s);
                    for (int i = threadIdx.x; i < (int)(sizeof(Model) / 4); i += NT) dst[i] = src[i];
                    __syncthreads();
                    cur = mi;
                }
                const int local = item - first_item[mi];
                const int ntiles = d.g.ntx * d.g.nty;
                const bool ok =
                    p == 0 ? vel_item_call<FAST>(d.zm, m_s, ph_s, d.g, d.sr, it0 + k, local % ntiles, local / ntiles,
                                                 smem, bar_v, boxes, pv)
                           : str_item_call<FAST>(d.zm, m_s, ph_s, d.g, d.sr, it0 + k, local % ntiles, local / ntiles,
                                                 smem, bar_s, boxes, ps);
                if (!ok) {
                    if (threadIdx.x == 0) atomicExch(status, kBatchWaitTma);
                    return;
                }
            }
            ++phases;
            if (!grid_sync(ctl, phases * barrier_ctas, status, kBatchWaitGrid, &ok_sh)) return;
        }
    }
}

// One step with 16-bit storage: the source injection before the velocity
// update, the velocity receivers after it, the stress receivers and the
// rescale after the stress update (kernels_half.cu, half_phase).
template <bool FAST, int ST>
void launch16(const Model &m, const Physics &ph, const SourceRec &sr, const HalfState &hs, const ZGeom &g,
              const ZMaps &zm, int it, float src_value, bool uw, cudaStream_t s, cudaEvent_t *ev) {
    const dim3 grid(g.ntx * g.nty, g.nchunks);
    half_phase(m, ph, sr, hs, it, src_value, uw, s, 0);
    if (ev) cudaEventRecord(ev[0], s);
    k_velocity_zmarch16<FAST, ST><<<grid, NT, vel_smem16(), s>>>(zm, m, ph, g, sr, hs, it);
    if (ev) cudaEventRecord(ev[1], s);
    half_phase(m, ph, sr, hs, it, src_value, uw, s, 1);
    if (ev) cudaEventRecord(ev[2], s);
    k_stress_zmarch16<FAST, ST><<<grid, NT, str_smem16(), s>>>(zm, m, ph, g, sr, hs, it);
    if (ev) cudaEventRecord(ev[3], s);
    half_phase(m, ph, sr, hs, it, src_value, uw, s, 2);
}

template <bool FAST, int CELLS>
void launch(const Model &m, const Physics &ph, const SourceRec &sr, const ZGeom &g, const ZMaps &zm, int it,
            float src_value, int uw, cudaStream_t s, cudaEvent_t *ev, int phases, int parts) {
    // chunk ranges of the selected parts: inner chunks lie 5 or more planes
    // from both ends (they read no frame plane), outer chunks are the rest
    int range[3][2];
    const int nr = part_ranges(m.nzc, g.zc, g.nchunks, parts, range);
    auto each = [&](auto fn) {
        for (int r = 0; r < nr; ++r) {
            if (range[r][1] <= range[r][0]) continue;
            ZGeom gr = g;
            gr.c0 = range[r][0];
            fn(dim3(g.ntx * g.nty, range[r][1] - range[r][0]), gr);
        }
    };
    if (phases & 1) {
        if (ev) cudaEventRecord(ev[0], s);
        each([&](dim3 grid, const ZGeom &gr) {
            k_velocity_zmarch<FAST, CELLS><<<grid, NT, vel_smem<CELLS>(), s>>>(zm, m, ph, gr, sr, it, src_value, uw);
        });
        if (ev) cudaEventRecord(ev[1], s);
    }
    if (phases & 2) {
        if (ev) cudaEventRecord(ev[2], s);
        each([&](dim3 grid, const ZGeom &gr) {
            k_stress_zmarch<FAST, CELLS><<<grid, NT, str_smem<CELLS>(), s>>>(zm, m, ph, gr, sr, it, src_value, uw);
        });
        if (ev) cudaEventRecord(ev[3], s);
    }
}

}  // namespace

// 3-D FP32 tensor map over one padded array (base = allocation start).
bool make_box_map(CUtensorMap *map, const float *grid_origin, const Model &m, int bx, int by) {
    auto enc = get_encoder();
    if (!enc) return false;
    void *base = const_cast<float *>(grid_origin - kXOff);
    cuuint64_t dims[3] = {(cuuint64_t)(m.nx + kXOff), (cuuint64_t)m.ny, (cuuint64_t)m.nz};
    cuuint64_t strides[2] = {(cuuint64_t)m.px * 4, (cuuint64_t)m.plane * 4};
    cuuint32_t box[3] = {(cuuint32_t)bx, (cuuint32_t)by, 1};
    cuuint32_t es[3] = {1, 1, 1};
    CUresult r = enc(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, base, dims, strides, box, es,
                     CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                     CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS;
}

bool make_box_map16(CUtensorMap *map, const uint16_t *grid_origin, const Model &m, int bx, int by) {
    auto enc = get_encoder();
    if (!enc) return false;
    void *base = const_cast<uint16_t *>(grid_origin - kXOff);
    cuuint64_t dims[3] = {(cuuint64_t)(m.nx + kXOff), (cuuint64_t)m.ny, (cuuint64_t)m.nz};
    cuuint64_t strides[2] = {(cuuint64_t)m.px * 2, (cuuint64_t)m.plane * 2};
    cuuint32_t box[3] = {(cuuint32_t)bx, (cuuint32_t)by, 1};
    cuuint32_t es[3] = {1, 1, 1};
    CUresult r = enc(map, CU_TENSOR_MAP_DATA_TYPE_UINT16, 3, base, dims, strides, box, es,
                     CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                     CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS;
}

bool zmarch_supported(const Model &m) {
    // Halo boxes start 8 cells left of the tile and 5 rows above: always inside
    // the padded array because the frame is 5 cells and kXOff is 27.  The
    // kernels address cells and PML split values with 32-bit offsets: cell
    // offsets below 2^31, split offsets (the blocked split array) below 2^32
    const bool small = m.plane * (int64_t)m.nz < ((int64_t)1 << 31) && split_elems(m.npml) <= ((int64_t)1 << 32);
    return small && m.nxc >= 1 && m.nyc >= 1 && m.nzc >= 1 && get_encoder() != nullptr;
}

// 4-D FP32 tensor map over `count` arrays of the pool, `stride` bytes apart,
// the first at `first`, with a bx x by x 1 x count box.
bool make_pool_map(CUtensorMap *map, const float *first, const Model &m, size_t stride, int count, int bx, int by) {
    auto enc = get_encoder();
    if (!enc) return false;
    void *base = const_cast<float *>(first - kXOff);
    cuuint64_t dims[4] = {(cuuint64_t)(m.nx + kXOff), (cuuint64_t)m.ny, (cuuint64_t)m.nz, (cuuint64_t)count};
    cuuint64_t strides[3] = {(cuuint64_t)m.px * 4, (cuuint64_t)m.plane * 4, (cuuint64_t)stride};
    cuuint32_t box[4] = {(cuuint32_t)bx, (cuuint32_t)by, 1, (cuuint32_t)count};
    cuuint32_t es[4] = {1, 1, 1, 1};
    CUresult r = enc(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, base, dims, strides, box, es,
                     CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                     CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS;
}

// The same over 16-bit arrays of the same layout.
bool make_pool_map16(CUtensorMap *map, const uint16_t *first, const Model &m, size_t stride, int count, int bx,
                     int by) {
    auto enc = get_encoder();
    if (!enc) return false;
    void *base = const_cast<uint16_t *>(first - kXOff);
    cuuint64_t dims[4] = {(cuuint64_t)(m.nx + kXOff), (cuuint64_t)m.ny, (cuuint64_t)m.nz, (cuuint64_t)count};
    cuuint64_t strides[3] = {(cuuint64_t)m.px * 2, (cuuint64_t)m.plane * 2, (cuuint64_t)stride};
    cuuint32_t box[4] = {(cuuint32_t)bx, (cuuint32_t)by, 1, (cuuint32_t)count};
    cuuint32_t es[4] = {1, 1, 1, 1};
    CUresult r = enc(map, CU_TENSOR_MAP_DATA_TYPE_UINT16, 4, base, dims, strides, box, es,
                     CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                     CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS;
}

cudaError_t zmarch_prepare(const Model &m, int cells, size_t st, ZMaps *zm, const HalfState *hs, size_t st16) {
    if (cells != 1 && cells != 2) return cudaErrorInvalidValue;
    if (hs) {
        // 16-bit storage: the stored wavefields (evenly spaced 16-bit arrays) and the FP32 medium
        if (cells != 1) return cudaErrorInvalidValue;
        for (int k = 0; k < 9; ++k)
            if (hs->f[k] != reinterpret_cast<const uint16_t *>(reinterpret_cast<const char *>(hs->f[0]) + k * st16))
                return cudaErrorInvalidValue;
        const float *med[5] = {m.lam, m.mu, m.mxy, m.mxz, m.myz};
        for (int k = 0; k < 5; ++k)
            if (med[k] != reinterpret_cast<const float *>(reinterpret_cast<const char *>(m.lam) + k * st))
                return cudaErrorInvalidValue;
        const int ty = 8;
        bool ok = true;
        ok &= make_pool_map16(&zm->v_sxx_sxz, hs->f[3], m, 4 * st16, 2, W48, ty);
        ok &= make_pool_map16(&zm->v_syy_syz, hs->f[4], m, 4 * st16, 2, W32, ty + 10);
        ok &= make_pool_map16(&zm->v_sxy, hs->f[6], m, st16, 1, W48, ty + 10);
        ok &= make_pool_map(&zm->v_b, m.b, m, st, 1, W36, ty + 1);
        ok &= make_pool_map16(&zm->v_lead_xz_yz, hs->f[7], m, st16, 2, W32, ty);
        ok &= make_pool_map16(&zm->v_lead_zz, hs->f[5], m, st16, 1, W32, ty);
        ok &= make_pool_map(&zm->v_lead_b, m.b, m, st, 1, W32, ty);
        ok &= make_pool_map16(&zm->v_own, hs->f[0], m, st16, 3, W32, ty);
        ok &= make_pool_map16(&zm->s_v, hs->f[0], m, st16, 3, W48, ty + 10);
        ok &= make_pool_map16(&zm->s_lead_xy, hs->f[0], m, st16, 2, W32, ty);
        ok &= make_pool_map16(&zm->s_lead_z, hs->f[2], m, st16, 1, W32, ty);
        ok &= make_pool_map16(&zm->s_own, hs->f[3], m, st16, 6, W32, ty);
        ok &= make_pool_map(&zm->s_med, m.lam, m, st, 5, W32, ty);
        if (!ok) return cudaErrorInvalidValue;
        cudaError_t e = set_attrs16<false, SGFD_STORE_BF16>();
        if (e == cudaSuccess) e = set_attrs16<true, SGFD_STORE_BF16>();
        if (e == cudaSuccess) e = set_attrs16<false, SGFD_STORE_F16>();
        if (e == cudaSuccess) e = set_attrs16<true, SGFD_STORE_F16>();
        return e;
    }
    // the pool order the merged copies rely on: vx..tyz, lambda, mu, mxy, mxz, myz
    auto at = [&](int k) { return reinterpret_cast<const float *>(reinterpret_cast<const char *>(m.f[0]) + k * st); };
    const float *order[14] = {m.f[0], m.f[1], m.f[2], m.f[3], m.f[4], m.f[5], m.f[6], m.f[7],
                              m.f[8], m.lam, m.mu, m.mxy, m.mxz, m.myz};
    for (int k = 0; k < 14; ++k)
        if (order[k] != at(k)) return cudaErrorInvalidValue;
    const int ty = 8 * cells;
    bool ok = true;
    ok &= make_pool_map(&zm->v_sxx_sxz, m.f[3], m, 4 * st, 2, W48, ty);        // sigma_xx, sigma_xz
    ok &= make_pool_map(&zm->v_syy_syz, m.f[4], m, 4 * st, 2, W32, ty + 10);   // sigma_yy, sigma_yz
    ok &= make_pool_map(&zm->v_sxy, m.f[6], m, st, 1, W48, ty + 10);
    ok &= make_pool_map(&zm->v_b, m.b, m, st, 1, W36, ty + 1);
    ok &= make_pool_map(&zm->v_lead_xz_yz, m.f[7], m, st, 2, W32, ty);
    ok &= make_pool_map(&zm->v_lead_zz, m.f[5], m, st, 1, W32, ty);
    ok &= make_pool_map(&zm->v_lead_b, m.b, m, st, 1, W32, ty);
    ok &= make_pool_map(&zm->v_own, m.f[0], m, st, 3, W32, ty);
    ok &= make_pool_map(&zm->s_v, m.f[0], m, st, 3, W48, ty + 10);
    ok &= make_pool_map(&zm->s_lead_xy, m.f[0], m, st, 2, W32, ty);
    ok &= make_pool_map(&zm->s_lead_z, m.f[2], m, st, 1, W32, ty);
    ok &= make_pool_map(&zm->s_own, m.f[3], m, st, 11, W32, ty);
    zm->s_med = zm->s_own;   // unused by FP32 storage (its own-cell copy brings the medium too)
    if (!ok) return cudaErrorInvalidValue;
    cudaError_t e = cells == 1 ? set_attrs<false, 1>() : set_attrs<false, 2>();
    if (e == cudaSuccess) e = cells == 1 ? set_attrs<true, 1>() : set_attrs<true, 2>();
    return e;
}

void zmarch_tiles(const Model &m, int cells, int *ntx, int *nty) {
    *ntx = (m.nxc + TX - 1) / TX;
    *nty = (m.nyc + 8 * cells - 1) / (8 * cells);
}

cudaError_t zmarch_step(const Model &m, const Physics &ph, const SourceRec &sr, const ZGeom &g, const ZMaps &zm,
                        int it, float src_value, bool use_wavelet, cudaStream_t s, cudaEvent_t *ev,
                        const HalfState *hs, int phases, int parts) {
    if (hs) {
        if (hs->storage == SGFD_STORE_BF16) {
            if (ph.fast) launch16<true, SGFD_STORE_BF16>(m, ph, sr, *hs, g, zm, it, src_value, use_wavelet, s, ev);
            else launch16<false, SGFD_STORE_BF16>(m, ph, sr, *hs, g, zm, it, src_value, use_wavelet, s, ev);
        } else {
            if (ph.fast) launch16<true, SGFD_STORE_F16>(m, ph, sr, *hs, g, zm, it, src_value, use_wavelet, s, ev);
            else launch16<false, SGFD_STORE_F16>(m, ph, sr, *hs, g, zm, it, src_value, use_wavelet, s, ev);
        }
        return cudaGetLastError();
    }
    const int uw = use_wavelet ? 1 : 0;
    if (ph.fast) {
        if (g.cells == 1) launch<true, 1>(m, ph, sr, g, zm, it, src_value, uw, s, ev, phases, parts);
        else launch<true, 2>(m, ph, sr, g, zm, it, src_value, uw, s, ev, phases, parts);
    } else {
        if (g.cells == 1) launch<false, 1>(m, ph, sr, g, zm, it, src_value, uw, s, ev, phases, parts);
        else launch<false, 2>(m, ph, sr, g, zm, it, src_value, uw, s, ev, phases, parts);
    }
    return cudaGetLastError();
}

int zmarch_batch_ctas(int device) {
    int sms = 0, per = 0, per2 = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) return 0;
    if (cudaFuncSetAttribute(k_batch_zmarch<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, batch_smem()) !=
            cudaSuccess ||
        cudaFuncSetAttribute(k_batch_zmarch<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, batch_smem()) !=
            cudaSuccess)
        return 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_batch_zmarch<true>, NT, batch_smem()) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per2, k_batch_zmarch<false>, NT, batch_smem()) != cudaSuccess)
        return 0;
    return sms * (per < per2 ? per : per2);
}

cudaError_t zmarch_batch_run(const ZModel *models, int nmodels, const int *first_item, int it0, int nsteps,
                             unsigned *ctl, int barrier_ctas, int ctas, bool fast, int *status, cudaStream_t s) {
    unsigned target = (unsigned)barrier_ctas;
    void *args[] = {(void *)&models, (void *)&nmodels, (void *)&first_item, (void *)&it0, (void *)&nsteps,
                    (void *)&ctl, (void *)&target, (void *)&status};
    const void *fn = fast ? (const void *)k_batch_zmarch<true> : (const void *)k_batch_zmarch<false>;
    return cudaLaunchCooperativeKernel(fn, dim3(ctas), dim3(NT), args, batch_smem(), s);
}

}  // namespace sgfd
