// kernels_zmarch.cu — the "zmarch" kernel family: 2.5-D z-marching velocity
// and stress updates for sm_100a.
//
// Work decomposition.  A CTA of 256 threads owns a 32 x TY tile of computed
// cells in the xy plane (TY = 8 * CELLS, each thread owning CELLS vertically
// adjacent cells, whose y differences share one window of staged values) and
// marches along z over a chunk of planes.
//
// Data movement per plane z (all HBM traffic is TMA or coalesced 128-byte rows):
//   * TMA (cp.async.bulk.tensor.3d, no multicast) stages
//     the xy boxes the x/y derivatives need — tile plus its 5-cell halo on the
//     sides a field is differentiated along — and the "lead" planes that feed
//     the z register queues, and the cell's own read-modify-write data, into
//     a 3-stage shared-memory ring guarded by one mbarrier per stage (expect-tx
//     bytes, parity wait with an iteration cap); lane 0 of each warp issues a
//     share of a stage's boxes so that no warp carries the issue alone.
//     A stage is refilled with plane z + 3 as soon as plane z is done, so
//     every load has two plane-iterations to land.
//   * Each thread keeps the 10 z-taps of the fields it differentiates along z
//     in a register queue (sigma_xz, sigma_yz, sigma_zz for the velocity
//     update; vx, vy, vz for the stress update), shifted by one per plane.
//   * The velocity update loads the PML split fields of its cell into
//     registers before the plane's TMA wait; the stress update, which needs
//     15 of them, loads them where they are used, so that it fits the 80
//     registers per thread of three resident CTAs per SM.
// Every row starts at a 128-byte boundary (the device arrays are shifted by
// kXOff), so x-halo boxes start 8 cells left of the tile (48 wide), centre
// boxes are exactly 32 wide, and every TMA x coordinate is a multiple of 4.
// One block barrier per plane separates the reads of a stage from its refill
// and carries the abort vote of the bounded waits.
//
// PML cells take the split-field path (cell_math.cuh), interior cells the
// plain update; a tile-plane with no PML cell never enters the PML code.
// The source (dt*dt*s(it) on txx, tyy, tzz, OPT/ElasticWaveEquation.cu:206-221)
// is applied to the staged copies the velocity update reads and to the old
// value the stress update accumulates onto, which reproduces the reference's
// store-then-read order exactly; receivers are written from registers.
// Arithmetic per cell is the same sequence as kernels_simple.cu and the oracle.
#include <cuda.h>
#include <cudaTypedefs.h>

#include <type_traits>

#include "cell_math.cuh"
#include "zmarch.h"
#include "zmarch_dev.cuh"

namespace sgfd {

namespace {

using namespace zdev;

constexpr int TX = kZTileX, NT = 256, S = 3;
constexpr int W48 = 48, W32 = 32, W36 = 36;

constexpr int al128(int b) { return (b + 127) / 128 * 128; }

// Shared-memory stage layout of the velocity update (bytes, 128-aligned boxes).
// Arrays that arrive in one 4-D copy are adjacent (sigma_xx, sigma_xz;
// sigma_yy, sigma_yz; the two lead planes at z+4; vx, vy, vz).
template <int TY>
struct VelL {
    static constexpr int SXX = 0;                                  // 48 x TY       sigma_xx (x halo)
    static constexpr int SXZ = SXX + W48 * TY * 4;                 // 48 x TY       sigma_xz (x halo)
    static constexpr int SYY = SXZ + al128(W48 * TY * 4);          // 32 x (TY+10)  sigma_yy (y halo)
    static constexpr int SYZ = SYY + W32 * (TY + 10) * 4;          // 32 x (TY+10)  sigma_yz (y halo)
    static constexpr int SXY = SYZ + al128(W32 * (TY + 10) * 4);   // 48 x (TY+10)  sigma_xy (x, y halo)
    static constexpr int B = SXY + al128(W48 * (TY + 10) * 4);     // 36 x (TY+1)   buoyancy (x+1, y+1)
    static constexpr int LXZ = B + al128(W36 * (TY + 1) * 4);      // 32 x TY       sigma_xz at z+4
    static constexpr int LYZ = LXZ + al128(W32 * TY * 4);          // 32 x TY       sigma_yz at z+4
    static constexpr int LZZ = LYZ + al128(W32 * TY * 4);          // 32 x TY       sigma_zz at z+5
    static constexpr int LB = LZZ + al128(W32 * TY * 4);           // 32 x TY       buoyancy at z+1
    static constexpr int OV = LB + al128(W32 * TY * 4);            // 3 x 32 x TY   own vx, vy, vz at z
    static constexpr int STAGE = OV + 3 * al128(W32 * TY * 4);
    static constexpr uint32_t TXB = 4 * (2 * W48 * TY + 2 * W32 * (TY + 10) + W48 * (TY + 10) +
                                         W36 * (TY + 1) + 7 * W32 * TY);
    static_assert(W48 * TY * 4 % 128 == 0 && W32 * (TY + 10) * 4 % 128 == 0 && W32 * TY * 4 % 128 == 0,
                  "arrays of one copy must be contiguous and 128-byte aligned");
};
// Shared-memory stage layout of the stress update.
template <int TY>
struct StrL {
    static constexpr int VX = 0;                                   // 48 x (TY+10)  vx (x, y halo)
    static constexpr int VY = VX + al128(W48 * (TY + 10) * 4);     // 48 x (TY+10)  vy
    static constexpr int VZ = VY + al128(W48 * (TY + 10) * 4);     // 48 x (TY+10)  vz
    static constexpr int LX = VZ + al128(W48 * (TY + 10) * 4);     // 32 x TY       vx at z+5
    static constexpr int LY = LX + al128(W32 * TY * 4);            // 32 x TY       vy at z+5
    static constexpr int LZ = LY + al128(W32 * TY * 4);            // 32 x TY       vz at z+4
    // own-cell data at z, 32 x TY each: txx tyy tzz txy txz tyz, lambda, mu,
    // the shear moduli of txy, txz, tyz
    static constexpr int OWN = LZ + al128(W32 * TY * 4);
    static constexpr int NOWN = 11;
    static constexpr int STAGE = OWN + NOWN * al128(W32 * TY * 4);
    static constexpr uint32_t TXB = 4 * (3 * W48 * (TY + 10) + (3 + NOWN) * W32 * TY);
    static_assert(W48 * (TY + 10) * 4 % 128 == 0 && W32 * TY * 4 % 128 == 0,
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
constexpr int kStrBoxes = 4;

// Box q of the velocity stage.
template <int TY>
__device__ __forceinline__ TmaBox vel_box(const ZMaps &mp, const Tile &t, int q) {
    using L = VelL<TY>;
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
template <int TY>
__device__ __forceinline__ void vel_issue(const TmaBox *b, int n, unsigned char *st, uint64_t *bar, int cz, int warp) {
    if (warp == 0) mbar_expect_tx(bar, VelL<TY>::TXB);
    issue_boxes(b, n, st, bar, cz + kHalo);
}

// The velocity update of one work item: the tile `tile` (x fastest) over z
// chunk `chunk`.  smem: the stage ring; bar: its S initialised mbarriers,
// whose phase parities pbits carries from item to item (bit s: the parity
// the next wait on stage s expects); boxes: per-warp TMA box scratch.
// Returns false after a bounded wait gave up (g.err set, copies drained).
// MANY: the CTA runs several items (persistent batch); a single-item launch
// keeps one parity for the whole ring and skips the fences a previous item needs.
template <bool FAST, int CELLS, bool MANY>
__device__ __forceinline__ bool vel_item(const ZMaps &mp, const Model &m, const Physics &ph, const ZGeom &g,
                                         const SourceRec &sr, int it_arg, float src_value, int use_wavelet, int tile,
                                         int chunk, unsigned char *smem, uint64_t *bar,
                                         TmaBox (*boxes)[kMaxBoxesPerWarp], uint32_t &pbits) {
    constexpr int TY = 8 * CELLS;
    using L = VelL<TY>;
    const Tile t = make_tile<TY>(m, g, tile, chunk);
    const int tid = threadIdx.x, lx = tid & 31, ty = tid >> 5;
    const int warp = tid >> 5;
    const TmaBox *mybox = boxes[warp];
    const int nbox = (kVelBoxes - warp + kWarps - 1) / kWarps;
    if (lx == 0) {
        for (int j = 0; j < nbox; ++j) boxes[warp][j] = vel_box<TY>(mp, t, warp + j * kWarps);
        if (MANY) fence_proxy_async();   // a previous item's stages were read through the generic proxy
        for (int s = 0; s < S && t.zs + s < t.ze; ++s)
            vel_issue<TY>(mybox, nbox, smem + s * L::STAGE, &bar[s], t.zs + s, warp);
    }
    int issued_end = min(t.zs + S, t.ze);   // planes [zs, issued_end) issued
    int stage = 0;                          // stage of plane cz
    uint32_t parity = 0;                    // single item: the parity of every stage's next wait

    const int it = step_index(sr, it_arg);
    const float inj = ph.inj_dt2 * ((use_wavelet && sr.wavelet) ? sr.wavelet[it] : src_value);
    int sx = -1, sy = -1, sz = -1;
    if (sr.src >= 0) {
        const int64_t r = sr.src;
        sz = (int)(r / m.plane);
        sy = (int)((r - (int64_t)sz * m.plane) / m.px);
        sx = (int)(r - (int64_t)sz * m.plane - (int64_t)sy * m.px);
    }

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
            qxz[c][k + 1] = m.f[7][col[c] + (uint32_t)(gz0 - 5 + k) * PL];
            qyz[c][k + 1] = m.f[8][col[c] + (uint32_t)(gz0 - 5 + k) * PL];
            float zz = m.f[5][col[c] + (uint32_t)(gz0 - 4 + k) * PL];
            if (gx == sx && gyc[c] == sy && gz0 - 4 + k == sz) zz = zz + inj;
            qzz[c][k + 1] = zz;
        }
    }

    // receivers of this tile, sorted by z: skip those below the chunk
    int rp = g.rec_off[tile];
    const int rend = g.rec_off[tile + 1];
    while (rp < rend && g.rec_list[rp].z < gz0) ++rp;
    int rz = rp < rend ? g.rec_list[rp].z : 0x7fffffff;   // z of the next receiver

    bool failed = false, abort = false;
    int cz = t.zs;
    const bool src_near = sr.src >= 0 && sy >= t.gy0 - 5 && sy < t.gy0 + TY + 5 && sx >= t.gx0 - 8 &&
                          sx < t.gx0 + TX + 8;
    // One plane.  GEN selects the general path (PML cells, source, receivers);
    // the interior-only path is used for every other tile-plane.  Returns
    // false when the block votes to abort.
    auto plane = [&](auto gen_tag) -> bool {
        constexpr bool GEN = decltype(gen_tag)::value;
        const int s = stage;
        unsigned char *st = smem + s * L::STAGE;
        const int gz = cz + kHalo;
        const int kz = band(gz, m.nz, m.pml);
        const bool plane_pml = GEN && (t.xy_pml || kz != 0);


        // PML cells: splits and the medium of the damping, loaded before the
        // stage wait so that their latency overlaps the wait and the stencil
        float opre[CELLS][9], mupre[CELLS], lampre[CELLS];
        if (plane_pml) {
            const uint32_t N = (uint32_t)m.npml;
#pragma unroll
            for (int c = 0; c < CELLS; ++c) {
                if (act[c] && (kx | kyc[c] | kz)) {
                    const uint32_t ci = col[c] + (uint32_t)gz * PL;
                    const float *sp = m.split + pml_plane_index(m, pcol[c], cz);
#pragma unroll
                    for (int q = 0; q < 9; ++q) opre[c][q] = sp[q * N];
                    mupre[c] = m.mu[ci];
                    lampre[c] = ph.damping == 1 ? m.lam[ci] : 0.f;
                }
            }
        }

        if (!mbar_wait(&bar[s], MANY ? (pbits >> s) & 1u : parity)) failed = true;

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

        const float *sxx = reinterpret_cast<const float *>(st + L::SXX);
        const float *syy = reinterpret_cast<const float *>(st + L::SYY);
        const float *sxy = reinterpret_cast<const float *>(st + L::SXY);
        const float *sxz = reinterpret_cast<const float *>(st + L::SXZ);
        const float *syz = reinterpret_cast<const float *>(st + L::SYZ);
        const float *bb = reinterpret_cast<const float *>(st + L::B);
        const float *lxz = reinterpret_cast<const float *>(st + L::LXZ);
        const float *lyz = reinterpret_cast<const float *>(st + L::LYZ);
        const float *lzz = reinterpret_cast<const float *>(st + L::LZZ);
        const float *lb = reinterpret_cast<const float *>(st + L::LB);
        const float *ov = reinterpret_cast<const float *>(st + L::OV);
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
                float *sp = m.split + pml_plane_index(m, pcol[c], cz);
                const uint32_t N = (uint32_t)m.npml;
                const float *o = opre[c];
                float a0, a1, a2;
                a0 = split_update<FAST>(o[S_VXX], ax, xX, kx, mx, px);
                a1 = split_update<FAST>(o[S_VXY], ax, xY, ky, my, py);
                a2 = split_update<FAST>(o[S_VXZ], ax, xZ, kz, mz, pz);
                sp[S_VXX * N] = a0; sp[S_VXY * N] = a1; sp[S_VXZ * N] = a2;
                vnew[0] = (a0 + a1) + a2;
                a0 = split_update<FAST>(o[S_VYX], ay, yX, kx, mx, px);
                a1 = split_update<FAST>(o[S_VYY], ay, yY, ky, my, py);
                a2 = split_update<FAST>(o[S_VYZ], ay, yZ, kz, mz, pz);
                sp[S_VYX * N] = a0; sp[S_VYY * N] = a1; sp[S_VYZ * N] = a2;
                vnew[1] = (a0 + a1) + a2;
                a0 = split_update<FAST>(o[S_VZX], az, zX, kx, mx, px);
                a1 = split_update<FAST>(o[S_VZY], az, zY, ky, my, py);
                a2 = split_update<FAST>(o[S_VZZ], az, zZ, kz, mz, pz);
                sp[S_VZX * N] = a0; sp[S_VZY * N] = a1; sp[S_VZZ * N] = a2;
                vnew[2] = (a0 + a1) + a2;
            }
            m.f[0][ci] = vnew[0];
            m.f[1][ci] = vnew[1];
            m.f[2][ci] = vnew[2];
            // receivers of velocity components at this cell (list sorted by z)
            if (GEN && gz == rz && it >= 0 && it < sr.nt) {
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
                vel_issue<TY>(mybox, nbox, st, &bar[s], cz + S, warp);
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
        const bool gen = t.xy_pml || band(gzp, m.nz, m.pml) != 0 || (src_near && (gzp == sz || gzp + 5 == sz)) || gzp == rz;
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
    vel_item<FAST, CELLS, false>(mp, m, ph, g, sr, it_arg, src_value, use_wavelet, blockIdx.x, blockIdx.y,
                          align_smem(smem_raw), bar, boxes, pbits);
}

// ---------------------------------------------------------------------------
// stress update
// ---------------------------------------------------------------------------

// Box q of the stress stage.
template <int TY>
__device__ __forceinline__ TmaBox str_box(const ZMaps &mp, const Tile &t, int q) {
    using L = StrL<TY>;
    switch (q) {
    case 0: return {&mp.s_v, L::VX, t.xd - 8, t.gy0 - 5, 0};
    case 1: return {&mp.s_lead_xy, L::LX, t.xd, t.gy0, 5};
    case 2: return {&mp.s_lead_z, L::LZ, t.xd, t.gy0, 4};
    default: return {&mp.s_own, L::OWN, t.xd, t.gy0, 0};
    }
}

// Stage the stress inputs of computed plane cz, as vel_issue.
template <int TY>
__device__ __forceinline__ void str_issue(const TmaBox *b, int n, unsigned char *st, uint64_t *bar, int cz, int warp) {
    if (warp == 0) mbar_expect_tx(bar, StrL<TY>::TXB);
    issue_boxes(b, n, st, bar, cz + kHalo);
}

// The stress update of one work item, as vel_item.
template <bool FAST, int CELLS, bool MANY>
__device__ __forceinline__ bool str_item(const ZMaps &mp, const Model &m, const Physics &ph, const ZGeom &g,
                                         const SourceRec &sr, int it_arg, float src_value, int use_wavelet, int tile,
                                         int chunk, unsigned char *smem, uint64_t *bar,
                                         TmaBox (*boxes)[kMaxBoxesPerWarp], uint32_t &pbits) {
    constexpr int TY = 8 * CELLS;
    using L = StrL<TY>;
    const Tile t = make_tile<TY>(m, g, tile, chunk);
    const int tid = threadIdx.x, lx = tid & 31, ty = tid >> 5;
    const int warp = tid >> 5;
    const TmaBox *mybox = boxes[warp];
    const int nbox = (kStrBoxes - warp + kWarps - 1) / kWarps;
    if (lx == 0) {
        for (int j = 0; j < nbox; ++j) boxes[warp][j] = str_box<TY>(mp, t, warp + j * kWarps);
        if (MANY) fence_proxy_async();   // a previous item's stages were read through the generic proxy
        for (int s = 0; s < S && t.zs + s < t.ze; ++s)
            str_issue<TY>(mybox, nbox, smem + s * L::STAGE, &bar[s], t.zs + s, warp);
    }
    int issued_end = min(t.zs + S, t.ze);   // planes [zs, issued_end) issued
    int stage = 0;                          // stage of plane cz
    uint32_t parity = 0;                    // single item: the parity of every stage's next wait

    const int it = step_index(sr, it_arg);
    const float inj = ph.inj_dt2 * ((use_wavelet && sr.wavelet) ? sr.wavelet[it] : src_value);
    const int64_t src = sr.src;

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
            qx[c][k] = m.f[0][col[c] + (uint32_t)(gz0 - 4 + k) * PL];
            qy[c][k] = m.f[1][col[c] + (uint32_t)(gz0 - 4 + k) * PL];
            qz[c][k] = m.f[2][col[c] + (uint32_t)(gz0 - 5 + k) * PL];
        }
    }

    int rp = g.rec_off[tile];
    const int rend = g.rec_off[tile + 1];
    while (rp < rend && g.rec_list[rp].z < gz0) ++rp;
    int rz = rp < rend ? g.rec_list[rp].z : 0x7fffffff;

    bool failed = false, abort = false;
    int cz = t.zs;
    int sz = -1;
    if (src >= 0) sz = (int)(src / m.plane);
    // One plane, as in the velocity update (GEN: general path; P: place in
    // the pair).  Returns false when the block votes to abort.
    auto plane = [&](auto gen_tag, auto p_tag) -> bool {
        constexpr bool GEN = decltype(gen_tag)::value;
        constexpr int P = decltype(p_tag)::value;
        const int s = stage;
        unsigned char *st = smem + s * L::STAGE;
        const int gz = cz + kHalo;
        const int kz = band(gz, m.nz, m.pml);
        const bool plane_pml = GEN && (t.xy_pml || kz != 0);

        if (!mbar_wait(&bar[s], MANY ? (pbits >> s) & 1u : parity)) failed = true;

        const float *svx = reinterpret_cast<const float *>(st + L::VX);
        const float *svy = reinterpret_cast<const float *>(st + L::VY);
        const float *svz = reinterpret_cast<const float *>(st + L::VZ);
        const float *llx = reinterpret_cast<const float *>(st + L::LX);
        const float *lly = reinterpret_cast<const float *>(st + L::LY);
        const float *llz = reinterpret_cast<const float *>(st + L::LZ);
        // own-cell boxes: txx..tyz at q = 0..5, lambda 6, mu 7, shear moduli 8..10
        const float *own = reinterpret_cast<const float *>(st + L::OWN);
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
            const float l = own[6 * OS + e], mu_c = own[7 * OS + e];
            const float l2m = __fmaf_rn(2.0f, mu_c, l);
            const float mxy = own[8 * OS + e], mxz = own[9 * OS + e], myz = own[10 * OS + e];

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
                float *sp = m.split + pml_plane_index(m, pcol[c], cz);
                const uint32_t N = (uint32_t)m.npml;
                float o[15];
#pragma unroll
                for (int q = 0; q < 15; ++q) o[q] = sp[(S_XXX + q) * N];
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
                sp[S_XXX * N] = a0; sp[S_XXY * N] = a1; sp[S_XXZ * N] = a2;
                snew[0] = (a0 + a1) + a2;
                a0 = split_update<FAST>(o[S_YYX - S_XXX], dt, l * dXx, kx, mx, px);
                a1 = split_update<FAST>(o[S_YYY - S_XXX], dl, dYy, ky, my, py);
                a2 = split_update<FAST>(o[S_YYZ - S_XXX], dt, l * dZz, kz, mz, pz);
                sp[S_YYX * N] = a0; sp[S_YYY * N] = a1; sp[S_YYZ * N] = a2;
                snew[1] = (a0 + a1) + a2;
                a0 = split_update<FAST>(o[S_ZZX - S_XXX], dt, l * dXx, kx, mx, px);
                a1 = split_update<FAST>(o[S_ZZY - S_XXX], dt, l * dYy, ky, my, py);
                a2 = split_update<FAST>(o[S_ZZZ - S_XXX], dl, dZz, kz, mz, pz);
                sp[S_ZZX * N] = a0; sp[S_ZZY * N] = a1; sp[S_ZZZ * N] = a2;
                snew[2] = (a0 + a1) + a2;
                const float axy = dt * mxy, axz = dt * mxz, ayz = dt * myz;
                a0 = split_update<FAST>(o[S_XYX - S_XXX], axy, xyX, kx, mx, px);
                a1 = split_update<FAST>(o[S_XYY - S_XXX], axy, xyY, ky, my, py);
                sp[S_XYX * N] = a0; sp[S_XYY * N] = a1;
                snew[3] = a0 + a1;
                a0 = split_update<FAST>(o[S_XZX - S_XXX], axz, xzX, kx, mx, px);
                a1 = split_update<FAST>(o[S_XZZ - S_XXX], axz, xzZ, kz, mz, pz);
                sp[S_XZX * N] = a0; sp[S_XZZ * N] = a1;
                snew[4] = a0 + a1;
                a0 = split_update<FAST>(o[S_YZY - S_XXX], ayz, yzY, ky, my, py);
                a1 = split_update<FAST>(o[S_YZZ - S_XXX], ayz, yzZ, kz, mz, pz);
                sp[S_YZY * N] = a0; sp[S_YZZ * N] = a1;
                snew[5] = a0 + a1;
            }
#pragma unroll
            for (int q = 0; q < 6; ++q) m.f[3 + q][ci] = snew[q];
            if (GEN && gz == rz && it >= 0 && it < sr.nt) {
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
                str_issue<TY>(mybox, nbox, st, &bar[s], cz + S, warp);
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
        const bool gen = t.xy_pml || band(gzp, m.nz, m.pml) != 0 || gzp == sz || gzp == rz;
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
    str_item<FAST, CELLS, false>(mp, m, ph, g, sr, it_arg, src_value, use_wavelet, blockIdx.x, blockIdx.y,
                          align_smem(smem_raw), bar, boxes, pbits);
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

template <bool FAST, int CELLS>
void launch(const Model &m, const Physics &ph, const SourceRec &sr, const ZGeom &g, const ZMaps &zm, int it,
            float src_value, int uw, cudaStream_t s, cudaEvent_t *ev) {
    const dim3 grid(g.ntx * g.nty, g.nchunks);
    if (ev) cudaEventRecord(ev[0], s);
    k_velocity_zmarch<FAST, CELLS><<<grid, NT, vel_smem<CELLS>(), s>>>(zm, m, ph, g, sr, it, src_value, uw);
    if (ev) cudaEventRecord(ev[1], s);
    if (ev) cudaEventRecord(ev[2], s);
    k_stress_zmarch<FAST, CELLS><<<grid, NT, str_smem<CELLS>(), s>>>(zm, m, ph, g, sr, it, src_value, uw);
    if (ev) cudaEventRecord(ev[3], s);
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
    // offsets below 2^31, split offsets (component * npml + PML cell) below 2^32
    const bool small = m.plane * (int64_t)m.nz < ((int64_t)1 << 31) &&
                       (int64_t)kNumSplit * m.npml <= ((int64_t)1 << 32);
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

cudaError_t zmarch_prepare(const Model &m, int cells, size_t st, ZMaps *zm) {
    if (cells != 1 && cells != 2) return cudaErrorInvalidValue;
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
    ok &= make_pool_map(&zm->s_own, m.f[3], m, st, StrL<8>::NOWN, W32, ty);
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
                        int it, float src_value, bool use_wavelet, cudaStream_t s, cudaEvent_t *ev) {
    const int uw = use_wavelet ? 1 : 0;
    if (ph.fast) {
        if (g.cells == 1) launch<true, 1>(m, ph, sr, g, zm, it, src_value, uw, s, ev);
        else launch<true, 2>(m, ph, sr, g, zm, it, src_value, uw, s, ev);
    } else {
        if (g.cells == 1) launch<false, 1>(m, ph, sr, g, zm, it, src_value, uw, s, ev);
        else launch<false, 2>(m, ph, sr, g, zm, it, src_value, uw, s, ev);
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
