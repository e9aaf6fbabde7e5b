// zmarch.h — host interface of the z-marching kernel family (kernels_zmarch.cu).
#pragma once

#include <cuda.h>

#include "sgfd_internal.h"

namespace sgfd {

// Single-cell tiling (kernels_zmarch.cu): tiles 32 computed cells wide and
// 8 * cells high (cells = 1 or 2 per thread, stacked along y).
constexpr int kZTileX = 32;
// Paired tiling (kernels_zpair.cu): tiles 64 x 8, two x-adjacent cells per thread.
constexpr int kPairTileX = 64;

// TMA descriptors of the single-cell z-march kernels: 4-D maps over the array
// pool (x, y, z, array), so that arrays one update reads with the same box
// shape at the same plane arrive in one copy (one box per map and plane).
// Arrays of one map are evenly spaced in the pool; the stress update's own
// cell arrays (txx..tyz, lambda, mu, mxy, mxz, myz) are 11 consecutive ones.
struct ZMaps {
    // velocity update, plane z: sigma_xx + sigma_xz (48 x TY), sigma_yy +
    // sigma_yz (32 x TY+10), sigma_xy (48 x TY+10), buoyancy (36 x TY+1);
    // lead planes: sigma_xz + sigma_yz at z+4, sigma_zz at z+5, buoyancy at
    // z+1; own vx, vy, vz (32 x TY each)
    CUtensorMap v_sxx_sxz, v_syy_syz, v_sxy, v_b, v_lead_xz_yz, v_lead_zz, v_lead_b, v_own;
    // stress update: vx, vy, vz (48 x TY+10); lead vx + vy at z+5, vz at z+4;
    // own txx..myz (11 arrays, 32 x TY each; with 16-bit storage the 6
    // stored stresses in s_own and the FP32 lambda..myz in s_med)
    CUtensorMap s_v, s_lead_xy, s_lead_z, s_own, s_med;
};

// TMA descriptors of the paired velocity update (kernels_zpair.cu): x/y-halo
// boxes of the current plane and centre boxes of the planes that feed the z
// register queues.
struct VelMaps {
    CUtensorMap sxx, syy, sxy, sxz, syz, b;      // current plane
    CUtensorMap sxz_c, syz_c, szz_c, b_c;        // lead planes (centre boxes)
    CUtensorMap own[3];                          // own-cell vx, vy, vz (centre boxes)
};
// TMA descriptors of the paired stress update.
struct StrMaps {
    CUtensorMap vx, vy, vz;                      // current plane
    CUtensorMap vx_c, vy_c, vz_c;                // lead planes
    static constexpr int kOwn = 11;
    CUtensorMap own[kOwn];                       // own-cell txx..tyz, lambda, mu, mxy, mxz, myz
};

// Launch geometry: tiles of kZTileX x (8 * cells) computed cells, z chunks of
// zc planes; receivers bucketed per tile and sorted by z.
struct ZGeom {
    int pair;               // 1: paired tiling (64 x 8 tiles), 0: single-cell tiling
    int tw;                 // tile width in computed cells (kZTileX or kPairTileX)
    int cells;
    int ntx, nty;
    int zc, nchunks;
    int c0;                 // first z chunk of this launch (blockIdx.y = chunk - c0); 0 for a whole half step
    const int *rec_off;     // ntx*nty + 1 offsets into rec_list / rec_idx
    const int4 *rec_list;   // GRID x, y, z, component
    const int *rec_idx;     // receiver index (trace column)
    int *err;               // device error flag (1: a bounded wait gave up)
};

// 3-D FP32 tensor map over one padded device array with a bx x by x 1 box;
// the same over a 16-bit array of the same layout.
bool make_box_map(CUtensorMap *map, const float *grid_origin, const Model &m, int bx, int by);
bool make_box_map16(CUtensorMap *map, const uint16_t *grid_origin, const Model &m, int bx, int by);

// zmarch_prepare: the maps of the single-cell family over the model's array
// pool, whose arrays are array_stride bytes apart in the order the stress
// update reads them (cudaErrorInvalidValue when the pointers are otherwise);
// with hs (16-bit storage, cells = 1), the wavefield maps cover the 16-bit
// arrays, stride16 bytes apart.  zmarch_step: one step (velocity + stress);
// with hs also the 16-bit source, receiver and rescale kernels.  phases
// (FP32 storage): bit 0 the velocity update, bit 1 the stress update; parts
// (FP32 storage): kPartInner the z chunks whose planes read no frame plane,
// kPartOuter the others.
bool zmarch_supported(const Model &m);
cudaError_t zmarch_prepare(const Model &m, int cells, size_t array_stride, ZMaps *zm, const HalfState *hs = nullptr,
                           size_t stride16 = 0);
void zmarch_tiles(const Model &m, int cells, int *ntx, int *nty);
cudaError_t zmarch_step(const Model &m, const Physics &ph, const SourceRec &sr, const ZGeom &g, const ZMaps &zm,
                        int it, float src_value, bool use_wavelet, cudaStream_t s, cudaEvent_t *ev = nullptr,
                        const HalfState *hs = nullptr, int phases = 3, int parts = 3);
// One model of a persistent batch, in device memory (the kernel's TMA reads
// its tensor maps from there: 64-byte alignment).  Its work items are the
// (tile, z chunk) pairs of the single-cell 32 x 8 tiling, tile fastest.
struct alignas(64) ZModel {
    ZMaps zm;
    Model m;
    Physics ph;
    ZGeom g;
    SourceRec sr;       // it_dev null: the kernel passes the step index
    int items;          // tiles x z chunks
};
// Status words of a persistent batch launch (device int): 1 a TMA wait gave
// up (the model's own flag is set too), 2 a grid barrier wait gave up.
constexpr int kBatchWaitTma = 1, kBatchWaitGrid = 2;

// Persistent batch: CTAs that fit at once on the device (cooperative launch),
// and nsteps steps of all models in one launch.  first_item[nmodels + 1]:
// prefix sums of the models' items; ctl: 1 + 2 * nsteps zeroed counters
// (grid-barrier arrivals, then one work counter per step and phase); each
// grid barrier waits for barrier_ctas arrivals (the launched CTAs unless a
// caller asks otherwise), at most about a second, then the launch stops with
// *status = kBatchWaitGrid.  All models FAST or all REF (fast).
int zmarch_batch_ctas(int device);
cudaError_t zmarch_batch_run(const ZModel *models, int nmodels, const int *first_item, int it0, int nsteps,
                             unsigned *ctl, int barrier_ctas, int ctas, bool fast, int *status, cudaStream_t s);

// Paired tiling: tensor maps, tile counts and one step (velocity + stress).
// hs: null for FP32 storage, else the 16-bit storage state (the step then
// also launches the 16-bit source, receiver and rescale kernels).
cudaError_t zpair_prepare(const Model &m, const HalfState *hs, VelMaps *vm, StrMaps *sm);
void zpair_tiles(const Model &m, int *ntx, int *nty);
cudaError_t zpair_step(const Model &m, const Physics &ph, const SourceRec &sr, const HalfState *hs, const ZGeom &g,
                       const VelMaps &vm, const StrMaps &sm, int it, float src_value, bool use_wavelet, cudaStream_t s,
                       cudaEvent_t *ev = nullptr);

}  // namespace sgfd
