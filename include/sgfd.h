/*
 * sgfd.h — C ABI of the B200 staggered-grid elastic solver (libsgfd.so).
 *
 * One handle = one 3-D velocity–stress model on one GPU: 9 wavefields
 * (vx, vy, vz, txx, tyy, tzz, txy, txz, tyz), the medium (buoyancy, lambda,
 * mu), the split-field PML state, one explosive point source and a list of
 * receivers.  The time step is 10th-order staggered differences in space and
 * leapfrog in time, the scheme of the reference's single-GPU PML program
 * (3DGPUwithPML_1DArraySingleGPU_optimization/, cited as OPT/ below).
 *
 * Geometry follows the reference GRID convention: nx, ny, nz count every
 * allocated cell, including a 5-cell frame on each side that is never
 * updated (OPT/ElasticMacro.h:30-39).  Cells [5, n-5) are computed; the outer
 * `pml` cells of that range form the absorbing layer.  Host arrays are
 * x-fastest, index = ix + iy*nx + iz*nx*ny (OPT/ElasticMacro.h:22).
 *
 * Every call returns an sgfd_status; nothing exits the process.  The last
 * error message of a handle is returned by sgfd_last_error().  A handle is
 * not thread-safe; distinct handles are independent.
 *
 * Reference interfaces replaced (file:line in the reference project):
 *   sgfd_create          ElasticWaveEquation::ElasticWaveEquation  OPT/ElasticWaveEquation.cu:8-45
 *                        + calStartEndPoint / vsPMLCPUTovsPML      OPT/ElasticWaveEquation.cu:47-113
 *   sgfd_set_medium      the medium upload in run()               OPT/ElasticWaveEquation.cu:143-147
 *   sgfd_set_source      sourceLocationCPUTosourceLocationGPU     OPT/ElasticWaveEquation.cu:115-118
 *   sgfd_set_receivers   stationLocationCPUTostationLocationGPU   OPT/ElasticWaveEquation.cu:120-123
 *   sgfd_ricker_ref      ElasticWaveEquation::sourceFunction      OPT/ElasticWaveEquation.cu:184-189
 *   sgfd_step            ElasticWaveEquation::propagate           OPT/ElasticWaveEquation.cu:191-204
 *                        (locateSource, velocityUpdate, stressUpdate, recordStationData:
 *                         OPT/ElasticWaveEquation.cu:206-841)
 *   sgfd_run             the time loop of run()                   OPT/ElasticWaveEquation.cu:153-172
 *   sgfd_get_traces      station D2H copy                         OPT/ElasticWaveEquation.cu:174
 *   sgfd_get_field       snapshot D2H copy                        OPT/ElasticWaveEquation.cu:162
 *   sgfd_destroy         ElasticWaveEquation::~ElasticWaveEquation OPT/ElasticWaveEquation.cu:125-138
 */
#ifndef SGFD_H
#define SGFD_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SGFD_ABI_VERSION 1

typedef enum sgfd_status {
    SGFD_OK = 0,
    SGFD_ERR_INVALID = 1,      /* bad argument or configuration */
    SGFD_ERR_ALLOC = 2,        /* device or host allocation failed */
    SGFD_ERR_CUDA = 3,         /* a CUDA runtime call failed */
    SGFD_ERR_STATE = 4,        /* call out of order (e.g. step before set_medium) */
    SGFD_ERR_UNSUPPORTED = 5,  /* option not built into this library */
    SGFD_ERR_NO_DEVICE = 6,    /* no usable CUDA device */
    SGFD_ERR_NONFINITE = 7     /* a NaN/Inf was found in the wavefield */
} sgfd_status;

/* Wavefield ids (also receiver components). */
typedef enum sgfd_field {
    SGFD_VX = 0, SGFD_VY = 1, SGFD_VZ = 2,
    SGFD_TXX = 3, SGFD_TYY = 4, SGFD_TZZ = 5,
    SGFD_TXY = 6, SGFD_TXZ = 7, SGFD_TYZ = 8,
    SGFD_NFIELDS = 9
} sgfd_field;

/* Medium ids for sgfd_get_medium. */
typedef enum sgfd_medium_id {
    SGFD_BUOYANCY = 0, SGFD_LAMBDA = 1, SGFD_MU = 2
} sgfd_medium_id;

/* Damping profiles of the split-field PML.
 *  REFGPU: d = tau*Vs/dx*(8/15 - 0.03 p + p^2/1500)*(k/p)^2, tau=4.3, Vs local
 *          shear velocity sqrt(mu*b), k = 1..p from the inner edge
 *          (OPT/ElasticMacro.h:26-27, OPT/ElasticWaveEquation.cu:282-288).
 *  LOGR:   d = d0*(k/p)^2, d0 = 3*Vp*ln(1/R)/(2*p*dx), Vp local P velocity
 *          sqrt((lambda+2mu)*b); the classic quadratic profile.
 *  REFCPU: d = log10(1/R)*3.4*Vconst/(p*dx)*(k/p)^2 with a constant velocity
 *          (3DCPUwithPML_3DArray_GridIncludePMLandOrder/ElasticMacro.h:18-23). */
/* Regions summed by sgfd_energy. */
typedef enum sgfd_region {
    SGFD_REGION_COMPUTED = 0,   /* interior + PML shell */
    SGFD_REGION_INTERIOR = 1,
    SGFD_REGION_PML = 2
} sgfd_region;

typedef enum sgfd_damping {
    SGFD_DAMP_REFGPU = 0,
    SGFD_DAMP_LOGR = 1,
    SGFD_DAMP_REFCPU = 2
} sgfd_damping;

/* Medium averaging.  REF keeps the reference's two index quirks:
 *  - the PML velocity split update uses the x-averaged buoyancy for all three
 *    components (OPT/ElasticMacro.h:424-456);
 *  - the harmonic mu average for txz takes mu[ix+1,iy+1,iz] as its fourth
 *    point (OPT/ElasticMacro.h:116-117).
 * FIXED uses the staggered-grid averages for every component. */
typedef enum sgfd_quirks {
    SGFD_QUIRKS_REF = 0,
    SGFD_QUIRKS_FIXED = 1
} sgfd_quirks;

/* Wavefield storage type in HBM (arithmetic is always FP32).  BF16 / F16
 * store every wavefield and its PML splits as 16-bit values with a per-field
 * power-of-two scale 2^e (value = float(stored) * 2^e; binary16 saturates at
 * +-65504), halving the wavefield bytes.  The scales are re-chosen after steps
 * 0, 1, 3, 7, 15, 31, 49 and then every 50 steps from the largest magnitude
 * each field wrote in that step, so that it is stored near 2^7.  16-bit storage
 * runs on the z-marching kernels with 32 x 8 tiles (16-bit boxes staged by
 * TMA and widened once per plane; 64 x 8 tiles through sgfd_set_tile) or,
 * with SGFD_KERNEL_SIMPLE, on the per-cell kernels; all give the same bits.
 * The per-step audit (sgfd_set_audit) is not available with it. */
typedef enum sgfd_storage {
    SGFD_STORE_F32 = 0,
    SGFD_STORE_BF16 = 1,
    SGFD_STORE_F16 = 2
} sgfd_storage;

/* Rounding of the staggered differences.
 *  REF:  sum_i c_i (f[+] - f[-]), then divided by the cell size — the
 *        reference's expression (OPT/ElasticWaveEquation.cu:244-250).
 *  FAST: sum_i (c_i / d) (f[+] - f[-]) with the coefficients divided by the
 *        cell size once on the host, so no division per cell.  Differs from
 *        REF by rounding only (relative L2 of traces well below 1e-5). */
typedef enum sgfd_arith {
    SGFD_ARITH_REF = 0,
    SGFD_ARITH_FAST = 1
} sgfd_arith;

/* Kernel family.  AUTO picks the fastest built variant for the storage type. */
typedef enum sgfd_kernel {
    SGFD_KERNEL_AUTO = 0,
    SGFD_KERNEL_SIMPLE = 1,   /* one thread per cell, global loads */
    SGFD_KERNEL_ZMARCH = 2    /* 2.5-D z-marching, TMA-staged xy planes */
} sgfd_kernel;

typedef struct sgfd_config {
    int32_t nx, ny, nz;       /* GRID incl. the 5-cell frame (reference GRID) */
    int32_t pml;              /* PML width in cells (reference `pml`) */
    float dt, dx, dy, dz;     /* reference Delta {t, x, y, z} */
    float coef[5];            /* staggered difference coefficients (reference diff_coef) */
    int32_t damping;          /* sgfd_damping */
    float damping_R;          /* reflection coefficient for LOGR / REFCPU (reference R = 0.001) */
    float damping_vconst;     /* constant velocity for REFCPU (reference 2000) */
    int32_t quirks;           /* sgfd_quirks */
    int32_t storage;          /* sgfd_storage */
    int32_t kernel;           /* sgfd_kernel */
    int32_t device;           /* CUDA device ordinal */
    int32_t arith;            /* sgfd_arith */
    int32_t nz_total;         /* 0: the handle is a whole model; else the GRID z extent of the
                                 whole model this handle is a z-slab of (see sgfd_halo_pack) */
    int32_t z_offset;         /* z-slab: computed planes of the whole model below the slab */
    int32_t reserved[5];      /* must be zero */
} sgfd_config;

typedef struct sgfd_solver sgfd_solver;

/* Fill *cfg with the reference defaults: coefficients of the reference
 * main.cu (CON/main.cu:40-44), REFGPU damping, REF quirks, FP32, AUTO. */
void sgfd_config_default(sgfd_config *cfg);

int sgfd_abi_version(void);

/* Create a solver and allocate its device state (fields zeroed). */
int sgfd_create(const sgfd_config *cfg, sgfd_solver **out);
void sgfd_destroy(sgfd_solver *h);
const char *sgfd_last_error(const sgfd_solver *h);
/* Message for errors where no handle exists (e.g. sgfd_create failures). */
const char *sgfd_global_error(void);

/* Use this CUDA stream (a cudaStream_t passed as void*) for all device work
 * of the handle; NULL selects the handle's own stream. */
int sgfd_set_stream(sgfd_solver *h, void *stream);

/* Upload the medium from HOST arrays of nx*ny*nz floats (x fastest). */
int sgfd_set_medium(sgfd_solver *h, const float *buoyancy, const float *lambda,
                    const float *mu);
/* Same from DEVICE arrays with the same dense layout. */
int sgfd_set_medium_device(sgfd_solver *h, const float *buoyancy,
                           const float *lambda, const float *mu);

/* Explosive point source added to txx, tyy, tzz as dt*dt*s(it) before the
 * velocity update of step it (OPT/ElasticWaveEquation.cu:206-221). */
int sgfd_set_source(sgfd_solver *h, int32_t x, int32_t y, int32_t z);

/* Receivers: n points (xyz[3*i..3*i+2]) each recording component comp[i]
 * (sgfd_field) into a trace of nt samples.  Velocity components are sampled
 * after the velocity update of step it, stresses after the stress update
 * (OPT/ElasticWaveEquation.cu:223-232).  Replaces any earlier receiver set
 * and zeroes the traces. */
int sgfd_set_receivers(sgfd_solver *h, int32_t n, const int32_t *xyz,
                       const int32_t *comp, int32_t nt);

/* Source wavelet for sgfd_run: values[it] for it in [0, nt). */
int sgfd_set_wavelet(sgfd_solver *h, int32_t nt, const float *values);

/* One time step with a host-supplied source value (reference propagate()). */
int sgfd_step(sgfd_solver *h, int32_t it, float source_value);

/* Steps it0 .. it0+nsteps-1 with the wavelet of sgfd_set_wavelet.
 * Asynchronous on the handle's stream.  With use_graph != 0, runs of 16
 * steps replay one captured CUDA graph whose kernels take the step index
 * from a device counter; the graph is captured on first use and again after
 * any setter changes what the kernels are given.  Results are identical to
 * sgfd_step with the wavelet's values. */
int sgfd_run(sgfd_solver *h, int32_t it0, int32_t nsteps, int32_t use_graph);
/* Capture (if out of date) and upload the graph of sgfd_run now, so that the
 * next sgfd_run with use_graph != 0 starts replaying at once. */
int sgfd_prepare_run(sgfd_solver *h);

int sgfd_synchronize(sgfd_solver *h);

/* Zero all wavefields, PML state and traces (medium, source, receivers kept). */
int sgfd_reset(sgfd_solver *h);

/* Overwrite one wavefield from a host array (nx*ny*nz, x fastest): initial
 * conditions, or a state taken from another run.  The 5-cell frame should
 * hold zeros, as the reference's does. */
int sgfd_set_field(sgfd_solver *h, int32_t field, const float *src);

/* Copy traces to host: out[r*nt + it] (receiver-major). */
int sgfd_get_traces(sgfd_solver *h, float *out);
/* Copy the n receiver samples of one step `it` to out[0..n) (blocking);
 * the per-step readback of a drop-in loop (OPT/ElasticWaveEquation.cu:153-174). */
int sgfd_get_trace_step(sgfd_solver *h, int32_t it, float *out);
/* Copy the samples of steps it0 .. it0+n-1 to out[(it - it0)*nrec + r]
 * (time-major, as recorded) in one transfer, waiting for the steps queued
 * before it: the station readback at the end of a run
 * (OPT/ElasticWaveEquation.cu:174, stationDataOutput :950-960) for only the
 * steps taken.  out may be pinned memory. */
int sgfd_get_trace_range(sgfd_solver *h, int32_t it0, int32_t n, float *out);
/* Copy one wavefield (sgfd_field) to a host array of nx*ny*nz floats. */
int sgfd_get_field(sgfd_solver *h, int32_t field, float *out);
/* Copy one medium array (sgfd_medium_id) back to host (nx*ny*nz floats). */
int sgfd_get_medium(sgfd_solver *h, int32_t which, float *out);

/* Reference Ricker wavelet value of step it (OPT/ElasticWaveEquation.cu:184-189):
 * t0 = ceil(1/(f0*dt)); a = pi*f0*((it - t0)*dt - 1/f0); (1 - 2a^2)*exp(-a^2). */
float sgfd_ricker_ref(float f0, float dt, int32_t it);
/* Ricker wavelet with an explicit delay t0 (seconds): a = pi*f0*(it*dt - t0). */
float sgfd_ricker_t0(float f0, float dt, float t0, int32_t it);

/* Steps it0 .. it0+nsteps-1 (wavelet source) with CUDA events around each
 * kernel; returns the summed device time of the velocity-update and the
 * stress-update kernels in milliseconds.  Blocking.  For roofline accounting. */
int sgfd_profile(sgfd_solver *h, int32_t it0, int32_t nsteps, float *ms_velocity, float *ms_stress);

/* z-marching kernels: planes per z chunk (0 = automatic).  Larger chunks
 * re-read fewer warm-up planes; smaller ones give more CTAs to balance. */
int sgfd_set_zchunk(sgfd_solver *h, int32_t planes);

/* Switch the kernel family of an existing handle (SGFD_KERNEL_AUTO means
 * z-marching).  z-marching is available when the handle was created with
 * AUTO or ZMARCH on a supported grid; otherwise SGFD_ERR_UNSUPPORTED.
 * Results are bit-identical across families. */
int sgfd_set_kernel(sgfd_solver *h, int32_t kernel);

/* z-marching kernels: tile height in cells (8 or 16; one or two cells per
 * thread) and planes per z chunk (0 = automatic).  No effect on the simple
 * family.  Results do not depend on the tiling.  Same as sgfd_set_tile with
 * 32 tile columns. */
int sgfd_set_tiling(sgfd_solver *h, int32_t tile_rows, int32_t zchunk);
/* z-marching kernels: tile shape and planes per z chunk (0 = automatic).
 * 32 x 8 and 32 x 16: one or two y-adjacent cells per thread; 64 x 8: two
 * x-adjacent cells per thread, differences and updates of the pair on packed
 * FP32x2.  16-bit storage: 32 x 8 or 64 x 8.  Results do not depend on the
 * tiling (bit-identical). */
int sgfd_set_tile(sgfd_solver *h, int32_t tile_cols, int32_t tile_rows, int32_t zchunk);
/* The z-marching tile shape and z chunk in use (zeros for the simple family). */
int sgfd_get_tile(const sgfd_solver *h, int32_t *tile_cols, int32_t *tile_rows, int32_t *zchunk);

/* ---- z-slabs: one model split along z over several handles, on one GPU or
 * one handle per GPU (no counterpart in the reference, whose model must fit
 * one GPU and whose 32-bit `memsize` caps it at 2^29 cells:
 * OPT/ElasticWaveEquation.cu:20,143) ----
 * A handle created with nz_total != 0 holds computed planes [z_offset,
 * z_offset + nz - 10) of a model whose GRID has nz_total planes; every slab of
 * the model has the same nx, ny, pml and physics.  The PML is the whole
 * model's: z bands only where the slab reaches the model's z ends, damping
 * distances and the compact split order counted in the whole model.  At a cut
 * between two slabs, each slab's 5 frame planes hold its neighbour's values
 * (the reach of the 10th-order z differences): before every velocity update
 * the neighbour's txz, tyz, tzz (SGFD_HALO_STRESS), before every stress update
 * its vx, vy, vz (SGFD_HALO_VELOCITY).  sgfd_halo_pack copies the slab's own 5
 * computed planes beside a cut (3 fields, sgfd_halo_bytes in all) to a DEVICE
 * buffer; sgfd_halo_unpack writes a received buffer into the 5 frame planes
 * on that side.  The caller moves the buffer to the neighbour: a device copy
 * between slabs on one GPU, NCCL send/recv or a peer copy between GPUs.  Both
 * are ordered on the handle's stream.  A step of the whole model is then, per
 * slab: exchange STRESS, sgfd_step_phase(VELOCITY), exchange VELOCITY,
 * sgfd_step_phase(STRESS), and the slabs together give the whole model's
 * results bit for bit (sgfd_step_phase_part splits each half step so that
 * its inner part runs while the halos travel).  Each slab is given the whole model's medium on its
 * GRID planes (frame planes included), the receivers that lie in its planes,
 * and the source if it lies there; the source must lie 5 or more computed
 * planes from every cut (its injection is not part of the exchanged planes).
 * Slabs have FP32 storage, the z-marching kernels with 32-column tiles or the simple kernels,
 * no learned strip and no per-step audit. */
#define SGFD_HALO_LOW 0        /* the cut below the slab (smaller z) */
#define SGFD_HALO_HIGH 1       /* the cut above it */
#define SGFD_HALO_STRESS 0     /* txz, tyz, tzz: exchanged before the velocity update */
#define SGFD_HALO_VELOCITY 1   /* vx, vy, vz: exchanged before the stress update */
#define SGFD_PHASE_VELOCITY 0  /* source injection, velocity update, velocity receivers */
#define SGFD_PHASE_STRESS 1    /* stress update, stress receivers */
int sgfd_halo_bytes(const sgfd_solver *h, int64_t *bytes);
int sgfd_halo_pack(sgfd_solver *h, int32_t side, int32_t kind, void *dst);
int sgfd_halo_unpack(sgfd_solver *h, int32_t side, int32_t kind, const void *src);
/* Half of sgfd_step: SGFD_PHASE_VELOCITY then SGFD_PHASE_STRESS with the same
 * it and source value is one step.  Any handle (whole model or slab). */
int sgfd_step_phase(sgfd_solver *h, int32_t it, float source_value, int32_t phase);
/* Part of a half step, to overlap a slab's halo exchange with its own work.
 * SGFD_PART_INNER updates the planes 5 or more computed planes from both ends
 * of the handle's planes (z chunks of the z-marching kernels, planes of the
 * simple ones): they read no frame plane, so they may run while the halos are
 * in flight.  SGFD_PART_OUTER updates the rest, after the unpack.  Run INNER
 * before OUTER (the simple kernels inject the source with INNER and record
 * the receivers with OUTER); INNER | OUTER is sgfd_step_phase. */
#define SGFD_PART_INNER 1
#define SGFD_PART_OUTER 2
int sgfd_step_phase_part(sgfd_solver *h, int32_t it, float source_value, int32_t phase, int32_t parts);

/* ---- autotuning and batches (no counterpart in the reference, which runs
 * one model with a fixed launch shape: OPT/main.cu's GPUDim) ---- */

/* Result of sgfd_autotune: the fastest candidate and its measured time. */
typedef struct sgfd_tuning {
    int32_t kernel;       /* SGFD_KERNEL_SIMPLE or SGFD_KERNEL_ZMARCH */
    int32_t tile_rows;    /* z-marching tile height: 8 or 16 */
    int32_t zchunk;       /* planes per z chunk; 0 = automatic */
    int32_t candidates;   /* candidates timed */
    float ms_per_step;    /* mean step time of the chosen candidate */
    int32_t tile_cols;    /* z-marching tile width: 32 or 64 */
    int32_t reserved[2];
} sgfd_tuning;

/* Time the launch-shape candidates (kernel family = halo staging through
 * TMA + shared memory or through the caches; tiles 32 x 8, 32 x 16, 64 x 8; z chunk of
 * automatic, 16, 32, 64 planes) over probe_steps steps each (0 = 4), keep the
 * fastest, then zero the wavefields, splits and traces (as sgfd_reset), since
 * timing steps the model.  Call it after sgfd_set_medium and before the run.
 * Results never depend on the choice (bit-identical). */
int sgfd_autotune(sgfd_solver *h, int32_t probe_steps, sgfd_tuning *out);

/* A batch advances several independent models (uneven sizes allowed, all on
 * one device) together: one CUDA graph per 16 steps holds every model's
 * kernels in parallel branches, so small models fill the GPU side by side.
 * Each model keeps its own medium, source, receivers and wavelet (set through
 * its handle before the run); the batch only launches.  The models stay
 * owned by the caller and must outlive the batch. */
typedef struct sgfd_batch sgfd_batch;
int sgfd_batch_create(sgfd_solver *const *models, int32_t n, sgfd_batch **out);
void sgfd_batch_destroy(sgfd_batch *b);
const char *sgfd_batch_last_error(const sgfd_batch *b);
/* Steps it0 .. it0+nsteps-1 of every model, from each model's wavelet.
 * Ordered after work already queued on the models' streams, and work queued
 * on them afterwards waits for it; asynchronous otherwise. */
int sgfd_batch_run(sgfd_batch *b, int32_t it0, int32_t nsteps);
int sgfd_batch_synchronize(sgfd_batch *b);
/* Persistent mode (on != 0): each sgfd_batch_run becomes ONE cooperative
 * launch that runs all its steps for all models.  The CTAs that fit on the
 * GPU at once take the models' (tile, z chunk) work items, 32 x 8 tiles, from
 * a global counter, velocity phase and stress phase in turn, with a grid
 * barrier between phases.  Results are bit-identical to the models' own
 * runs.  Requires FP32 storage, z-marching kernels, no learned strip and no
 * per-step audit on every model, and one rounding mode for all.  The models
 * are switched to the 32 x 8 tiling.  Every wait is bounded: a grid barrier
 * that does not complete within about a second ends the launch, and
 * sgfd_batch_synchronize reports SGFD_ERR_CUDA.  barrier_ctas = 0 waits for
 * the CTAs launched; another value sets the number of arrivals each barrier
 * waits for (a diagnostic of the bounded wait).  on = 0 returns to graph
 * replays. */
int sgfd_batch_set_persistent(sgfd_batch *b, int32_t on, int32_t barrier_ctas);
/* The batch's launch stream (a cudaStream_t), for timing with events. */
void *sgfd_batch_stream(sgfd_batch *b);
/* Kernel launches one sgfd_batch_run(b, *, nsteps) issues. */
int sgfd_batch_run_launches(const sgfd_batch *b, int32_t nsteps);

/* ---- learned absorbing strip (no counterpart in the reference) ----
 * A model created with pml = 0 ends at the zero frame.  sgfd_set_learned_strip
 * makes its outer `width` computed cells a learned absorbing strip: after
 * every step each strip cell's 9 fields get a correction predicted by an MLP
 * (252 inputs: the 9 fields of the cell's 3x3x3 neighbourhood, velocities times
 * rho*vp, over their RMS s; vp/3000, vs/1732, rho/2000; per axis the depth into
 * the strip over width and the side; 64 and 64 GELU units; 9 outputs times s,
 * velocities divided back by rho*vp).  params: sgfd_mlp_param_count() floats,
 * W1[252][64], b1[64], W2[64][64], b2[64], W3[64][9], b3[9].  width 0 removes
 * the strip.  FP32 storage only.  The network runs on the tensor cores with
 * FP16 operands and FP32 accumulation (see sgfd_mlp_infer). */
int sgfd_set_learned_strip(sgfd_solver *h, int32_t width, const float *params);
/* The 252 MLP inputs of n strip cells (computed coordinates cx, cy, cz per
 * cell) from the current state, with each cell's s and rho*vp (training data). */
int sgfd_strip_features(sgfd_solver *h, int32_t width, int32_t n, const int32_t *cells, float *X, float *scale,
                        float *zimp);
/* Training data for the strip (no counterpart in the reference).
 * sgfd_copy_window: dst's 9 fields (its whole GRID) from the window of src
 * whose GRID origin is (x0, y0, z0), with dst's 5-cell frame set to zero; both
 * models FP32 on one device, dst with pml = 0; ordered after the work queued
 * on both models' streams.  sgfd_sample_fields: the 9 fields of n cells
 * (computed coordinates cx, cy, cz per cell) to out[i*9 + k]; waits for the
 * queued steps. */
int sgfd_copy_window(sgfd_solver *dst, sgfd_solver *src, int32_t x0, int32_t y0, int32_t z0);
int sgfd_sample_fields(sgfd_solver *h, int32_t n, const int32_t *cells, float *out);
/* The MLP on the GPU of `device`, host arrays in and out: parameter count,
 * forward pass of n input rows, loss (mean squared error over the 9 outputs)
 * and its gradient for n rows, and minibatch Adam training (lr, betas 0.9 and
 * 0.999) over `epochs` passes of the n rows in order, params updated in place
 * and the mean minibatch loss of every epoch in epoch_loss. */
int sgfd_mlp_param_count(void);
int sgfd_mlp_forward(int32_t device, const float *params, const float *X, int64_t n, float *out);
/* The strip's inference path on n given input rows: the three layers on the
 * tensor cores with FP16 operands (inputs, weights and hidden activations
 * rounded to binary16) and FP32 accumulation, outputs before the energy limit
 * and the scale s.  Checks the tensor-core path on inputs of the caller's
 * choosing; n <= 2^30. */
int sgfd_mlp_infer(int32_t device, const float *params, const float *X, int64_t n, float *out);
int sgfd_mlp_gradient(int32_t device, const float *params, const float *X, const float *Y, int32_t n, float *loss,
                      float *grad);
int sgfd_mlp_train(int32_t device, float *params, const float *X, const float *Y, int64_t n, int32_t epochs,
                   int32_t batch, float lr, float *epoch_loss);

/* FP64 energy audit (no counterpart in the reference): kinetic
 * 1/2 rho |v|^2 and strain energy (s:s - lambda/(3 lambda + 2 mu) tr(s)^2) /
 * (4 mu) of the current wavefield, fields and medium taken at the same cell,
 * summed in FP64 on the GPU over the computed cells of `region` and
 * multiplied by dx*dy*dz.  Waits for the handle's queued steps.  Energy left
 * in SGFD_REGION_INTERIOR after the direct wave has left the interior is what
 * the absorbing boundary reflected.  In a model with a learned strip
 * (pml = 0) the strip takes the PML's place in the regions. */
int sgfd_energy(sgfd_solver *h, int32_t region, double *kinetic, double *strain);

/* sgfd_energy without any allocation; no counterpart in the reference.
 * For callers that cannot let the library call cudaMalloc once they are
 * running (device memory held by another allocator such as PyTorch's caching
 * allocator, or a footprint fixed when the handles were created): the
 * partial sums go to a 32 KiB device array compiled into the library, at
 * most 2047 partial-sum blocks; nblocks = 0 uses sgfd_energy's launch shape
 * capped at 2047 blocks, a larger nblocks than 2047 is rejected
 * (SGFD_ERR_INVALID).  The first call on a device looks up that array's
 * address; make it before any stream capture (a call that finds a new CUDA
 * context on the device, e.g. after cudaDeviceReset, looks it up again).
 * All calls share the array: calls that overlap on one GPU race. */
int sgfd_energy_noalloc(sgfd_solver *h, int32_t region, int32_t nblocks, double *kinetic, double *strain);

/* Per-step FP64 energy audit.  With every > 0, after the stress update of
 * each step it with it % every == 0 and it / every < nsamples, the kinetic
 * and strain energy of `region` (as sgfd_energy) are recorded on the GPU as
 * sample it / every; the history is zeroed here and by sgfd_reset.  Works in
 * sgfd_step, sgfd_run (graphs included) and batches; adds two launches per
 * step.  every = 0 switches it off. */
int sgfd_set_audit(sgfd_solver *h, int32_t every, int32_t region, int32_t nsamples);
/* Copy the history: out[2k] kinetic, out[2k+1] strain energy of sample k. */
int sgfd_get_audit(sgfd_solver *h, double *out);

/* ---- checkpoint / resume (no counterpart in the reference, which writes
 * only text slices: OPT/ElasticWaveEquation.cu:843-948) ----
 * A checkpoint holds the dynamic state: the 9 wavefields, the 24 PML split
 * fields, the traces and the caller's next step index it_next.  The static
 * inputs (medium, source, receivers, wavelet) are not in it: a resuming
 * handle is created with the same configuration, given the same inputs, then
 * loads the checkpoint and continues with step it_next.  Layout: a 128-byte
 * header (magic "SGFDCKP1", version 1, grid, pml, receivers x steps, it_next,
 * physics, payload size, 64-bit checksum, storage type, the 16-bit field
 * scales and, for a z-slab, its place in the whole model), then the payload: 9 x nx*ny*nz
 * float32 fields (x fastest), 24 x npml float32 splits, nt x nrec float32
 * traces (time-major).  Loading checks the grid, physics and checksum; a
 * checksum or length failure zeroes the state (as sgfd_reset) and returns
 * SGFD_ERR_INVALID.  All four wait for the handle's queued steps. */
int sgfd_checkpoint_bytes(sgfd_solver *h, int64_t *bytes);
int sgfd_checkpoint_save(sgfd_solver *h, int32_t it_next, void *buf, int64_t bytes);
int sgfd_checkpoint_load(sgfd_solver *h, const void *buf, int64_t bytes, int32_t *it_next);
int sgfd_checkpoint_write(sgfd_solver *h, int32_t it_next, const char *path);
int sgfd_checkpoint_read(sgfd_solver *h, const char *path, int32_t *it_next);

/* Multi-component station files, extending the reference's single txx
 * stationData.txt (OPT/ElasticWaveEquation.cu:950-960):
 *   <prefix>_receivers.txt   one line per receiver: index x y z component column
 *   <prefix>_<comp>.txt      for each recorded component (vx vy vz txx tyy tzz
 *                            txy txz tyz): nsteps lines, one column per
 *                            receiver of that component in receiver order,
 *                            values printed as %g (the reference's ofstream
 *                            format)
 *   <prefix>_<comp>.bin      with binary != 0: int32 nsteps, int32 ncols, then
 *                            float32 [nsteps][ncols]
 * nsteps = 0 writes all nt steps of sgfd_set_receivers. */
int sgfd_write_stations(sgfd_solver *h, const char *prefix, int32_t nsteps, int32_t binary);

/* Counts for roofline accounting: computed cells that are interior / PML. */
int sgfd_cell_counts(const sgfd_solver *h, int64_t *n_interior, int64_t *n_pml);
/* Device allocations (cudaMalloc calls) the handle has made since
 * sgfd_create, counting those freed since; no counterpart in the reference.
 * A caller that must not see the library allocate once it runs can check
 * that this count stays put across its steady-state calls. */
int sgfd_device_allocations(const sgfd_solver *h, int64_t *count);
/* Number of kernel launches issued by one sgfd_step / one step of sgfd_run. */
int sgfd_launches_per_step(const sgfd_solver *h);
/* Number of kernel launches sgfd_run(h, *, nsteps, use_graph) issues. */
int sgfd_run_launches(const sgfd_solver *h, int32_t nsteps, int32_t use_graph);
/* Name of the kernel family in use ("simple", "zmarch"). */
const char *sgfd_kernel_name(const sgfd_solver *h);

#ifdef __cplusplus
}
#endif

#endif /* SGFD_H */
