// solver.h — the handle behind sgfd_solver* and the error helpers shared by
// the translation units of the C ABI (sgfd_api.cu, checkpoint.cu).
#pragma once

#include <string>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "../../include/sgfd.h"
#include "sgfd_internal.h"
#include "zmarch.h"

namespace sgfd {
// Every value a captured step passes to its kernels.  A graph is replayed
// only while a fresh copy compares equal byte for byte; any setter that
// changes a pointer, a size or a tiling therefore forces a new capture.
struct GraphKey {
    Model m;
    Physics ph;
    SourceRec sr;
    ZGeom zg;
    VelMaps vm;
    StrMaps sm;
    ZMaps zm;
    int kernel;
    int audit_every, audit_region, audit_count;
    double *audit_hist, *audit;
    int strip_w, strip_n;
    int4 *strip_cells;   // tiles
    float *strip_buf;
};
// Steps per captured graph; sgfd_run launches the remainder directly.
constexpr int kGraphSteps = 16;

// A named range on the host timeline of the calling thread, from here to the
// end of the scope: what a profiler (Nsight Systems, Nsight Compute's
// --nvtx filters) shows around the launches of a call.  Without a profiler
// attached the calls return at once.
struct TraceRange {
    explicit TraceRange(const char *name) { nvtxRangePushA(name); }
    ~TraceRange() { nvtxRangePop(); }
    TraceRange(const TraceRange &) = delete;
    TraceRange &operator=(const TraceRange &) = delete;
};
}  // namespace sgfd

struct sgfd_solver {
    sgfd_config cfg{};
    sgfd::Model m{};
    sgfd::Physics ph{};
    sgfd::SourceRec sr{};
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaStream_t own_stream = nullptr;
    char *field_pool = nullptr;   // 9 fields, lambda, mu, 3 shear moduli, b, 1/mu
    float *split = nullptr;
    int4 *rec = nullptr;
    float *traces = nullptr;
    float *wavelet = nullptr;
    int wavelet_nt = 0;
    bool medium_set = false;
    int kernel = SGFD_KERNEL_SIMPLE;
    // z-marching family: single-cell maps (zm) or paired maps (vm, sm)
    sgfd::ZMaps zm{};
    sgfd::VelMaps vm{};
    sgfd::StrMaps sm{};
    sgfd::ZGeom zg{};
    int zchunk_req = 0;
    std::vector<int4> rec_host;   // receivers, for re-bucketing when the tiling changes
    int *zrec_off = nullptr;
    int4 *zrec_list = nullptr;
    int *zrec_idx = nullptr;
    int *dev_err = nullptr;
    // CUDA-graph replay of sgfd_run
    cudaStream_t cap_stream = nullptr;
    cudaGraphExec_t graph = nullptr;
    int *step_ctr = nullptr;      // device step counter read by the replayed kernels
    sgfd::GraphKey graph_key{};   // launch parameters the graph was captured with
    // 16-bit wavefield storage (storage != SGFD_STORE_F32): the stored
    // fields and splits and their scale state; Model::f / Model::split then
    // hold FP32 copies made for the read-out paths (sync_views)
    int storage = SGFD_STORE_F32;
    char *h16_pool = nullptr;
    void *hstate = nullptr;
    sgfd::HalfState hs{};
    // learned absorbing strip (pml = 0 models): cells of the strip, then the
    // MLP parameters followed by one correction per cell and field
    int strip_w = 0, strip_n = 0;
    int4 *strip_cells = nullptr;
    float *strip_buf = nullptr;
    // energy audit scratch: 2 doubles per partial block, then the 2 results
    double *audit = nullptr;
    int audit_blocks = 0;
    // per-step audit (sgfd_set_audit): sample k = energy after step k*every
    int audit_every = 0, audit_region = 0, audit_count = 0;
    double *audit_hist = nullptr;
    // device allocations this handle has made since sgfd_create (dev_malloc)
    int64_t dev_allocs = 0;
    std::string err;
};

namespace sgfd {

// Record an error message on the handle (or, with h == nullptr, in the
// thread's global slot read by sgfd_global_error) and return code.
int fail(sgfd_solver *h, int code, const char *fmt, ...);
int cuda_fail(sgfd_solver *h, cudaError_t e, const char *what);
// Null check and cudaSetDevice of the handle's device.
int check_handle(sgfd_solver *h);
// Read and clear the kernels' device error flag.
int check_device_error(sgfd_solver *h);
// 16-bit storage: refresh the FP32 copies Model::f / Model::split from the
// stored values (no-op for FP32 storage), or the stored values from them.
int sync_views(sgfd_solver *h);
int sync_from_views(sgfd_solver *h);
// 16-bit storage: reset the scale state (exponents 0, maxima 0).
int reset_scales(sgfd_solver *h);
// 16-bit storage: exponents of the 9 field scales, to the host / from the host.
int get_scale_exponents(sgfd_solver *h, int *e);
int set_scale_exponents(sgfd_solver *h, const int *e);

// Launch one step of h's kernels on stream s with the given receiver /
// source record (h->sr, or a copy whose it_dev points at a step counter).
cudaError_t dispatch_on(sgfd_solver *h, const SourceRec &sr, cudaStream_t s, int it, float value,
                        bool use_wavelet, cudaEvent_t *ev);
// Byte image of everything a captured step passes to h's kernels.
void graph_key(const sgfd_solver *h, GraphKey *k);

// Learned strip (learned.cu): the strip's tiles (boxes of at most 128 cells),
// the size of its device buffer (weight image, corrections, error flag), the
// error flag inside it, the kernel set-up, and one correction pass (network
// then apply).
int strip_tile_list(const Model &m, int w, std::vector<int4> &tiles);
size_t strip_buffer_bytes(int ntiles);
int *strip_error_flag(float *buf, int ntiles);
cudaError_t strip_prepare();
cudaError_t launch_strip(const Model &m, int w, const int4 *tiles, int ntiles, float *buf, cudaStream_t s);
int mlp_params();

// cudaMalloc on behalf of handle h, counted in h->dev_allocs.
template <class T>
inline cudaError_t dev_malloc(sgfd_solver *h, T **p, size_t bytes) {
    const cudaError_t e = cudaMalloc(reinterpret_cast<void **>(p), bytes);
    if (e == cudaSuccess) ++h->dev_allocs;
    return e;
}

inline size_t round_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

// The model as the energy audit sees it: for a model with a learned strip
// (pml = 0) the strip plays the PML's part in the audit's regions.
inline sgfd::Model audit_model(const sgfd_solver *h) {
    sgfd::Model m = h->m;
    if (m.pml == 0) m.pml = h->strip_w;
    return m;
}

// Bytes of one padded device array (fields and medium share this size).
inline size_t array_bytes(const Model &m) { return round_up((size_t)m.plane * m.nz * sizeof(float), 256); }

}  // namespace sgfd

#define SG_CUDA(h, call, what)                                        \
    do {                                                              \
        cudaError_t e_ = (call);                                      \
        if (e_ != cudaSuccess) return sgfd::cuda_fail(h, e_, what);   \
    } while (0)
