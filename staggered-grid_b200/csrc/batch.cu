// batch.cu — launch-shape autotuning of one model and batches of independent
// models advanced together under one CUDA graph.
//
// The reference runs one model with the launch shape its main.cu hard-codes
// (GPUDim, OPT/main.cu) and synchronises the device after every step
// (OPT/ElasticWaveEquation.cu:201).  Here a batch of uneven models shares the
// GPU: each graph replay holds 16 steps of every model, one parallel branch
// per model (up to kMaxBranches streams, models dealt round-robin), so the
// hardware schedules the small models' CTAs side by side; a device step
// counter, advanced by the graph's last node, gives the kernels their step
// index, as in sgfd_run.  In persistent mode (sgfd_batch_set_persistent) one
// cooperative launch runs all steps of all models instead: its CTAs take the
// models' (tile, z chunk) work items from a global counter, velocity phase
// then stress phase, with a bounded grid barrier between the phases
// (kernels_zmarch.cu, k_batch_zmarch; the models run the 32 x 8 tiling).
#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "solver.h"

using namespace sgfd;

struct sgfd_batch {
    std::vector<sgfd_solver *> models;
    int device = 0;
    cudaStream_t stream = nullptr;   // replays and the remainder steps
    cudaStream_t cap = nullptr;      // capture origin
    std::vector<cudaStream_t> branch;
    cudaEvent_t fork = nullptr, done = nullptr;
    std::vector<cudaEvent_t> join, ev_in;
    cudaGraphExec_t graph = nullptr;
    std::vector<GraphKey> keys;
    int *step_ctr = nullptr;
    // persistent mode: one cooperative launch runs every model's work items
    bool persistent = false;
    bool pfast = false;
    int barrier_ctas = 0;                 // 0: as many as launched
    int ctas = 0;                         // CTAs that fit at once
    ZModel *pdesc = nullptr;              // device copies of the models' descriptors
    int *pfirst = nullptr;                // prefix sums of the models' work items
    unsigned *pctl = nullptr;             // barrier arrivals + work counters
    int pctl_steps = 0;
    int *pstatus = nullptr;
    std::vector<GraphKey> pkeys;          // model state the descriptors were built from
    std::string err;
};

namespace {

constexpr int kMaxBranches = 32;

int bfail(sgfd_batch *b, int code, const char *fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    std::vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    if (b) b->err = buf;
    else fail(nullptr, code, "%s", buf);
    return code;
}

#define BATCH_CUDA(b, call, what)                                                                   \
    do {                                                                                            \
        cudaError_t e_ = (call);                                                                    \
        if (e_ != cudaSuccess) return bfail(b, SGFD_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e_)); \
    } while (0)

void release(sgfd_batch *b) {
    if (b->graph) cudaGraphExecDestroy(b->graph);
    b->graph = nullptr;
}

bool keys_current(const sgfd_batch *b) {
    if (!b->graph) return false;
    for (size_t i = 0; i < b->models.size(); ++i) {
        GraphKey k;
        graph_key(b->models[i], &k);
        if (std::memcmp(&k, &b->keys[i], sizeof k) != 0) return false;
    }
    return true;
}

int capture(sgfd_batch *b) {
    release(b);
    BATCH_CUDA(b, cudaStreamBeginCapture(b->cap, cudaStreamCaptureModeThreadLocal), "begin capture");
    cudaError_t e = cudaEventRecord(b->fork, b->cap);
    const int nb = (int)b->branch.size();
    for (int j = 0; j < nb && e == cudaSuccess; ++j) e = cudaStreamWaitEvent(b->branch[j], b->fork, 0);
    for (size_t i = 0; i < b->models.size() && e == cudaSuccess; ++i) {
        sgfd_solver *h = b->models[i];
        SourceRec sr = h->sr;
        sr.it_dev = b->step_ctr;
        for (int k = 0; k < kGraphSteps && e == cudaSuccess; ++k)
            e = dispatch_on(h, sr, b->branch[i % nb], k, 0.0f, true, nullptr);
    }
    for (int j = 0; j < nb && e == cudaSuccess; ++j) {
        e = cudaEventRecord(b->join[j], b->branch[j]);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(b->cap, b->join[j], 0);
    }
    if (e == cudaSuccess) e = launch_counter(b->step_ctr, kGraphSteps, true, b->cap);
    cudaGraph_t g = nullptr;
    const cudaError_t e_end = cudaStreamEndCapture(b->cap, &g);
    if (e == cudaSuccess) e = e_end;
    if (e == cudaSuccess) e = cudaGraphInstantiate(&b->graph, g, 0);
    if (g) cudaGraphDestroy(g);
    if (e != cudaSuccess) {
        b->graph = nullptr;
        cudaGetLastError();
        return bfail(b, SGFD_ERR_CUDA, "batch graph capture: %s", cudaGetErrorString(e));
    }
    b->keys.resize(b->models.size());
    for (size_t i = 0; i < b->models.size(); ++i) graph_key(b->models[i], &b->keys[i]);
    return SGFD_OK;
}

// Whether a model can run in a persistent batch (single-cell z-march tiling).
const char *persistent_blocker(const sgfd_solver *h) {
    if (h->storage != SGFD_STORE_F32) return "16-bit storage";
    if (!h->dev_err) return "no z-marching kernels on this grid";
    if (h->strip_n > 0) return "a learned strip";
    if (h->audit_every > 0) return "a per-step audit";
    return nullptr;
}

// Device descriptors of the models, rebuilt when a model changed since.
int build_descriptors(sgfd_batch *b) {
    const int n = (int)b->models.size();
    bool current = b->pdesc && (int)b->pkeys.size() == n;
    for (int i = 0; i < n && current; ++i) {
        GraphKey k;
        graph_key(b->models[i], &k);
        current = std::memcmp(&k, &b->pkeys[i], sizeof k) == 0;
    }
    if (current) return SGFD_OK;
    std::vector<ZModel> d(n);
    std::vector<int> first(n + 1, 0);
    for (int i = 0; i < n; ++i) {
        const sgfd_solver *h = b->models[i];
        std::memset(static_cast<void *>(&d[i]), 0, sizeof d[i]);
        d[i].zm = h->zm;
        d[i].m = h->m;
        d[i].ph = h->ph;
        d[i].g = h->zg;
        d[i].sr = h->sr;
        d[i].sr.it_dev = nullptr;
        d[i].items = h->zg.ntx * h->zg.nty * h->zg.nchunks;
        first[i + 1] = first[i] + d[i].items;
    }
    if (!b->pdesc) {
        BATCH_CUDA(b, cudaMalloc(&b->pdesc, (size_t)n * sizeof(ZModel)), "batch descriptors");
        BATCH_CUDA(b, cudaMalloc(&b->pfirst, (size_t)(n + 1) * sizeof(int)), "batch descriptors");
        BATCH_CUDA(b, cudaMalloc(&b->pstatus, sizeof(int)), "batch status");
        BATCH_CUDA(b, cudaMemset(b->pstatus, 0, sizeof(int)), "batch status");
    }
    BATCH_CUDA(b, cudaMemcpy(b->pdesc, d.data(), (size_t)n * sizeof(ZModel), cudaMemcpyHostToDevice),
               "batch descriptors");
    BATCH_CUDA(b, cudaMemcpy(b->pfirst, first.data(), (size_t)(n + 1) * sizeof(int), cudaMemcpyHostToDevice),
               "batch descriptors");
    b->pkeys.resize(n);
    for (int i = 0; i < n; ++i) graph_key(b->models[i], &b->pkeys[i]);
    return SGFD_OK;
}

int run_persistent(sgfd_batch *b, int it0, int nsteps) {
    if (nsteps == 0) return SGFD_OK;
    for (size_t i = 0; i < b->models.size(); ++i) {
        const char *why = persistent_blocker(b->models[i]);
        if (why) return bfail(b, SGFD_ERR_STATE, "model %zu cannot run persistently: %s", i, why);
        const sgfd_solver *h = b->models[i];
        if (h->zg.pair != 0 || h->zg.cells != 1 || (bool)h->ph.fast != b->pfast)
            return bfail(b, SGFD_ERR_STATE, "model %zu changed tiling or rounding since sgfd_batch_set_persistent", i);
    }
    int r = build_descriptors(b);
    if (r) return r;
    if (nsteps > b->pctl_steps) {
        cudaFree(b->pctl);
        b->pctl = nullptr;
        b->pctl_steps = 0;
        BATCH_CUDA(b, cudaMalloc(&b->pctl, (size_t)(1 + 2 * nsteps) * sizeof(unsigned)), "batch counters");
        b->pctl_steps = nsteps;
    }
    BATCH_CUDA(b, cudaMemsetAsync(b->pctl, 0, (size_t)(1 + 2 * nsteps) * sizeof(unsigned), b->stream),
               "batch counters");
    const int bar = b->barrier_ctas > 0 ? b->barrier_ctas : b->ctas;
    BATCH_CUDA(b, zmarch_batch_run(b->pdesc, (int)b->models.size(), b->pfirst, it0, nsteps, b->pctl, bar, b->ctas,
                                   b->pfast, b->pstatus, b->stream),
               "persistent batch launch");
    return SGFD_OK;
}

}  // namespace

extern "C" {

int sgfd_batch_set_persistent(sgfd_batch *b, int32_t on, int32_t barrier_ctas) {
    if (!b) return fail(nullptr, SGFD_ERR_INVALID, "null batch");
    BATCH_CUDA(b, cudaSetDevice(b->device), "cudaSetDevice");
    if (barrier_ctas < 0) return bfail(b, SGFD_ERR_INVALID, "negative barrier count");
    if (!on) {
        b->persistent = false;
        return SGFD_OK;
    }
    for (size_t i = 0; i < b->models.size(); ++i) {
        const char *why = persistent_blocker(b->models[i]);
        if (why) return bfail(b, SGFD_ERR_UNSUPPORTED, "model %zu cannot run persistently: %s", i, why);
        if ((bool)b->models[i]->ph.fast != (bool)b->models[0]->ph.fast)
            return bfail(b, SGFD_ERR_UNSUPPORTED, "models %zu and 0 differ in rounding mode", i);
    }
    b->ctas = zmarch_batch_ctas(b->device);
    if (b->ctas <= 0) return bfail(b, SGFD_ERR_UNSUPPORTED, "the persistent batch kernel does not fit this device");
    for (size_t i = 0; i < b->models.size(); ++i) {
        sgfd_solver *h = b->models[i];
        if ((h->zg.pair != 0 || h->zg.cells != 1) && sgfd_set_tile(h, kZTileX, 8, h->zchunk_req) != SGFD_OK)
            return bfail(b, SGFD_ERR_CUDA, "model %zu: %s", i, h->err.c_str());
    }
    b->pfast = b->models[0]->ph.fast != 0;
    b->barrier_ctas = barrier_ctas;
    b->persistent = true;
    b->pkeys.clear();
    return SGFD_OK;
}

int sgfd_autotune(sgfd_solver *h, int32_t probe_steps, sgfd_tuning *out) {
    int r = check_handle(h);
    if (r) return r;
    if (!h->medium_set) return fail(h, SGFD_ERR_STATE, "sgfd_set_medium must come before sgfd_autotune");
    if (probe_steps < 0) return fail(h, SGFD_ERR_INVALID, "negative probe length");
    if (probe_steps == 0) probe_steps = 4;
    struct Cand { int kernel, cols, rows, zchunk; };
    std::vector<Cand> cands;
    if (h->dev_err) {
        for (int shape = 0; shape < 3; ++shape) {
            if (shape == 1 && h->storage != SGFD_STORE_F32) continue;   // 16-bit: 32 x 8 and 64 x 8
            for (int zc : {0, 16, 32, 64})
                if (zc == 0 || zc < h->m.nzc)
                    cands.push_back({SGFD_KERNEL_ZMARCH, shape == 2 ? kPairTileX : kZTileX, shape == 1 ? 16 : 8, zc});
        }
    }
    cands.push_back({SGFD_KERNEL_SIMPLE, 0, 8, 0});
    cudaEvent_t e0, e1;
    SG_CUDA(h, cudaEventCreate(&e0), "event");
    if (cudaEventCreate(&e1) != cudaSuccess) {
        cudaEventDestroy(e0);
        return fail(h, SGFD_ERR_CUDA, "event create");
    }
    float best_ms = 0.0f;
    int best = -1;
    for (size_t c = 0; c < cands.size() && r == SGFD_OK; ++c) {
        r = sgfd_set_kernel(h, cands[c].kernel);
        if (r == SGFD_OK && cands[c].kernel == SGFD_KERNEL_ZMARCH)
            r = sgfd_set_tile(h, cands[c].cols, cands[c].rows, cands[c].zchunk);
        if (r) break;
        cudaError_t e = dispatch_on(h, h->sr, h->stream, 0, 0.0f, false, nullptr);   // warm-up step
        if (e == cudaSuccess) e = cudaEventRecord(e0, h->stream);
        for (int k = 0; k < probe_steps && e == cudaSuccess; ++k)
            e = dispatch_on(h, h->sr, h->stream, k, 0.0f, false, nullptr);
        if (e == cudaSuccess) e = cudaEventRecord(e1, h->stream);
        if (e == cudaSuccess) e = cudaEventSynchronize(e1);
        float ms = 0.0f;
        if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
        if (e != cudaSuccess) { r = cuda_fail(h, e, "autotune probe"); break; }
        ms /= (float)probe_steps;
        if (best < 0 || ms < best_ms) { best = (int)c; best_ms = ms; }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (r == SGFD_OK) r = check_device_error(h);
    if (r) return r;
    const Cand &w = cands[best];
    r = sgfd_set_kernel(h, w.kernel);
    if (r == SGFD_OK && w.kernel == SGFD_KERNEL_ZMARCH) r = sgfd_set_tile(h, w.cols, w.rows, w.zchunk);
    if (r == SGFD_OK) r = sgfd_reset(h);
    if (r) return r;
    if (out) {
        std::memset(out, 0, sizeof *out);
        out->kernel = w.kernel;
        out->tile_rows = w.rows;
        out->tile_cols = w.cols;
        out->zchunk = w.zchunk;
        out->candidates = (int32_t)cands.size();
        out->ms_per_step = best_ms;
    }
    return SGFD_OK;
}

int sgfd_batch_create(sgfd_solver *const *models, int32_t n, sgfd_batch **out) {
    if (!out) return fail(nullptr, SGFD_ERR_INVALID, "null output");
    *out = nullptr;
    if (!models || n <= 0) return fail(nullptr, SGFD_ERR_INVALID, "a batch needs at least one model");
    for (int i = 0; i < n; ++i) {
        if (!models[i]) return fail(nullptr, SGFD_ERR_INVALID, "model %d is null", i);
        if (models[i]->device != models[0]->device)
            return fail(nullptr, SGFD_ERR_INVALID, "model %d is on device %d, model 0 on %d", i, models[i]->device,
                        models[0]->device);
        for (int j = 0; j < i; ++j)
            if (models[j] == models[i]) return fail(nullptr, SGFD_ERR_INVALID, "model %d appears twice", i);
    }
    sgfd_batch *b = new (std::nothrow) sgfd_batch;
    if (!b) return fail(nullptr, SGFD_ERR_ALLOC, "out of host memory");
    b->models.assign(models, models + n);
    b->device = models[0]->device;
    const int nb = std::min(n, kMaxBranches);
    cudaError_t e = cudaSetDevice(b->device);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&b->cap, cudaStreamNonBlocking);
    for (int j = 0; j < nb && e == cudaSuccess; ++j) {
        cudaStream_t s = nullptr;
        e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
        if (e == cudaSuccess) b->branch.push_back(s);
        cudaEvent_t ev = nullptr;
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
        if (e == cudaSuccess) b->join.push_back(ev);
    }
    for (int i = 0; i < n && e == cudaSuccess; ++i) {
        cudaEvent_t ev = nullptr;
        e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
        if (e == cudaSuccess) b->ev_in.push_back(ev);
    }
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->done, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaMalloc(&b->step_ctr, sizeof(int));
    if (e == cudaSuccess) e = cudaMemset(b->step_ctr, 0, sizeof(int));
    if (e != cudaSuccess) {
        const int r = fail(nullptr, SGFD_ERR_CUDA, "batch set-up: %s", cudaGetErrorString(e));
        sgfd_batch_destroy(b);
        return r;
    }
    *out = b;
    return SGFD_OK;
}

void sgfd_batch_destroy(sgfd_batch *b) {
    if (!b) return;
    cudaSetDevice(b->device);
    if (b->stream) cudaStreamSynchronize(b->stream);
    release(b);
    for (cudaStream_t s : b->branch) cudaStreamDestroy(s);
    for (cudaEvent_t ev : b->join) cudaEventDestroy(ev);
    for (cudaEvent_t ev : b->ev_in) cudaEventDestroy(ev);
    if (b->fork) cudaEventDestroy(b->fork);
    if (b->done) cudaEventDestroy(b->done);
    if (b->cap) cudaStreamDestroy(b->cap);
    if (b->stream) cudaStreamDestroy(b->stream);
    cudaFree(b->step_ctr);
    cudaFree(b->pdesc);
    cudaFree(b->pfirst);
    cudaFree(b->pctl);
    cudaFree(b->pstatus);
    delete b;
}

const char *sgfd_batch_last_error(const sgfd_batch *b) { return b ? b->err.c_str() : ""; }

int sgfd_batch_run(sgfd_batch *b, int32_t it0, int32_t nsteps) {
    TraceRange trace("sgfd_batch_run");
    if (!b) return fail(nullptr, SGFD_ERR_INVALID, "null batch");
    BATCH_CUDA(b, cudaSetDevice(b->device), "cudaSetDevice");
    if (nsteps < 0 || it0 < 0 || (int64_t)it0 + nsteps > INT32_MAX) return bfail(b, SGFD_ERR_INVALID, "bad step range");
    for (size_t i = 0; i < b->models.size(); ++i) {
        const sgfd_solver *h = b->models[i];
        if (!h->medium_set) return bfail(b, SGFD_ERR_STATE, "model %zu has no medium", i);
        if (h->sr.src >= 0 && (int64_t)it0 + nsteps > h->wavelet_nt)
            return bfail(b, SGFD_ERR_STATE, "model %zu: wavelet covers %d steps, run needs %d", i, h->wavelet_nt,
                         it0 + nsteps);
    }
    for (size_t i = 0; i < b->models.size(); ++i) {   // after the models' queued work
        BATCH_CUDA(b, cudaEventRecord(b->ev_in[i], b->models[i]->stream), "order after model streams");
        BATCH_CUDA(b, cudaStreamWaitEvent(b->stream, b->ev_in[i], 0), "order after model streams");
    }
    if (b->persistent) {
        const int r = run_persistent(b, it0, nsteps);
        if (r) return r;
        BATCH_CUDA(b, cudaEventRecord(b->done, b->stream), "order model streams after the batch");
        for (sgfd_solver *h : b->models)
            BATCH_CUDA(b, cudaStreamWaitEvent(h->stream, b->done, 0), "order model streams after the batch");
        return SGFD_OK;
    }
    int it = it0, left = nsteps;
    if (left >= kGraphSteps) {
        if (!keys_current(b)) {
            const int r = capture(b);
            if (r) return r;
        }
        BATCH_CUDA(b, launch_counter(b->step_ctr, it, false, b->stream), "step counter");
        for (; left >= kGraphSteps; left -= kGraphSteps, it += kGraphSteps)
            BATCH_CUDA(b, cudaGraphLaunch(b->graph, b->stream), "batch graph launch");
    }
    for (; left > 0; --left, ++it)
        for (sgfd_solver *h : b->models)
            BATCH_CUDA(b, dispatch_on(h, h->sr, b->stream, it, 0.0f, true, nullptr), "batch step launch");
    BATCH_CUDA(b, cudaEventRecord(b->done, b->stream), "order model streams after the batch");
    for (sgfd_solver *h : b->models)
        BATCH_CUDA(b, cudaStreamWaitEvent(h->stream, b->done, 0), "order model streams after the batch");
    return SGFD_OK;
}

int sgfd_batch_synchronize(sgfd_batch *b) {
    if (!b) return fail(nullptr, SGFD_ERR_INVALID, "null batch");
    BATCH_CUDA(b, cudaSetDevice(b->device), "cudaSetDevice");
    BATCH_CUDA(b, cudaStreamSynchronize(b->stream), "batch synchronize");
    if (b->pstatus) {
        int st = 0;
        BATCH_CUDA(b, cudaMemcpy(&st, b->pstatus, sizeof st, cudaMemcpyDeviceToHost), "batch status");
        if (st) {
            BATCH_CUDA(b, cudaMemset(b->pstatus, 0, sizeof st), "batch status");
            for (sgfd_solver *h : b->models) check_device_error(h);   // clear the models' flags too
            return bfail(b, SGFD_ERR_CUDA, "persistent batch: a bounded %s wait gave up",
                         st == kBatchWaitGrid ? "grid-barrier" : "TMA");
        }
    }
    for (size_t i = 0; i < b->models.size(); ++i)
        if (check_device_error(b->models[i]) != SGFD_OK)
            return bfail(b, SGFD_ERR_CUDA, "model %zu: %s", i, b->models[i]->err.c_str());
    return SGFD_OK;
}

void *sgfd_batch_stream(sgfd_batch *b) { return b ? static_cast<void *>(b->stream) : nullptr; }

int sgfd_batch_run_launches(const sgfd_batch *b, int32_t nsteps) {
    if (!b || nsteps < 0) return -1;
    if (b->persistent) return nsteps > 0 ? 1 : 0;
    int per = 0;
    for (const sgfd_solver *h : b->models) per += sgfd_launches_per_step(h);
    const int replays = nsteps >= kGraphSteps ? nsteps / kGraphSteps : 0;
    return nsteps * per + (replays ? 1 + replays : 0);
}

}  // extern "C"
