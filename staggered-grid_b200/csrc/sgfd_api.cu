// sgfd_api.cu — the C ABI of include/sgfd.h: handle lifetime, device memory,
// uploads/downloads and the time loop.  Kernels live in kernels_*.cu.
//
// Reference counterparts (3DGPUwithPML_1DArraySingleGPU_optimization/):
//   sgfd_create    ElasticWaveEquation.cu:8-45 (ctor), :47-108 (region table)
//   sgfd_set_medium ElasticWaveEquation.cu:143-147
//   sgfd_step      ElasticWaveEquation.cu:191-204 (propagate)
//   sgfd_run       ElasticWaveEquation.cu:153-172 (time loop of run())
//   sgfd_get_traces ElasticWaveEquation.cu:174
//   sgfd_destroy   ElasticWaveEquation.cu:125-138
// Differences by design: status codes instead of exit(1) (OPT/common.h:6-16),
// 64-bit sizes (the reference's int memsize overflows past 2^29 cells,
// OPT/ElasticWaveEquation.cu:20), one stream per handle instead of a device
// synchronisation per step (OPT/ElasticWaveEquation.cu:201).
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <algorithm>
#include <mutex>
#include <new>
#include <string>
#include <vector>

#include "solver.h"

using namespace sgfd;

namespace {
thread_local std::string g_error;
}  // namespace

namespace sgfd {

int fail(sgfd_solver *h, int code, const char *fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    std::vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    if (h) h->err = buf; else g_error = buf;
    return code;
}

int cuda_fail(sgfd_solver *h, cudaError_t e, const char *what) {
    return fail(h, SGFD_ERR_CUDA, "%s: %s (%s)", what, cudaGetErrorName(e), cudaGetErrorString(e));
}

int check_handle(sgfd_solver *h) {
    if (!h) return fail(nullptr, SGFD_ERR_INVALID, "null handle");
    cudaError_t e = cudaSetDevice(h->device);
    if (e != cudaSuccess) return cuda_fail(h, e, "cudaSetDevice");
    return SGFD_OK;
}

int check_device_error(sgfd_solver *h) {
    int *flags[2] = {h->dev_err, h->strip_n > 0 ? strip_error_flag(h->strip_buf, h->strip_n) : nullptr};
    for (int *f : flags) {
        if (!f) continue;
        int flag = 0;
        SG_CUDA(h, cudaMemcpyAsync(&flag, f, sizeof(int), cudaMemcpyDeviceToHost, h->stream), "error flag");
        SG_CUDA(h, cudaStreamSynchronize(h->stream), "error flag");
        if (flag) {
            cudaMemsetAsync(f, 0, sizeof(int), h->stream);
            return fail(h, SGFD_ERR_CUDA, "a kernel's bounded wait for its %s gave up (flag %d)",
                        f == h->dev_err ? "TMA copies" : "tensor-core results", flag);
        }
    }
    return SGFD_OK;
}

int sync_views(sgfd_solver *h) {
    if (h->storage == SGFD_STORE_F32) return SGFD_OK;
    SG_CUDA(h, half_to_views(h->m, h->hs, h->stream), "16-bit fields to FP32");
    return SGFD_OK;
}

int sync_from_views(sgfd_solver *h) {
    if (h->storage == SGFD_STORE_F32) return SGFD_OK;
    SG_CUDA(h, half_from_views(h->m, h->hs, h->stream), "FP32 fields to 16-bit");
    return SGFD_OK;
}

int set_scale_exponents(sgfd_solver *h, const int *e) {
    if (h->storage == SGFD_STORE_F32) return SGFD_OK;
    struct { int e[9], e_new[9]; float sc[9], inv[9]; unsigned amax[9]; } st{};
    for (int g = 0; g < 9; ++g) {
        st.e[g] = st.e_new[g] = e[g];
        st.sc[g] = std::ldexp(1.0f, e[g]);
        st.inv[g] = std::ldexp(1.0f, -e[g]);
    }
    SG_CUDA(h, cudaMemcpyAsync(h->hstate, &st, sizeof st, cudaMemcpyHostToDevice, h->stream), "scale state");
    SG_CUDA(h, cudaStreamSynchronize(h->stream), "scale state");
    return SGFD_OK;
}

int reset_scales(sgfd_solver *h) {
    const int zero[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    return set_scale_exponents(h, zero);
}

int get_scale_exponents(sgfd_solver *h, int *e) {
    if (h->storage == SGFD_STORE_F32) {
        for (int g = 0; g < 9; ++g) e[g] = 0;
        return SGFD_OK;
    }
    SG_CUDA(h, cudaMemcpyAsync(e, h->hs.e, 9 * sizeof(int), cudaMemcpyDeviceToHost, h->stream), "scale state");
    SG_CUDA(h, cudaStreamSynchronize(h->stream), "scale state");
    return SGFD_OK;
}

// Bytes between consecutive 16-bit wavefield arrays (0 with FP32 storage).
size_t stride16(const sgfd_solver *h) {
    if (h->storage == SGFD_STORE_F32) return 0;
    return (size_t)(reinterpret_cast<const char *>(h->hs.f[1]) - reinterpret_cast<const char *>(h->hs.f[0]));
}

cudaError_t dispatch_on(sgfd_solver *h, const SourceRec &sr, cudaStream_t s, int it, float value,
                        bool use_wavelet, cudaEvent_t *ev) {
    const bool h16 = h->storage != SGFD_STORE_F32;
    cudaError_t e = h->kernel == SGFD_KERNEL_ZMARCH
                        ? (h->zg.pair ? zpair_step(h->m, h->ph, sr, h16 ? &h->hs : nullptr, h->zg, h->vm, h->sm, it,
                                                   value, use_wavelet, s, ev)
                                      : zmarch_step(h->m, h->ph, sr, h->zg, h->zm, it, value, use_wavelet, s, ev,
                                                    h16 ? &h->hs : nullptr))
                    : h16 ? half_step(h->m, h->ph, sr, h->hs, it, value, use_wavelet, s, ev)
                        : simple_step(h->m, h->ph, sr, it, value, use_wavelet, s, ev);
    if (e == cudaSuccess && h->strip_n > 0)
        e = launch_strip(h->m, h->strip_w, h->strip_cells, h->strip_n, h->strip_buf, s);
    if (e == cudaSuccess && h->audit_every > 0) {
        const AuditGate gt{sr.it_dev, it, h->audit_every, h->audit_count, h->audit_hist};
        e = launch_energy_step(audit_model(h), h->ph, h->audit_region, h->audit, h->audit_blocks, gt, s);
    }
    return e;
}

int ensure_audit_scratch(sgfd_solver *h) {
    if (h->audit) return SGFD_OK;
    int sms = 0;
    SG_CUDA(h, cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, h->device), "SM count");
    h->audit_blocks = energy_blocks(sms);
    SG_CUDA(h, dev_malloc(h, &h->audit, (size_t)(2 * h->audit_blocks + 2) * sizeof(double)), "audit scratch");
    return SGFD_OK;
}

void graph_key(const sgfd_solver *h, GraphKey *k) {
    std::memset(static_cast<void *>(k), 0, sizeof *k);
    std::memcpy(static_cast<void *>(&k->m), &h->m, sizeof h->m);
    std::memcpy(static_cast<void *>(&k->ph), &h->ph, sizeof h->ph);
    std::memcpy(static_cast<void *>(&k->sr), &h->sr, sizeof h->sr);
    std::memcpy(static_cast<void *>(&k->zg), &h->zg, sizeof h->zg);
    std::memcpy(static_cast<void *>(&k->vm), &h->vm, sizeof h->vm);
    std::memcpy(static_cast<void *>(&k->sm), &h->sm, sizeof h->sm);
    std::memcpy(static_cast<void *>(&k->zm), &h->zm, sizeof h->zm);
    k->kernel = h->kernel;
    k->audit_every = h->audit_every;
    k->audit_region = h->audit_region;
    k->audit_count = h->audit_count;
    k->audit_hist = h->audit_hist;
    k->audit = h->audit;
    k->strip_w = h->strip_w;
    k->strip_n = h->strip_n;
    k->strip_cells = h->strip_cells;
    k->strip_buf = h->strip_buf;
}

}  // namespace sgfd

namespace {

bool finite_pos(float v) { return std::isfinite(v) && v > 0.0f; }

// Whether the single-precision correction step of div_cell (cell_math.cuh)
// returns RN(a/d) for every significand of a in [1, 2), which by scaling
// covers every |a| in [2^-100, 2^100].  Checked once per divisor value (about
// 2^23 divisions on the host) and remembered.
bool correction_step_exact(float d) {
    static std::mutex mu;
    static std::vector<std::pair<uint32_t, bool>> known;
    uint32_t key;
    std::memcpy(&key, &d, 4);
    {
        std::lock_guard<std::mutex> lock(mu);
        for (auto &k : known)
            if (k.first == key) return k.second;
    }
    bool ok = std::isfinite(d) && std::fabs(d) >= 0x1p-20f && std::fabs(d) <= 0x1p20f;
    const float y = 1.0f / d;
    for (uint32_t sig = 0; ok && sig < (1u << 23); ++sig) {
        float a;
        const uint32_t bits = (127u << 23) | sig;
        std::memcpy(&a, &bits, 4);
        const volatile float want = a / d;
        const float q0 = a * y;
        const float t = std::fma(q0, d, -a);
        const float q = std::fma(-t, y, q0);
        ok = q == want;
    }
    std::lock_guard<std::mutex> lock(mu);
    known.push_back({key, ok});
    return ok;
}

void set_physics(sgfd_solver *h) {
    const sgfd_config &c = h->cfg;
    Physics &ph = h->ph;
    for (int i = 0; i < 5; ++i) ph.c[i] = c.coef[i];
    ph.dt = c.dt; ph.dx = c.dx; ph.dy = c.dy; ph.dz = c.dz;
    for (int i = 0; i < 5; ++i) {
        ph.cs[0][i] = c.coef[i] / c.dx;
        ph.cs[1][i] = c.coef[i] / c.dy;
        ph.cs[2][i] = c.coef[i] / c.dz;
    }
    for (int i = 0; i < 5; ++i) {
        for (int a = 0; a < 3; ++a) ph.cp[a][i] = make_float2(ph.cs[a][i], ph.cs[a][i]);
        ph.cp[3][i] = make_float2(ph.cs[0][i], ph.cs[1][i]);
    }
    ph.fast = c.arith == SGFD_ARITH_FAST;
    ph.inj_dt2 = c.dt * c.dt;
    ph.damping = c.damping;
    ph.quirks = c.quirks;
    const int p = std::max(c.pml, 1);   // pml = 0: no PML cell uses the damping constants
    ph.q_refgpu = 0.5f * c.dt * kTau;
    ph.poly = (8.0f / 15.0f - 0.03f * (float)p) + (1.0f / 1500.0f) * (float)(p * p);
    const double R = c.damping_R > 0 ? (double)c.damping_R : 1e-3;
    ph.q_logr = (float)(0.5 * (double)c.dt * 3.0 * std::log(1.0 / R) / (2.0 * (double)p));
    const double dd[3] = {c.dx, c.dy, c.dz};
    for (int a = 0; a < 3; ++a)
        ph.q_refcpu[a] = (float)(0.5 * (double)c.dt * std::log10(1.0 / R) * 3.4 *
                                 (double)c.damping_vconst / ((double)p * dd[a]));
    const float d3[3] = {c.dx, c.dy, c.dz};
    for (int a = 0; a < 3; ++a)
        ph.qf[a] = c.damping == SGFD_DAMP_LOGR ? ph.q_logr / d3[a] : (ph.q_refgpu / d3[a]) * ph.poly;
    for (int k = 0; k < kPwTable; ++k) {
        const float r = (float)k / (float)p;
        ph.pw[k] = r * r;
    }
    for (int i = 0; i < 5; ++i) ph.cr[i] = make_float2(c.coef[i], c.coef[i]);
    ph.mdiv = 0;
    for (int a = 0; a < 3; ++a) {
        ph.rd[a] = 1.0f / d3[a];
        ph.rd64[a] = 1.0 / (double)d3[a];
        if (correction_step_exact(d3[a])) ph.mdiv |= 1 << a;
    }
}

cudaError_t dispatch_step(sgfd_solver *h, int it, float value, bool use_wavelet, cudaEvent_t *ev) {
    return dispatch_on(h, h->sr, h->stream, it, value, use_wavelet, ev);
}

void release_graph(sgfd_solver *h) {
    if (h->graph) cudaGraphExecDestroy(h->graph);
    h->graph = nullptr;
}

// Capture kGraphSteps steps on a private stream.  Step k of the graph runs
// step *step_ctr + k; the last node adds kGraphSteps to the counter, so
// consecutive replays walk through consecutive steps.
int capture_graph(sgfd_solver *h) {
    release_graph(h);
    if (!h->cap_stream)
        SG_CUDA(h, cudaStreamCreateWithFlags(&h->cap_stream, cudaStreamNonBlocking), "capture stream");
    if (!h->step_ctr) {
        SG_CUDA(h, dev_malloc(h, &h->step_ctr, sizeof(int)), "step counter");
        SG_CUDA(h, cudaMemset(h->step_ctr, 0, sizeof(int)), "step counter");
    }
    SourceRec sr = h->sr;
    sr.it_dev = h->step_ctr;
    SG_CUDA(h, cudaStreamBeginCapture(h->cap_stream, cudaStreamCaptureModeThreadLocal), "begin capture");
    cudaError_t e = cudaSuccess;
    for (int k = 0; k < kGraphSteps && e == cudaSuccess; ++k)
        e = dispatch_on(h, sr, h->cap_stream, k, 0.0f, true, nullptr);
    if (e == cudaSuccess) e = launch_counter(h->step_ctr, kGraphSteps, true, h->cap_stream);
    cudaGraph_t g = nullptr;
    const cudaError_t e_end = cudaStreamEndCapture(h->cap_stream, &g);
    if (e == cudaSuccess) e = e_end;
    if (e == cudaSuccess) e = cudaGraphInstantiate(&h->graph, g, 0);
    if (g) cudaGraphDestroy(g);
    if (e != cudaSuccess) {
        h->graph = nullptr;
        cudaGetLastError();
        return cuda_fail(h, e, "graph capture");
    }
    graph_key(h, &h->graph_key);
    return SGFD_OK;
}

bool graph_current(const sgfd_solver *h) {
    if (!h->graph) return false;
    GraphKey k;
    graph_key(h, &k);
    return std::memcmp(&k, &h->graph_key, sizeof k) == 0;
}

int launch_step(sgfd_solver *h, int it, float value, bool use_wavelet) {
    cudaError_t e = dispatch_step(h, it, value, use_wavelet, nullptr);
    if (e != cudaSuccess) return cuda_fail(h, e, "step launch");
    return SGFD_OK;
}

// z chunking: chunks of at most 48 planes, shorter, down to 16 planes, when
// the grid has too few tiles for ~16 waves of three CTAs per SM (measured on
// B200 with 32 x 8 tiles: 24-, 32- and 48-plane chunks within 1 % on the 394^3
// cube, 48 planes 2 % faster than 24 on the 522^3 cube, where each chunk
// start re-reads 9 planes of the z-queued fields).
void set_zchunks(sgfd_solver *h) {
    ZGeom &g = h->zg;
    const int tiles = g.ntx * g.nty;
    int zc = h->zchunk_req;
    if (zc <= 0) {
        int sms = 148;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, h->device);
        const int target = 16 * 3 * sms;
        int nch = (target + tiles - 1) / tiles;
        nch = std::max(1, std::min(nch, (h->m.nzc + 15) / 16));
        zc = std::min(48, (h->m.nzc + nch - 1) / nch);
    }
    zc = std::max(1, std::min(zc, h->m.nzc));
    g.zc = zc;
    g.nchunks = (h->m.nzc + zc - 1) / zc;
}

// Receivers bucketed per z-march tile, sorted by z (device arrays).
int upload_zrec(sgfd_solver *h, const std::vector<int4> &rec) {
    const Model &m = h->m;
    const int tiles = h->zg.ntx * h->zg.nty;
    std::vector<std::vector<std::pair<int4, int>>> buckets(tiles);
    for (int i = 0; i < (int)rec.size(); ++i) {
        const int4 q = rec[i];
        const int cx = q.x - kHalo, cy = q.y - kHalo, cz = q.z - kHalo;
        if (cx < 0 || cy < 0 || cz < 0 || cx >= m.nxc || cy >= m.nyc || cz >= m.nzc) continue;  // frame: stays 0
        buckets[(cy / (8 * h->zg.cells)) * h->zg.ntx + cx / h->zg.tw].push_back({q, i});
    }
    std::vector<int> off(tiles + 1, 0);
    std::vector<int4> list;
    std::vector<int> idx;
    for (int t = 0; t < tiles; ++t) {
        auto &b = buckets[t];
        std::stable_sort(b.begin(), b.end(), [](const std::pair<int4, int> &a, const std::pair<int4, int> &c) {
            return a.first.z < c.first.z;
        });
        for (auto &e : b) { list.push_back(e.first); idx.push_back(e.second); }
        off[t + 1] = (int)list.size();
    }
    cudaFree(h->zrec_off); cudaFree(h->zrec_list); cudaFree(h->zrec_idx);
    h->zrec_off = nullptr; h->zrec_list = nullptr; h->zrec_idx = nullptr;
    const size_t nl = std::max<size_t>(list.size(), 1);
    cudaError_t e = dev_malloc(h, &h->zrec_off, off.size() * sizeof(int));
    if (e == cudaSuccess) e = dev_malloc(h, &h->zrec_list, nl * sizeof(int4));
    if (e == cudaSuccess) e = dev_malloc(h, &h->zrec_idx, nl * sizeof(int));
    if (e != cudaSuccess) { cudaGetLastError(); return fail(h, SGFD_ERR_ALLOC, "receiver lists"); }
    SG_CUDA(h, cudaMemcpy(h->zrec_off, off.data(), off.size() * sizeof(int), cudaMemcpyHostToDevice), "receiver lists");
    if (!list.empty()) {
        SG_CUDA(h, cudaMemcpy(h->zrec_list, list.data(), list.size() * sizeof(int4), cudaMemcpyHostToDevice), "receiver lists");
        SG_CUDA(h, cudaMemcpy(h->zrec_idx, idx.data(), idx.size() * sizeof(int), cudaMemcpyHostToDevice), "receiver lists");
    }
    h->zg.rec_off = h->zrec_off;
    h->zg.rec_list = h->zrec_list;
    h->zg.rec_idx = h->zrec_idx;
    return SGFD_OK;
}

}  // namespace

extern "C" {

int sgfd_abi_version(void) { return SGFD_ABI_VERSION; }

void sgfd_config_default(sgfd_config *cfg) {
    if (!cfg) return;
    std::memset(cfg, 0, sizeof *cfg);
    cfg->nx = cfg->ny = cfg->nz = 64;
    cfg->pml = 10;
    cfg->dt = 0.0005f; cfg->dx = cfg->dy = cfg->dz = 10.0f;
    // Coefficients of the reference driver (CON/main.cu:40-44).
    const float c[5] = {1.21124f, -8.97217e-2f, 1.38428e-2f, -1.76566e-3f, 1.18680e-4f};
    std::memcpy(cfg->coef, c, sizeof c);
    cfg->damping = SGFD_DAMP_REFGPU;
    cfg->damping_R = 0.001f;        // reference R (OPT/ElasticMacro.h:20)
    cfg->damping_vconst = 2000.0f;  // reference CPU constant Vs
    cfg->quirks = SGFD_QUIRKS_REF;
    cfg->storage = SGFD_STORE_F32;
    cfg->kernel = SGFD_KERNEL_AUTO;
    cfg->device = 0;
    cfg->arith = SGFD_ARITH_REF;
}

const char *sgfd_global_error(void) { return g_error.c_str(); }

const char *sgfd_last_error(const sgfd_solver *h) { return h ? h->err.c_str() : g_error.c_str(); }

int sgfd_create(const sgfd_config *cfg, sgfd_solver **out) {
    if (!cfg || !out) return fail(nullptr, SGFD_ERR_INVALID, "null config or output pointer");
    *out = nullptr;
    const sgfd_config &c = *cfg;
    for (int i = 0; i < 5; ++i)
        if (c.reserved[i] != 0) return fail(nullptr, SGFD_ERR_INVALID, "reserved config fields must be zero");
    const bool slab = c.nz_total != 0;
    if (slab) {
        // the whole model must be a valid model; the slab needs its own 5 computed planes beside each cut
        const int need_z = 2 * (kHalo + c.pml) + 1;
        if (c.nz_total < need_z)
            return fail(nullptr, SGFD_ERR_INVALID, "nz_total %d too small for pml %d (needs >= %d)", c.nz_total,
                        c.pml, need_z);
        if (c.nz < 3 * kHalo || c.z_offset < 0 || (int64_t)c.z_offset + c.nz - 2 * kHalo > c.nz_total - 2 * kHalo)
            return fail(nullptr, SGFD_ERR_INVALID,
                        "z-slab of %d GRID planes at computed offset %d does not fit a model of %d GRID planes "
                        "(a slab needs >= %d computed planes)", c.nz, c.z_offset, c.nz_total, kHalo);
        if (c.storage != SGFD_STORE_F32)
            return fail(nullptr, SGFD_ERR_UNSUPPORTED, "z-slabs need FP32 storage");
    } else if (c.z_offset != 0) {
        return fail(nullptr, SGFD_ERR_INVALID, "z_offset needs nz_total");
    }
    if (c.arith != SGFD_ARITH_REF && c.arith != SGFD_ARITH_FAST)
        return fail(nullptr, SGFD_ERR_INVALID, "unknown arithmetic mode %d", c.arith);
    if (c.pml < 0) return fail(nullptr, SGFD_ERR_INVALID, "pml must be >= 0 (got %d)", c.pml);
    const int need = 2 * (kHalo + c.pml) + 1;
    if (c.nx < need || c.ny < need || (!slab && c.nz < need))
        return fail(nullptr, SGFD_ERR_INVALID, "grid %dx%dx%d too small for pml %d (each axis needs >= %d)",
                    c.nx, c.ny, c.nz, c.pml, need);
    if (!finite_pos(c.dt) || !finite_pos(c.dx) || !finite_pos(c.dy) || !finite_pos(c.dz))
        return fail(nullptr, SGFD_ERR_INVALID, "dt, dx, dy, dz must be finite and positive");
    for (int i = 0; i < 5; ++i)
        if (!std::isfinite(c.coef[i])) return fail(nullptr, SGFD_ERR_INVALID, "non-finite coefficient %d", i);
    if (c.damping < SGFD_DAMP_REFGPU || c.damping > SGFD_DAMP_REFCPU)
        return fail(nullptr, SGFD_ERR_INVALID, "unknown damping profile %d", c.damping);
    if ((c.damping != SGFD_DAMP_REFGPU) && !(c.damping_R > 0.0f && c.damping_R < 1.0f))
        return fail(nullptr, SGFD_ERR_INVALID, "damping_R must be in (0, 1)");
    if (c.quirks != SGFD_QUIRKS_REF && c.quirks != SGFD_QUIRKS_FIXED)
        return fail(nullptr, SGFD_ERR_INVALID, "unknown quirks mode %d", c.quirks);
    if (c.storage != SGFD_STORE_F32 && c.storage != SGFD_STORE_BF16 && c.storage != SGFD_STORE_F16)
        return fail(nullptr, SGFD_ERR_UNSUPPORTED, "storage type %d is not built into this library", c.storage);
    if (c.kernel != SGFD_KERNEL_AUTO && c.kernel != SGFD_KERNEL_SIMPLE && c.kernel != SGFD_KERNEL_ZMARCH)
        return fail(nullptr, SGFD_ERR_UNSUPPORTED, "kernel family %d is not built into this library", c.kernel);
    const int64_t cells = (int64_t)c.nx * c.ny * c.nz;
    if (cells > ((int64_t)1 << 36)) return fail(nullptr, SGFD_ERR_INVALID, "grid has too many cells");

    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return fail(nullptr, SGFD_ERR_NO_DEVICE, "no CUDA device available");
    }
    if (c.device < 0 || c.device >= ndev) return fail(nullptr, SGFD_ERR_INVALID, "device %d out of range", c.device);

    sgfd_solver *h = new (std::nothrow) sgfd_solver();
    if (!h) return fail(nullptr, SGFD_ERR_ALLOC, "host allocation failed");
    h->cfg = c;
    h->device = c.device;
    h->kernel = SGFD_KERNEL_SIMPLE;
    cudaError_t e = cudaSetDevice(h->device);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&h->own_stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        int r = cuda_fail(nullptr, e, "device setup");
        delete h;
        return r;
    }
    h->stream = h->own_stream;

    Model &m = h->m;
    m.nx = c.nx; m.ny = c.ny; m.nz = c.nz;
    m.px = (int)round_up((size_t)c.nx + kXOff, 32);
    m.pml = c.pml;
    m.nxc = c.nx - 2 * kHalo; m.nyc = c.ny - 2 * kHalo; m.nzc = c.nz - 2 * kHalo;
    m.plane = (int64_t)m.px * m.ny;
    m.zoff = slab ? c.z_offset : 0;
    m.nzcg = slab ? c.nz_total - 2 * kHalo : m.nzc;
    m.pbase = pml_before(m.nxc, m.nyc, m.nzcg, m.pml, m.zoff);
    m.npml = pml_before(m.nxc, m.nyc, m.nzcg, m.pml, m.zoff + m.nzc) - m.pbase;
    const size_t arr_bytes = array_bytes(m);
    const size_t pool_bytes = arr_bytes * 16;
    e = dev_malloc(h, &h->field_pool, pool_bytes);
    if (e == cudaSuccess) e = dev_malloc(h, &h->split, (size_t)split_elems(m.npml) * sizeof(float));
    if (e != cudaSuccess) {
        cudaGetLastError();
        int r = fail(nullptr, SGFD_ERR_ALLOC, "device allocation of %.2f GB failed",
                     (pool_bytes + (double)split_elems(m.npml) * 4) / 1e9);
        sgfd_destroy(h);
        return r;
    }
    auto arr = [&](int k) { return reinterpret_cast<float *>(h->field_pool + k * arr_bytes) + kXOff; };
    // txx..tyz, lambda, mu and the shear moduli consecutive: the z-march
    // stress update stages a cell's 11 own values with one copy
    for (int k = 0; k < 9; ++k) m.f[k] = arr(k);
    m.lam = arr(9);
    m.mu = arr(10);
    m.mxy = arr(11);
    m.mxz = arr(12);
    m.myz = arr(13);
    m.b = arr(14);
    m.rmu = arr(15);
    m.split = h->split;
    e = cudaMemsetAsync(h->field_pool, 0, pool_bytes, h->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(h->split, 0, (size_t)split_elems(m.npml) * sizeof(float), h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) {
        int r = cuda_fail(nullptr, e, "zeroing device state");
        sgfd_destroy(h);
        return r;
    }
    set_physics(h);
    h->sr.src = -1;
    h->sr.nrec = 0;

    // kernel family
    // 16-bit storage: the stored fields and splits and their scale state
    if (c.storage != SGFD_STORE_F32) {
        h->storage = c.storage;
        const size_t a16 = round_up((size_t)m.plane * m.nz * 2, 256);
        const size_t s16 = round_up((size_t)split_elems(m.npml) * 2, 256);
        e = dev_malloc(h, &h->h16_pool, a16 * 9 + s16);
        if (e == cudaSuccess) e = dev_malloc(h, &h->hstate, 64 * sizeof(int));
        if (e == cudaSuccess) e = cudaMemsetAsync(h->h16_pool, 0, a16 * 9 + s16, h->stream);
        if (e != cudaSuccess) {
            cudaGetLastError();
            int r = fail(nullptr, SGFD_ERR_ALLOC, "16-bit storage allocation failed");
            sgfd_destroy(h);
            return r;
        }
        HalfState &hs = h->hs;
        for (int k = 0; k < 9; ++k) hs.f[k] = reinterpret_cast<uint16_t *>(h->h16_pool + k * a16) + kXOff;
        hs.split = reinterpret_cast<uint16_t *>(h->h16_pool + 9 * a16);
        int *hst = static_cast<int *>(h->hstate);
        hs.e = hst;
        hs.e_new = hst + 9;
        hs.sc = reinterpret_cast<float *>(hst + 18);
        hs.inv = reinterpret_cast<float *>(hst + 27);
        hs.amax = reinterpret_cast<unsigned *>(hst + 36);
        hs.storage = c.storage;
        int r = reset_scales(h);
        if (r) { g_error = h->err; sgfd_destroy(h); return r; }
    }

    if (c.kernel != SGFD_KERNEL_SIMPLE && zmarch_supported(m)) {
        // 32 x 8 tiles, with either storage (16-bit storage also runs on the paired 64 x 8 tiling)
        const bool h16 = c.storage != SGFD_STORE_F32;
        h->zg.cells = 1;
        h->zg.pair = 0;
        h->zg.tw = kZTileX;
        e = zmarch_prepare(m, h->zg.cells, arr_bytes, &h->zm, h16 ? &h->hs : nullptr, stride16(h));
        if (e == cudaSuccess) e = dev_malloc(h, &h->dev_err, sizeof(int));
        if (e == cudaSuccess) e = cudaMemset(h->dev_err, 0, sizeof(int));
        if (e != cudaSuccess) {
            int r = cuda_fail(nullptr, e, "z-march set-up");
            sgfd_destroy(h);
            return r;
        }
        h->kernel = SGFD_KERNEL_ZMARCH;
        zmarch_tiles(m, h->zg.cells, &h->zg.ntx, &h->zg.nty);
        h->zg.err = h->dev_err;
        set_zchunks(h);
        int r = upload_zrec(h, {});
        if (r) { g_error = h->err; sgfd_destroy(h); return r; }
    } else if (c.kernel == SGFD_KERNEL_ZMARCH) {
        sgfd_destroy(h);
        return fail(nullptr, SGFD_ERR_UNSUPPORTED, "z-marching kernels unavailable (no TMA encoder in the driver)");
    }
    *out = h;
    return SGFD_OK;
}

void sgfd_destroy(sgfd_solver *h) {
    if (!h) return;
    cudaSetDevice(h->device);
    if (h->stream) cudaStreamSynchronize(h->stream);
    cudaFree(h->field_pool);
    cudaFree(h->split);
    cudaFree(h->rec);
    cudaFree(h->traces);
    cudaFree(h->wavelet);
    cudaFree(h->zrec_off);
    cudaFree(h->zrec_list);
    cudaFree(h->zrec_idx);
    cudaFree(h->dev_err);
    cudaFree(h->h16_pool);
    cudaFree(h->hstate);
    cudaFree(h->audit);
    cudaFree(h->audit_hist);
    cudaFree(h->strip_cells);
    cudaFree(h->strip_buf);
    release_graph(h);
    cudaFree(h->step_ctr);
    if (h->cap_stream) cudaStreamDestroy(h->cap_stream);
    if (h->own_stream) cudaStreamDestroy(h->own_stream);
    delete h;
}

int sgfd_set_stream(sgfd_solver *h, void *stream) {
    int r = check_handle(h);
    if (r) return r;
    SG_CUDA(h, cudaStreamSynchronize(h->stream), "synchronising previous stream");
    h->stream = stream ? static_cast<cudaStream_t>(stream) : h->own_stream;
    return SGFD_OK;
}

static int upload_medium(sgfd_solver *h, const float *b, const float *l, const float *mu, cudaMemcpyKind kind) {
    int r = check_handle(h);
    if (r) return r;
    if (!b || !l || !mu) return fail(h, SGFD_ERR_INVALID, "null medium array");
    const Model &m = h->m;
    const size_t row = (size_t)m.nx * sizeof(float);
    const size_t rows = (size_t)m.ny * m.nz;
    const float *src[3] = {b, l, mu};
    float *dst[3] = {const_cast<float *>(m.b), const_cast<float *>(m.lam), const_cast<float *>(m.mu)};
    if (kind == cudaMemcpyHostToDevice) {
        // One contiguous transfer per array (short-row 2D copies from host
        // memory run far below the link's bandwidth) into the storage of the
        // three shear moduli, which are recomputed from b and mu below, then
        // into the padded rows on the device.
        float *stage[3] = {const_cast<float *>(m.mxy) - kXOff, const_cast<float *>(m.mxz) - kXOff,
                           const_cast<float *>(m.myz) - kXOff};
        for (int k = 0; k < 3; ++k)
            SG_CUDA(h, cudaMemcpyAsync(stage[k], src[k], row * rows, kind, h->stream), "medium upload");
        for (int k = 0; k < 3; ++k)
            SG_CUDA(h, launch_pitch_rows(dst[k], m.px, stage[k], m.nx, (int64_t)rows, h->stream), "medium rows");
    } else {
        for (int k = 0; k < 3; ++k)
            SG_CUDA(h, cudaMemcpy2DAsync(dst[k], (size_t)m.px * sizeof(float), src[k], row, row, rows, kind,
                                         h->stream), "medium upload");
    }
    cudaError_t e = launch_reciprocal(const_cast<float *>(m.rmu) - kXOff, m.mu - kXOff, m.plane * m.nz, h->stream);
    if (e == cudaSuccess)
        e = launch_shear_means(m, h->ph, const_cast<float *>(m.mxy), const_cast<float *>(m.mxz),
                               const_cast<float *>(m.myz), h->stream);
    if (e != cudaSuccess) return cuda_fail(h, e, "medium set-up kernels");
    SG_CUDA(h, cudaStreamSynchronize(h->stream), "medium upload");
    h->medium_set = true;
    return SGFD_OK;
}

int sgfd_set_medium(sgfd_solver *h, const float *b, const float *l, const float *mu) {
    TraceRange trace("sgfd_set_medium");
    return upload_medium(h, b, l, mu, cudaMemcpyHostToDevice);
}

int sgfd_set_medium_device(sgfd_solver *h, const float *b, const float *l, const float *mu) {
    return upload_medium(h, b, l, mu, cudaMemcpyDeviceToDevice);
}

int sgfd_set_source(sgfd_solver *h, int32_t x, int32_t y, int32_t z) {
    int r = check_handle(h);
    if (r) return r;
    const Model &m = h->m;
    if (x < kHalo || y < kHalo || z < kHalo || x >= m.nx - kHalo || y >= m.ny - kHalo || z >= m.nz - kHalo)
        return fail(h, SGFD_ERR_INVALID, "source (%d,%d,%d) outside the computed region [5, n-5)", x, y, z);
    h->sr.src = pidx(m, x, y, z);
    return SGFD_OK;
}

int sgfd_set_receivers(sgfd_solver *h, int32_t n, const int32_t *xyz, const int32_t *comp, int32_t nt) {
    int r = check_handle(h);
    if (r) return r;
    if (n < 0 || (n > 0 && (!xyz || !comp || nt < 1)))
        return fail(h, SGFD_ERR_INVALID, "bad receiver arguments (n=%d, nt=%d)", n, nt);
    const Model &m = h->m;
    std::vector<int4> host(n);
    for (int i = 0; i < n; ++i) {
        const int x = xyz[3 * i], y = xyz[3 * i + 1], z = xyz[3 * i + 2], c = comp[i];
        if (x < 0 || y < 0 || z < 0 || x >= m.nx || y >= m.ny || z >= m.nz)
            return fail(h, SGFD_ERR_INVALID, "receiver %d at (%d,%d,%d) outside the grid", i, x, y, z);
        if (c < 0 || c >= SGFD_NFIELDS) return fail(h, SGFD_ERR_INVALID, "receiver %d: bad component %d", i, c);
        host[i] = make_int4(x, y, z, c);
    }
    SG_CUDA(h, cudaStreamSynchronize(h->stream), "synchronise before receiver update");
    cudaFree(h->rec);
    cudaFree(h->traces);
    h->rec = nullptr;
    h->traces = nullptr;
    h->sr.nrec = 0;
    h->sr.nt = 0;
    if (n > 0) {
        const size_t tbytes = (size_t)n * nt * sizeof(float);
        cudaError_t e = dev_malloc(h, &h->rec, n * sizeof(int4));
        if (e == cudaSuccess) e = dev_malloc(h, &h->traces, tbytes);
        if (e != cudaSuccess) {
            cudaGetLastError();
            return fail(h, SGFD_ERR_ALLOC, "receiver buffers (%zu bytes)", tbytes);
        }
        SG_CUDA(h, cudaMemcpy(h->rec, host.data(), n * sizeof(int4), cudaMemcpyHostToDevice), "receiver upload");
        SG_CUDA(h, cudaMemset(h->traces, 0, tbytes), "trace clear");
    }
    h->sr.nrec = n;
    h->sr.nt = n > 0 ? nt : 0;
    h->sr.rec = h->rec;
    h->sr.traces = h->traces;
    h->rec_host = host;
    if (h->dev_err) return upload_zrec(h, host);   // z-march receiver lists, kept current while prepared
    return SGFD_OK;
}

int sgfd_set_wavelet(sgfd_solver *h, int32_t nt, const float *values) {
    int r = check_handle(h);
    if (r) return r;
    if (nt < 1 || !values) return fail(h, SGFD_ERR_INVALID, "bad wavelet");
    SG_CUDA(h, cudaStreamSynchronize(h->stream), "synchronise before wavelet update");
    if (nt > h->wavelet_nt) {
        cudaFree(h->wavelet);
        h->wavelet = nullptr;
        cudaError_t e = dev_malloc(h, &h->wavelet, (size_t)nt * sizeof(float));
        if (e != cudaSuccess) {
            cudaGetLastError();
            h->wavelet_nt = 0;
            return fail(h, SGFD_ERR_ALLOC, "wavelet buffer");
        }
    }
    h->wavelet_nt = nt;
    SG_CUDA(h, cudaMemcpy(h->wavelet, values, (size_t)nt * sizeof(float), cudaMemcpyHostToDevice), "wavelet upload");
    h->sr.wavelet = h->wavelet;
    return SGFD_OK;
}

int sgfd_step(sgfd_solver *h, int32_t it, float source_value) {
    TraceRange trace("sgfd_step");
    int r = check_handle(h);
    if (r) return r;
    if (!h->medium_set) return fail(h, SGFD_ERR_STATE, "sgfd_set_medium must come before stepping");
    return launch_step(h, it, source_value, false);
}

int sgfd_run(sgfd_solver *h, int32_t it0, int32_t nsteps, int32_t use_graph) {
    TraceRange trace("sgfd_run");
    int r = check_handle(h);
    if (r) return r;
    if (!h->medium_set) return fail(h, SGFD_ERR_STATE, "sgfd_set_medium must come before stepping");
    if (nsteps < 0 || it0 < 0) return fail(h, SGFD_ERR_INVALID, "bad step range");
    if ((int64_t)it0 + nsteps > INT32_MAX) return fail(h, SGFD_ERR_INVALID, "step range overflows int32");
    if (h->sr.src >= 0 && (int64_t)it0 + nsteps > h->wavelet_nt)
        return fail(h, SGFD_ERR_STATE, "wavelet covers %d steps, run needs %d", h->wavelet_nt, it0 + nsteps);
    int it = it0, left = nsteps;
    if (use_graph && left >= kGraphSteps) {
        if (!graph_current(h)) {
            r = capture_graph(h);
            if (r) return r;
        }
        SG_CUDA(h, launch_counter(h->step_ctr, it, false, h->stream), "step counter");
        for (; left >= kGraphSteps; left -= kGraphSteps, it += kGraphSteps)
            SG_CUDA(h, cudaGraphLaunch(h->graph, h->stream), "graph launch");
    }
    for (; left > 0; --left, ++it) {
        r = launch_step(h, it, 0.0f, true);
        if (r) return r;
    }
    return SGFD_OK;
}

int sgfd_step_phase(sgfd_solver *h, int32_t it, float source_value, int32_t phase) {
    return sgfd_step_phase_part(h, it, source_value, phase, SGFD_PART_INNER | SGFD_PART_OUTER);
}

int sgfd_step_phase_part(sgfd_solver *h, int32_t it, float source_value, int32_t phase, int32_t parts) {
    TraceRange trace("sgfd_step_phase_part");
    int r = check_handle(h);
    if (r) return r;
    if (!h->medium_set) return fail(h, SGFD_ERR_STATE, "sgfd_set_medium must come before stepping");
    if (phase != SGFD_PHASE_VELOCITY && phase != SGFD_PHASE_STRESS)
        return fail(h, SGFD_ERR_INVALID, "unknown phase %d", phase);
    if (parts < 1 || parts > (SGFD_PART_INNER | SGFD_PART_OUTER))
        return fail(h, SGFD_ERR_INVALID, "bad part mask %d", parts);
    if (h->storage != SGFD_STORE_F32 || (h->kernel == SGFD_KERNEL_ZMARCH && h->zg.pair))
        return fail(h, SGFD_ERR_UNSUPPORTED,
                    "half steps need FP32 storage and the simple kernels or 32-column z-march tiles");
    if (h->strip_n > 0 || h->audit_every > 0)
        return fail(h, SGFD_ERR_UNSUPPORTED, "half steps run neither a learned strip nor a per-step audit");
    const int phases = phase == SGFD_PHASE_VELOCITY ? 1 : 2;
    const cudaError_t e =
        h->kernel == SGFD_KERNEL_ZMARCH
            ? zmarch_step(h->m, h->ph, h->sr, h->zg, h->zm, it, source_value, false, h->stream, nullptr, nullptr,
                          phases, parts)
            : simple_step(h->m, h->ph, h->sr, it, source_value, false, h->stream, nullptr, phases, parts);
    if (e != cudaSuccess) return cuda_fail(h, e, "half-step launch");
    return SGFD_OK;
}

int sgfd_halo_bytes(const sgfd_solver *h, int64_t *bytes) {
    if (!h || !bytes) return fail(nullptr, SGFD_ERR_INVALID, "null handle or output pointer");
    *bytes = 3 * (int64_t)kHalo * h->m.plane * (int64_t)sizeof(float);
    return SGFD_OK;
}

namespace {

// The three fields of one halo kind, 5 padded GRID planes each, between the
// slab and buf: pack reads the slab's own computed planes beside the cut,
// unpack writes its frame planes there.  The 5 planes of a field are one
// contiguous range of its padded array.
int halo_copy(sgfd_solver *h, int32_t side, int32_t kind, void *buf, bool pack) {
    TraceRange trace("sgfd_halo");
    int r = check_handle(h);
    if (r) return r;
    if (!buf) return fail(h, SGFD_ERR_INVALID, "null halo buffer");
    if (side != SGFD_HALO_LOW && side != SGFD_HALO_HIGH) return fail(h, SGFD_ERR_INVALID, "bad halo side %d", side);
    if (kind != SGFD_HALO_STRESS && kind != SGFD_HALO_VELOCITY)
        return fail(h, SGFD_ERR_INVALID, "bad halo kind %d", kind);
    if (h->storage != SGFD_STORE_F32) return fail(h, SGFD_ERR_UNSUPPORTED, "halo exchange needs FP32 storage");
    static const int fields[2][3] = {{SGFD_TXZ, SGFD_TYZ, SGFD_TZZ}, {SGFD_VX, SGFD_VY, SGFD_VZ}};
    const Model &m = h->m;
    const int z0 = side == SGFD_HALO_LOW ? (pack ? kHalo : 0) : (pack ? m.nz - 2 * kHalo : m.nz - kHalo);
    const size_t n = (size_t)kHalo * (size_t)m.plane;
    for (int k = 0; k < 3; ++k) {
        float *f = m.f[fields[kind][k]] - kXOff + (int64_t)z0 * m.plane;   // padded array origin, plane z0
        float *b = static_cast<float *>(buf) + k * n;
        SG_CUDA(h, cudaMemcpyAsync(pack ? b : f, pack ? f : b, n * sizeof(float), cudaMemcpyDeviceToDevice,
                                   h->stream), "halo copy");
    }
    return SGFD_OK;
}

}  // namespace

int sgfd_halo_pack(sgfd_solver *h, int32_t side, int32_t kind, void *dst) { return halo_copy(h, side, kind, dst, true); }

int sgfd_halo_unpack(sgfd_solver *h, int32_t side, int32_t kind, const void *src) {
    return halo_copy(h, side, kind, const_cast<void *>(src), false);
}

int sgfd_prepare_run(sgfd_solver *h) {
    int r = check_handle(h);
    if (r) return r;
    if (!h->medium_set) return fail(h, SGFD_ERR_STATE, "sgfd_set_medium must come before stepping");
    if (!graph_current(h)) {
        r = capture_graph(h);
        if (r) return r;
    }
    SG_CUDA(h, cudaGraphUpload(h->graph, h->stream), "graph upload");
    return SGFD_OK;
}

int sgfd_run_launches(const sgfd_solver *h, int32_t nsteps, int32_t use_graph) {
    if (!h || nsteps < 0) return -1;
    const int per = sgfd_launches_per_step(h);
    const int replays = use_graph && nsteps >= kGraphSteps ? nsteps / kGraphSteps : 0;
    return nsteps * per + (replays ? 1 + replays : 0);   // counter set + one advance per replay
}

int sgfd_synchronize(sgfd_solver *h) {
    int r = check_handle(h);
    if (r) return r;
    SG_CUDA(h, cudaStreamSynchronize(h->stream), "synchronize");
    return check_device_error(h);
}

int sgfd_set_zchunk(sgfd_solver *h, int32_t planes) {
    int r = check_handle(h);
    if (r) return r;
    if (planes < 0) return fail(h, SGFD_ERR_INVALID, "negative chunk");
    h->zchunk_req = planes;
    if (h->dev_err) set_zchunks(h);
    return SGFD_OK;
}

int sgfd_set_kernel(sgfd_solver *h, int32_t kernel) {
    int r = check_handle(h);
    if (r) return r;
    if (kernel != SGFD_KERNEL_AUTO && kernel != SGFD_KERNEL_SIMPLE && kernel != SGFD_KERNEL_ZMARCH)
        return fail(h, SGFD_ERR_INVALID, "bad kernel family %d", kernel);
    const int want = kernel == SGFD_KERNEL_SIMPLE ? SGFD_KERNEL_SIMPLE : SGFD_KERNEL_ZMARCH;
    if (want == SGFD_KERNEL_ZMARCH && !h->dev_err)
        return fail(h, SGFD_ERR_UNSUPPORTED, "z-marching kernels are not prepared for this handle "
                                             "(created with SGFD_KERNEL_SIMPLE, or the grid is not supported)");
    SG_CUDA(h, cudaStreamSynchronize(h->stream), "synchronise before switching kernels");
    h->kernel = want;
    return SGFD_OK;
}

int sgfd_set_tile(sgfd_solver *h, int32_t tile_cols, int32_t tile_rows, int32_t zchunk) {
    int r = check_handle(h);
    if (r) return r;
    const bool pair = tile_cols == kPairTileX;
    if (tile_cols != kZTileX && !pair) return fail(h, SGFD_ERR_INVALID, "tile columns must be 32 or 64");
    if (pair ? tile_rows != 8 : (tile_rows != 8 && tile_rows != 16))
        return fail(h, SGFD_ERR_INVALID, "tiles are 32 x 8, 32 x 16 or 64 x 8");
    if (zchunk < 0) return fail(h, SGFD_ERR_INVALID, "negative chunk");
    if (!h->dev_err) return SGFD_OK;   // no z-marching kernels prepared: nothing to tile
    const bool h16 = h->storage != SGFD_STORE_F32;
    if (h16 && !pair && tile_rows != 8)
        return fail(h, SGFD_ERR_UNSUPPORTED, "16-bit storage runs on 32 x 8 or 64 x 8 tiles");
    SG_CUDA(h, cudaStreamSynchronize(h->stream), "synchronise before re-tiling");
    const int cells = tile_rows / 8;
    if (cells != h->zg.cells || (int)pair != h->zg.pair) {
        cudaError_t e = pair ? zpair_prepare(h->m, h16 ? &h->hs : nullptr, &h->vm, &h->sm)
                             : zmarch_prepare(h->m, cells, array_bytes(h->m), &h->zm, h16 ? &h->hs : nullptr,
                                              stride16(h));
        if (e != cudaSuccess) return cuda_fail(h, e, "z-march re-tiling");
        h->zg.cells = cells;
        h->zg.pair = pair ? 1 : 0;
        h->zg.tw = tile_cols;
        if (pair) zpair_tiles(h->m, &h->zg.ntx, &h->zg.nty);
        else zmarch_tiles(h->m, cells, &h->zg.ntx, &h->zg.nty);
        r = upload_zrec(h, h->rec_host);
        if (r) return r;
    }
    h->zchunk_req = zchunk;
    set_zchunks(h);
    return SGFD_OK;
}

int sgfd_set_tiling(sgfd_solver *h, int32_t tile_rows, int32_t zchunk) {
    return sgfd_set_tile(h, kZTileX, tile_rows, zchunk);
}

int sgfd_get_tile(const sgfd_solver *h, int32_t *tile_cols, int32_t *tile_rows, int32_t *zchunk) {
    if (!h) return SGFD_ERR_INVALID;
    if (tile_cols) *tile_cols = h->kernel == SGFD_KERNEL_ZMARCH ? h->zg.tw : 0;
    if (tile_rows) *tile_rows = h->kernel == SGFD_KERNEL_ZMARCH ? 8 * h->zg.cells : 0;
    if (zchunk) *zchunk = h->kernel == SGFD_KERNEL_ZMARCH ? h->zg.zc : 0;
    return SGFD_OK;
}

int sgfd_reset(sgfd_solver *h) {
    int r = check_handle(h);
    if (r) return r;
    const Model &m = h->m;
    const size_t arr_bytes = array_bytes(m);
    SG_CUDA(h, cudaMemsetAsync(h->field_pool, 0, arr_bytes * 9, h->stream), "reset fields");
    SG_CUDA(h, cudaMemsetAsync(h->split, 0, (size_t)split_elems(m.npml) * sizeof(float), h->stream), "reset splits");
    if (h->traces)
        SG_CUDA(h, cudaMemsetAsync(h->traces, 0, (size_t)h->sr.nrec * h->sr.nt * sizeof(float), h->stream), "reset traces");
    if (h->audit_hist)
        SG_CUDA(h, cudaMemsetAsync(h->audit_hist, 0, (size_t)h->audit_count * 2 * sizeof(double), h->stream),
                "reset audit history");
    if (h->h16_pool) {
        const size_t a16 = round_up((size_t)m.plane * m.nz * 2, 256);
        const size_t s16 = round_up((size_t)split_elems(m.npml) * 2, 256);
        SG_CUDA(h, cudaMemsetAsync(h->h16_pool, 0, a16 * 9 + s16, h->stream), "reset 16-bit fields");
        const int r = reset_scales(h);
        if (r) return r;
    }
    SG_CUDA(h, cudaStreamSynchronize(h->stream), "reset");
    return SGFD_OK;
}

int sgfd_get_traces(sgfd_solver *h, float *out) {
    int r = check_handle(h);
    if (r) return r;
    if (!out) return fail(h, SGFD_ERR_INVALID, "null output");
    const int n = h->sr.nrec, nt = h->sr.nt;
    if (n == 0) return SGFD_OK;
    // device traces are time-major [it][r]; the ABI returns receiver-major [r][it]
    std::vector<float> tm((size_t)n * nt);
    SG_CUDA(h, cudaMemcpyAsync(tm.data(), h->traces, tm.size() * sizeof(float), cudaMemcpyDeviceToHost, h->stream),
            "trace download");
    SG_CUDA(h, cudaStreamSynchronize(h->stream), "trace download");
    r = check_device_error(h);
    if (r) return r;
    for (int it = 0; it < nt; ++it)
        for (int q = 0; q < n; ++q) out[(size_t)q * nt + it] = tm[(size_t)it * n + q];
    return SGFD_OK;
}

int sgfd_get_trace_range(sgfd_solver *h, int32_t it0, int32_t n, float *out) {
    int r = check_handle(h);
    if (r) return r;
    if (!out && n > 0) return fail(h, SGFD_ERR_INVALID, "null output");
    if (it0 < 0 || n < 0 || (int64_t)it0 + n > h->sr.nt)
        return fail(h, SGFD_ERR_INVALID, "steps %d..%d outside the trace length %d", it0, it0 + n - 1, h->sr.nt);
    if (n == 0 || h->sr.nrec == 0) return SGFD_OK;
    SG_CUDA(h, cudaMemcpyAsync(out, h->traces + (size_t)it0 * h->sr.nrec, (size_t)n * h->sr.nrec * sizeof(float),
                               cudaMemcpyDeviceToHost, h->stream), "trace range download");
    SG_CUDA(h, cudaStreamSynchronize(h->stream), "trace range download");
    return check_device_error(h);
}

int sgfd_get_trace_step(sgfd_solver *h, int32_t it, float *out) {
    int r = check_handle(h);
    if (r) return r;
    if (!out) return fail(h, SGFD_ERR_INVALID, "null output");
    if (it < 0 || it >= h->sr.nt) return fail(h, SGFD_ERR_INVALID, "step %d outside the trace length %d", it, h->sr.nt);
    SG_CUDA(h, cudaMemcpyAsync(out, h->traces + (size_t)it * h->sr.nrec, (size_t)h->sr.nrec * sizeof(float),
                               cudaMemcpyDeviceToHost, h->stream), "trace step download");
    SG_CUDA(h, cudaStreamSynchronize(h->stream), "trace step download");
    return SGFD_OK;
}

int sgfd_profile(sgfd_solver *h, int32_t it0, int32_t nsteps, float *ms_velocity, float *ms_stress) {
    int r = check_handle(h);
    if (r) return r;
    if (!h->medium_set) return fail(h, SGFD_ERR_STATE, "sgfd_set_medium must come before stepping");
    if (nsteps < 1 || it0 < 0) return fail(h, SGFD_ERR_INVALID, "bad step range");
    if (h->sr.src >= 0 && (int64_t)it0 + nsteps > h->wavelet_nt)
        return fail(h, SGFD_ERR_STATE, "wavelet covers %d steps, profile needs %d", h->wavelet_nt, it0 + nsteps);
    cudaEvent_t ev[4];
    for (int k = 0; k < 4; ++k) SG_CUDA(h, cudaEventCreate(&ev[k]), "event create");
    double tv = 0, ts = 0;
    int rc = SGFD_OK;
    for (int it = it0; it < it0 + nsteps && rc == SGFD_OK; ++it) {
        cudaError_t e = dispatch_step(h, it, 0.0f, true, ev);
        if (e == cudaSuccess) e = cudaEventSynchronize(ev[3]);
        float a = 0, b = 0;
        if (e == cudaSuccess) e = cudaEventElapsedTime(&a, ev[0], ev[1]);
        if (e == cudaSuccess) e = cudaEventElapsedTime(&b, ev[2], ev[3]);
        if (e != cudaSuccess) rc = cuda_fail(h, e, "profiled step");
        tv += a; ts += b;
    }
    for (int k = 0; k < 4; ++k) cudaEventDestroy(ev[k]);
    if (ms_velocity) *ms_velocity = (float)tv;
    if (ms_stress) *ms_stress = (float)ts;
    return rc;
}

static int download(sgfd_solver *h, const float *src, float *out) {
    const Model &m = h->m;
    const size_t row = (size_t)m.nx * sizeof(float);
    SG_CUDA(h, cudaMemcpy2DAsync(out, row, src, (size_t)m.px * sizeof(float), row, (size_t)m.ny * m.nz,
                                 cudaMemcpyDeviceToHost, h->stream), "field download");
    SG_CUDA(h, cudaStreamSynchronize(h->stream), "field download");
    return SGFD_OK;
}

int sgfd_set_field(sgfd_solver *h, int32_t field, const float *src) {
    int r = check_handle(h);
    if (r) return r;
    if (!src) return fail(h, SGFD_ERR_INVALID, "null input");
    if (field < 0 || field >= SGFD_NFIELDS) return fail(h, SGFD_ERR_INVALID, "bad field id %d", field);
    r = sync_views(h);   // 16-bit storage: every FP32 copy current before re-storing them
    if (r) return r;
    const Model &m = h->m;
    const size_t row = (size_t)m.nx * sizeof(float);
    SG_CUDA(h, cudaMemcpy2DAsync(m.f[field], (size_t)m.px * sizeof(float), src, row, row, (size_t)m.ny * m.nz,
                                 cudaMemcpyHostToDevice, h->stream), "field upload");
    r = sync_from_views(h);
    if (r) return r;
    SG_CUDA(h, cudaStreamSynchronize(h->stream), "field upload");
    return SGFD_OK;
}

int sgfd_get_field(sgfd_solver *h, int32_t field, float *out) {
    int r = check_handle(h);
    if (r) return r;
    if (!out) return fail(h, SGFD_ERR_INVALID, "null output");
    if (field < 0 || field >= SGFD_NFIELDS) return fail(h, SGFD_ERR_INVALID, "bad field id %d", field);
    r = sync_views(h);
    if (r) return r;
    return download(h, h->m.f[field], out);
}

int sgfd_get_medium(sgfd_solver *h, int32_t which, float *out) {
    int r = check_handle(h);
    if (r) return r;
    if (!out) return fail(h, SGFD_ERR_INVALID, "null output");
    const float *src = which == SGFD_BUOYANCY ? h->m.b : which == SGFD_LAMBDA ? h->m.lam
                     : which == SGFD_MU ? h->m.mu : nullptr;
    if (!src) return fail(h, SGFD_ERR_INVALID, "bad medium id %d", which);
    return download(h, src, out);
}

int sgfd_energy(sgfd_solver *h, int32_t region, double *kinetic, double *strain) {
    int r = check_handle(h);
    if (r) return r;
    if (region < SGFD_REGION_COMPUTED || region > SGFD_REGION_PML)
        return fail(h, SGFD_ERR_INVALID, "bad region %d", region);
    r = ensure_audit_scratch(h);
    if (r == SGFD_OK) r = sync_views(h);
    if (r) return r;
    double *out = h->audit + 2 * h->audit_blocks;
    SG_CUDA(h, launch_energy(audit_model(h), h->ph, region, h->audit, h->audit_blocks, out, h->stream), "energy audit");
    double res[2];
    SG_CUDA(h, cudaMemcpyAsync(res, out, sizeof res, cudaMemcpyDeviceToHost, h->stream), "energy download");
    SG_CUDA(h, cudaStreamSynchronize(h->stream), "energy download");
    r = check_device_error(h);
    if (r) return r;
    if (kinetic) *kinetic = res[0];
    if (strain) *strain = res[1];
    return SGFD_OK;
}

int sgfd_set_audit(sgfd_solver *h, int32_t every, int32_t region, int32_t nsamples) {
    int r = check_handle(h);
    if (r) return r;
    if (every < 0 || nsamples < 0) return fail(h, SGFD_ERR_INVALID, "negative audit interval or length");
    if (region < SGFD_REGION_COMPUTED || region > SGFD_REGION_PML)
        return fail(h, SGFD_ERR_INVALID, "bad region %d", region);
    if (every > 0 && nsamples == 0) return fail(h, SGFD_ERR_INVALID, "an audit needs at least one sample");
    if (every > 0 && h->storage != SGFD_STORE_F32)
        return fail(h, SGFD_ERR_UNSUPPORTED, "the per-step audit needs FP32 storage (use sgfd_energy)");
    SG_CUDA(h, cudaStreamSynchronize(h->stream), "synchronise before changing the audit");
    if (every == 0) {
        h->audit_every = 0;
        return SGFD_OK;
    }
    r = ensure_audit_scratch(h);
    if (r) return r;
    if (nsamples != h->audit_count) {
        cudaFree(h->audit_hist);
        h->audit_hist = nullptr;
        h->audit_count = 0;
        SG_CUDA(h, dev_malloc(h, &h->audit_hist, (size_t)nsamples * 2 * sizeof(double)), "audit history");
        h->audit_count = nsamples;
    }
    SG_CUDA(h, cudaMemsetAsync(h->audit_hist, 0, (size_t)nsamples * 2 * sizeof(double), h->stream), "audit history");
    h->audit_every = every;
    h->audit_region = region;
    return SGFD_OK;
}

int sgfd_get_audit(sgfd_solver *h, double *out) {
    int r = check_handle(h);
    if (r) return r;
    if (!out) return fail(h, SGFD_ERR_INVALID, "null output");
    if (h->audit_every == 0 || !h->audit_hist) return fail(h, SGFD_ERR_STATE, "no audit set (sgfd_set_audit)");
    SG_CUDA(h, cudaMemcpyAsync(out, h->audit_hist, (size_t)h->audit_count * 2 * sizeof(double),
                               cudaMemcpyDeviceToHost, h->stream), "audit download");
    SG_CUDA(h, cudaStreamSynchronize(h->stream), "audit download");
    return check_device_error(h);
}

// Ricker wavelet of the reference (OPT/ElasticWaveEquation.cu:184-189): the
// reference squares with pow(float, 2) in double precision and rounds to
// float, which equals the float product a*a.
float sgfd_ricker_ref(float f0, float dt, int32_t it) {
    const float pi = 3.1415926f;   // reference PI (OPT/ElasticMacro.h:19)
    const float t0 = std::ceil(1.0f / (f0 * dt));
    const float a = pi * f0 * (((float)it - t0) * dt - 1.0f / f0);
    const float a2 = (float)((double)a * (double)a);
    return (1.0f - 2.0f * a2) * std::exp(-a2);
}

float sgfd_ricker_t0(float f0, float dt, float t0, int32_t it) {
    const double a = 3.14159265358979323846 * (double)f0 * ((double)it * (double)dt - (double)t0);
    const double a2 = a * a;
    return (float)((1.0 - 2.0 * a2) * std::exp(-a2));
}

int sgfd_cell_counts(const sgfd_solver *h, int64_t *n_interior, int64_t *n_pml) {
    if (!h) return SGFD_ERR_INVALID;
    const Model &m = h->m;
    const int64_t total = (int64_t)m.nxc * m.nyc * m.nzc;
    if (n_pml) *n_pml = m.npml;
    if (n_interior) *n_interior = total - m.npml;
    return SGFD_OK;
}

int sgfd_device_allocations(const sgfd_solver *h, int64_t *count) {
    if (!h || !count) return SGFD_ERR_INVALID;
    *count = h->dev_allocs;
    return SGFD_OK;
}

int sgfd_launches_per_step(const sgfd_solver *h) {
    if (!h) return -1;
    const int audit = (h->audit_every > 0 ? 2 : 0) + (h->strip_n > 0 ? 2 : 0);
    if (h->storage != SGFD_STORE_F32) return half_launches_per_step(h->sr) + audit;   // either family
    if (h->kernel == SGFD_KERNEL_ZMARCH) return 2 + audit;
    return simple_launches_per_step(h->sr) + audit;
}

const char *sgfd_kernel_name(const sgfd_solver *h) {
    if (!h) return "";
    return h->kernel == SGFD_KERNEL_ZMARCH ? "zmarch" : "simple";
}

}  // extern "C"
