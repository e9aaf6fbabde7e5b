// energy_noalloc.cu — sgfd_energy_noalloc: the FP64 energy audit of
// sgfd_energy, with its scratch in a fixed device array compiled into the
// library instead of memory the library asks the driver for on first use.
//
// Who needs it: sgfd_energy calls cudaMalloc for its partial sums the first
// time it runs on a handle.  Some callers cannot let a library allocate once
// they are running: a process whose device memory is held by another
// allocator (PyTorch's caching allocator, a serving framework's arena) can
// see that cudaMalloc fail although the pool has room, and a service that
// budgeted its device memory when it created its handles must not grow
// later.  This entry point allocates nothing: the partial sums live in
// g_energy_scratch, kNoAllocDoubles doubles (32 KiB) of file-scope device
// memory that every GPU which loads libsgfd.so holds until the process exits.
//
// Set-up: the first call on a device, with that device current, looks up the
// array's device address with cudaGetSymbolAddress and keeps it, with the
// identity of the device's current CUDA context, for later calls; make that
// first call before any stream capture.  The array belongs to the module the
// context loaded, so a later call that finds another context current (after
// cudaDeviceReset, or once the primary context was released and created
// again) looks the address up anew instead of using a stale one.  Every call
// on a device uses the same array and leaves its last contents there.
// Nothing in it has to start at zero: each partial-sum block writes its own
// slot before the final pass reads it, and the final pass writes both
// results.  Calls whose work overlaps on one GPU (two host threads, or two
// handles whose streams run at the same time) race on the array: serialise
// them.
#include <algorithm>
#include <mutex>

#include <cuda.h>
#include <cudaTypedefs.h>

#include "solver.h"

using namespace sgfd;

namespace {

// Largest number of partial-sum blocks the static scratch holds.
constexpr int kNoAllocBlocks = 2047;
constexpr int kNoAllocDoubles = 2 * kNoAllocBlocks + 2;   // partials, then (kinetic, strain)
constexpr int kMaxDevices = 64;

static __device__ __align__(256) double g_energy_scratch[kNoAllocDoubles];

std::mutex g_lookup_mu;
// Per device: the address of g_energy_scratch and the context it belongs to.
struct ScratchAddr {
    unsigned long long ctx_id = 0;
    double *ptr = nullptr;
};
ScratchAddr g_scratch[kMaxDevices];

// Identity of the CUDA context current on the calling thread (0 if none).
// The driver entry points come through the runtime, so the library does not
// link libcuda directly and still loads on a machine without a driver.
unsigned long long current_context_id() {
    static PFN_cuCtxGetCurrent_v4000 get_current = nullptr;
    static PFN_cuCtxGetId_v12000 get_id = nullptr;
    if (!get_current || !get_id) {
        void *p = nullptr, *q = nullptr;
        cudaDriverEntryPointQueryResult r1, r2;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &r1) != cudaSuccess ||
            r1 != cudaDriverEntryPointSuccess ||
            cudaGetDriverEntryPoint("cuCtxGetId", &q, cudaEnableDefault, &r2) != cudaSuccess ||
            r2 != cudaDriverEntryPointSuccess)
            return 0;
        get_current = reinterpret_cast<PFN_cuCtxGetCurrent_v4000>(p);
        get_id = reinterpret_cast<PFN_cuCtxGetId_v12000>(q);
    }
    CUcontext ctx = nullptr;
    unsigned long long id = 0;
    if (get_current(&ctx) != CUDA_SUCCESS || !ctx || get_id(ctx, &id) != CUDA_SUCCESS) return 0;
    return id;
}

}  // namespace

extern "C" int sgfd_energy_noalloc(sgfd_solver *h, int32_t region, int32_t nblocks, double *kinetic,
                                   double *strain) {
    int r = check_handle(h);   // also makes the handle's device current
    if (r) return r;
    if (region < SGFD_REGION_COMPUTED || region > SGFD_REGION_PML)
        return fail(h, SGFD_ERR_INVALID, "bad region %d", region);
    if (h->device < 0 || h->device >= kMaxDevices)
        return fail(h, SGFD_ERR_UNSUPPORTED, "device %d is beyond the %d devices the static scratch table covers",
                    h->device, kMaxDevices);
    if (nblocks < 0) return fail(h, SGFD_ERR_INVALID, "negative block count %d", nblocks);
    if (nblocks == 0) {   // the launch shape of sgfd_energy, within the static scratch
        int sms = 0;
        SG_CUDA(h, cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, h->device), "SM count");
        nblocks = std::min(energy_blocks(sms), kNoAllocBlocks);
    }
    if (nblocks > kNoAllocBlocks)
        return fail(h, SGFD_ERR_INVALID,
                    "%d partial-sum blocks need %d doubles of scratch; the static scratch holds %d "
                    "(at most %d blocks)", nblocks, 2 * nblocks + 2, kNoAllocDoubles, kNoAllocBlocks);
    // the context current on this device (check_handle's cudaSetDevice made
    // the device's primary context current)
    const unsigned long long ctx_id = current_context_id();
    if (!ctx_id) return fail(h, SGFD_ERR_CUDA, "no CUDA context current on device %d", h->device);
    double *scratch = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_lookup_mu);
        ScratchAddr &a = g_scratch[h->device];
        if (!a.ptr || a.ctx_id != ctx_id) {
            void *p = nullptr;
            SG_CUDA(h, cudaGetSymbolAddress(&p, g_energy_scratch), "device address of the static scratch");
            a.ptr = static_cast<double *>(p);
            a.ctx_id = ctx_id;
        }
        scratch = a.ptr;
    }
    r = sync_views(h);   // 16-bit storage: FP32 copies of the stored fields (no allocation)
    if (r) return r;
    double *out = scratch + 2 * nblocks;
    SG_CUDA(h, launch_energy(audit_model(h), h->ph, region, scratch, nblocks, out, h->stream), "energy audit");
    double res[2];
    SG_CUDA(h, cudaMemcpyAsync(res, out, sizeof res, cudaMemcpyDeviceToHost, h->stream), "energy download");
    SG_CUDA(h, cudaStreamSynchronize(h->stream), "energy download");
    r = check_device_error(h);
    if (r) return r;
    if (kinetic) *kinetic = res[0];
    if (strain) *strain = res[1];
    return SGFD_OK;
}
