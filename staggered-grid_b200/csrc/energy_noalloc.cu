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
// array's device address with cudaGetSymbolAddress and keeps it for later
// calls; make that first call before any stream capture.  Every call on a
// device uses the same array and leaves its last contents there.  Nothing in
// it has to start at zero: each partial-sum block writes its own slot before
// the final pass reads it, and the final pass writes both results.  Calls
// whose work overlaps on one GPU (two host threads, or two handles whose
// streams run at the same time) race on the array: serialise them.
#include <mutex>

#include "solver.h"

using namespace sgfd;

namespace {

// Largest number of partial-sum blocks the static scratch holds.
constexpr int kNoAllocBlocks = 2047;
constexpr int kNoAllocDoubles = 2 * kNoAllocBlocks + 2;   // partials, then (kinetic, strain)
constexpr int kMaxDevices = 64;

static __device__ __align__(256) double g_energy_scratch[kNoAllocDoubles];

std::mutex g_lookup_mu;
double *g_scratch_ptr[kMaxDevices] = {};   // device address of g_energy_scratch, per device

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
    if (nblocks == 0) {   // the launch shape of sgfd_energy
        int sms = 0;
        SG_CUDA(h, cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, h->device), "SM count");
        nblocks = energy_blocks(sms);
    }
    if (nblocks > kNoAllocBlocks)
        return fail(h, SGFD_ERR_INVALID,
                    "%d partial-sum blocks need %d doubles of scratch; the static scratch holds %d "
                    "(at most %d blocks)", nblocks, 2 * nblocks + 2, kNoAllocDoubles, kNoAllocBlocks);
    double *scratch = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_lookup_mu);
        if (!g_scratch_ptr[h->device]) {
            void *p = nullptr;
            SG_CUDA(h, cudaGetSymbolAddress(&p, g_energy_scratch), "device address of the static scratch");
            g_scratch_ptr[h->device] = static_cast<double *>(p);
        }
        scratch = g_scratch_ptr[h->device];
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
