// Allocation-free NATA forces (tbmd_nata_forces_noalloc in include/tbmd.h).
//
// Why it exists: some callers cannot allocate device memory at the moment they need forces.
// Examples are code that runs inside a fixed, pre-reserved device-memory budget (embedded or
// certified builds that forbid run-time allocation), code called back from another library
// while that library owns the allocator, and latency-critical loops that must not pay for
// cudaMalloc's implicit synchronisation.  Creating a context (tbmd_create) allocates, so this
// entry point takes no context.  The caller passes device buffers for the positions and the
// forces.  The only other memory is a fixed scratch area in this file: the NATA kernel's partial
// sums, one slot per (particle, j-block), plus its work counter.
//
// The scratch is a file-scope static __device__ array of NOALLOC_SCRATCH_BYTES (a little over
// 3 MiB).  Every GPU that loads the library holds it until the process exits.  On the host its
// name is only a stand-in for the device symbol, not a device address, so it is never passed to
// a kernel directly.  Instead, the first call on a device (with that device current) resolves the
// address with cudaGetSymbolAddress, checks the result and caches it for that device together
// with the unique id of the CUDA context that was current (cuCtxGetId); later calls reuse it while
// the same context is current.  A symbol's address belongs to one context, so when the context
// changes (after cudaDeviceReset, or when the caller made another context current on the device)
// the next call resolves it again instead of launching on a stale address.  Make the first call on
// a device, and the first call after such a change, before any stream capture.  All calls share
// the array and it keeps the last call's contents.  The work counter is cleared at the start of
// every call; every partial slot a call reads, that call has written first.  Calls that overlap on
// the GPU (on different streams, or from different host threads) race on the array and must be
// serialised by the caller.
//
// Limits: 1 <= n <= TBMD_NOALLOC_MAX_N (4096).  Larger n returns TBMD_TOO_LARGE before anything
// is launched.  No cudaMalloc, cudaFree or allocating library routine is called.
#include <cuda.h>
#include <cuda_runtime.h>

#include <cmath>
#include <mutex>

#include "../../include/tbmd.h"
#include "tbmd_internal.cuh"

namespace {

constexpr int kR = 4;                                                // j's per lane (JB = 128)
constexpr int kJB = 32 * kR;
constexpr int64_t kMaxN = TBMD_NOALLOC_MAX_N;
constexpr int64_t kMaxBlocks = (kMaxN - 2 + kJB) / kJB;              // j-blocks at kMaxN
constexpr size_t kPartialBytes = sizeof(double) * 3 * kMaxN * kMaxBlocks;  // 3 MiB
constexpr size_t NOALLOC_SCRATCH_BYTES = kPartialBytes + 256;       // + work counter

static __device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_SCRATCH_BYTES];

constexpr int kMaxDevices = 64;
struct DeviceScratch {
    bool ready = false;
    unsigned long long ctx_id = 0;  // unique id of the context the address belongs to
    void *ptr = nullptr;
    int sms = 0;
};
std::mutex g_mu;
DeviceScratch g_dev[kMaxDevices];

// Driver entry points for the current context's unique id, fetched through the runtime (no link
// against the driver library).  Both stay null on a driver without them; the address is then
// resolved on every call.
using CtxGetCurrentFn = CUresult (*)(CUcontext *);
using CtxGetIdFn = CUresult (*)(CUcontext, unsigned long long *);
CtxGetCurrentFn g_ctx_get_current = nullptr;
CtxGetIdFn g_ctx_get_id = nullptr;
std::once_flag g_entry_once;

void load_entry_points()
{
    void *f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &f, 12000, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
        g_ctx_get_current = (CtxGetCurrentFn)f;
    f = nullptr;
    if (cudaGetDriverEntryPointByVersion("cuCtxGetId", &f, 12000, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
        g_ctx_get_id = (CtxGetIdFn)f;
}

// Unique id of the context current on this thread; false when there is none or it is unknown.
bool current_context_id(unsigned long long *id)
{
    std::call_once(g_entry_once, load_entry_points);
    if (!g_ctx_get_current || !g_ctx_get_id) return false;
    CUcontext ctx = nullptr;
    if (g_ctx_get_current(&ctx) != CUDA_SUCCESS || ctx == nullptr) return false;
    return g_ctx_get_id(ctx, id) == CUDA_SUCCESS;
}

// With the device current: the device address of the scratch array in the current context,
// resolved once per (device, context) and cached.
cudaError_t device_scratch(int dev, void **ptr, int *sms)
{
    std::lock_guard<std::mutex> lock(g_mu);
    DeviceScratch &d = g_dev[dev];
    unsigned long long id = 0;
    const bool known = current_context_id(&id);
    if (!d.ready || !known || d.ctx_id != id) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);  // creates the context if needed
        if (e != cudaSuccess) return e;
        int n_sms = 0;
        e = cudaDeviceGetAttribute(&n_sms, cudaDevAttrMultiProcessorCount, dev);
        if (e != cudaSuccess) return e;
        d.ptr = p;
        d.sms = n_sms;
        // cache only when the context the address belongs to is known
        d.ready = current_context_id(&d.ctx_id);
        *ptr = p;
        *sms = n_sms;
        return cudaSuccess;
    }
    *ptr = d.ptr;
    *sms = d.sms;
    return cudaSuccess;
}

}  // namespace

extern "C" tbmd_status tbmd_nata_forces_noalloc(int64_t n, const double *x, const double *y, const double *z,
                                                double nu, int32_t precision, double *fx, double *fy, double *fz,
                                                void *stream)
{
    if (!x || !y || !z || !fx || !fy || !fz) return TBMD_INVALID_ARG;
    if (precision != TBMD_FP64 && precision != TBMD_MIXED) return TBMD_INVALID_ARG;
    if (!std::isfinite(nu)) return TBMD_INVALID_ARG;
    if (n < 1) return TBMD_INVALID_ARG;
    if (n > kMaxN) return TBMD_TOO_LARGE;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return TBMD_NO_DEVICE;
    void *scratch = nullptr;
    int sms = 0;
    if (device_scratch(dev, &scratch, &sms) != cudaSuccess) return TBMD_CUDA_ERROR;
    cudaStream_t st = (cudaStream_t)stream;
    using namespace tbmd;
    const Out out{fx, fy, fz, nullptr, nullptr, nullptr};
    if (n < 3) {  // no triplets: zero forces
        if (cudaMemsetAsync(fx, 0, sizeof(double) * n, st) != cudaSuccess ||
            cudaMemsetAsync(fy, 0, sizeof(double) * n, st) != cudaSuccess ||
            cudaMemsetAsync(fz, 0, sizeof(double) * n, st) != cudaSuccess)
            return TBMD_CUDA_ERROR;
        return TBMD_OK;
    }
    double *partial = (double *)scratch;
    unsigned int *counter = (unsigned int *)((char *)scratch + kPartialBytes);
    if (cudaMemsetAsync(counter, 0, sizeof(unsigned int), st) != cudaSuccess) return TBMD_CUDA_ERROR;
    const int nb = (int)((n - 2 + kJB) / kJB);
    SweepWork work{nullptr, nb, (int64_t)nb * n, counter};
    const Pos pos{x, y, z, nullptr, nullptr, nullptr};
    if (launch_nata(precision == TBMD_MIXED, false, kR, false, n, pos, out, nullptr, nu, work, partial, sms * 8, st) !=
        cudaSuccess)
        return TBMD_CUDA_ERROR;
    if (launch_nata_reduce(false, n, nb, partial, out, st) != cudaSuccess) return TBMD_CUDA_ERROR;
    return TBMD_OK;
}
