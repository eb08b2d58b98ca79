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
// address with cudaGetSymbolAddress, checks the result and caches it per device; later calls reuse
// it.  Make that first call before any stream capture.  All calls share the array and it keeps
// the last call's contents.  The work counter is cleared at the start of every call; every partial
// slot a call reads, that call has written first.  Calls that overlap on the GPU (on different
// streams, or from different host threads) race on the array and must be serialised by the caller.
//
// Limits: 1 <= n <= TBMD_NOALLOC_MAX_N (4096).  Larger n returns TBMD_TOO_LARGE before anything
// is launched.  No cudaMalloc, cudaFree or allocating library routine is called.
#include <cuda_runtime.h>

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
    void *ptr = nullptr;
    int sms = 0;
};
std::mutex g_mu;
DeviceScratch g_dev[kMaxDevices];

// Once per device, with that device current: the device address of the scratch array.
cudaError_t device_scratch(int dev, void **ptr, int *sms)
{
    std::lock_guard<std::mutex> lock(g_mu);
    DeviceScratch &d = g_dev[dev];
    if (!d.ready) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return e;
        int n_sms = 0;
        e = cudaDeviceGetAttribute(&n_sms, cudaDevAttrMultiProcessorCount, dev);
        if (e != cudaSuccess) return e;
        d.ptr = p;
        d.sms = n_sms;
        d.ready = true;
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
    if (!(nu == nu)) return TBMD_INVALID_ARG;
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
