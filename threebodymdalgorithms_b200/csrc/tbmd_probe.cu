// FMA pipe throughput probe (include/tbmd_probe.h).  Each thread runs 8 independent FMA chains
// (enough to cover the pipe latency with 8+ warps per scheduler) for `iters` rounds and stores
// the sum so the work stays live.
#include <cuda_runtime.h>

#include "../../include/tbmd_probe.h"

namespace {

template <class T>
__global__ void __launch_bounds__(256) k_fma(T *out, int iters, T a, T b)
{
    T x0 = threadIdx.x, x1 = x0 + 1, x2 = x0 + 2, x3 = x0 + 3, x4 = x0 + 4, x5 = x0 + 5, x6 = x0 + 6, x7 = x0 + 7;
#pragma unroll 4
    for (int i = 0; i < iters; ++i) {
        x0 = x0 * a + b;
        x1 = x1 * a + b;
        x2 = x2 * a + b;
        x3 = x3 * a + b;
        x4 = x4 * a + b;
        x5 = x5 * a + b;
        x6 = x6 * a + b;
        x7 = x7 * a + b;
    }
    out[blockIdx.x * blockDim.x + threadIdx.x] = ((x0 + x1) + (x2 + x3)) + ((x4 + x5) + (x6 + x7));
}

template <class T>
double run_on_current(int device)
{
    int sms = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess || sms < 1) return -1.0;
    const int blocks = sms * 8, threads = 256, iters = sizeof(T) == 8 ? 4096 : 8192;
    T *out = nullptr;
    if (cudaMalloc(&out, sizeof(T) * blocks * threads) != cudaSuccess) return -1.0;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    double result = -1.0;
    if (cudaEventCreate(&e0) == cudaSuccess && cudaEventCreate(&e1) == cudaSuccess) {
        k_fma<T><<<blocks, threads>>>(out, iters, T(0.999999), T(1e-7));  // warm-up
        float best = 1e30f;
        bool ok = cudaGetLastError() == cudaSuccess;
        for (int rep = 0; ok && rep < 5; ++rep) {
            ok = cudaEventRecord(e0) == cudaSuccess;
            k_fma<T><<<blocks, threads>>>(out, iters, T(0.999999), T(1e-7));
            ok = ok && cudaGetLastError() == cudaSuccess && cudaEventRecord(e1) == cudaSuccess &&
                 cudaEventSynchronize(e1) == cudaSuccess;
            float ms = 0;
            ok = ok && cudaEventElapsedTime(&ms, e0, e1) == cudaSuccess;
            if (ok && ms < best) best = ms;
        }
        if (ok && best > 0.f && best < 1e30f) {
            const double flops = 2.0 * 8.0 * (double)iters * blocks * threads;
            result = flops / (best * 1e-3) / 1e12;
        }
    }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    cudaFree(out);
    return result;
}

// Runs on `device` and leaves the caller's current device as it was.
template <class T>
double run(int device)
{
    int prev = 0;
    if (cudaGetDevice(&prev) != cudaSuccess) return -1.0;
    if (cudaSetDevice(device) != cudaSuccess) return -1.0;
    const double r = run_on_current<T>(device);
    if (cudaSetDevice(prev) != cudaSuccess) return -1.0;
    return r;
}

}  // namespace

extern "C" double tbmd_probe_fma_tflops(int32_t device, int32_t fp64)
{
    return fp64 ? run<double>(device) : run<float>(device);
}
