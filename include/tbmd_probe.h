/*
 * tbmd_probe.h - measurement helper exported by libtbmd.so (no counterpart in the reference).
 *
 * The roofline of the triplet kernels is the FP32 pipe (mixed precision) or the FP64 pipe (FP64
 * drop-in), not a tensor core or HBM figure, so the benchmark measures those pipe peaks on the
 * device it runs on with a dependent-chain-free FMA loop.
 */
#ifndef TBMD_PROBE_H
#define TBMD_PROBE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Measured FMA throughput of `device` in TFLOP/s (an FMA counts 2 FLOP): fp64 = 0 for the FP32
 * pipe, 1 for the FP64 pipe.  Runs about 0.1-0.3 s; returns a negative value on a CUDA error.  The
 * calling thread's current device is the same afterwards. */
double tbmd_probe_fma_tflops(int32_t device, int32_t fp64);

#ifdef __cplusplus
}
#endif

#endif
