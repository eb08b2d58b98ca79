// Particle generation on the device, identical to the reference's particlegenerator
// (src/tools/UniformGenerator.cpp:12-28, src/tools/ClusteredGaussGenerator.cpp:15-47) followed by its
// 6-significant-digit CSV round trip (src/tools/particleToCSV.cpp, src/utility/utility.cpp:14-23).
//
// Uniform: std::mt19937(seed0); per particle three std::uniform_real_distribution<double>(0, 1)
// draws, z first (GCC evaluates std::make_tuple's arguments right to left), each formed from two
// 32-bit outputs as (lo + hi * 2^32) / 2^64 (libstdc++ generate_canonical<double, 53>), and
// position = corner + u * box with separately rounded multiply and add (no contraction).
//
// Clustered Gaussian: numClusters centres drawn like uniform particles from std::mt19937(seed1);
// numParticles / numClusters particles per centre, each offset per axis (z, y, x) by a
// std::normal_distribution<double>(mean, stddev) of its own (three objects, each caching the second
// value of the Marsaglia polar method), all three driven by one std::default_random_engine(seed0)
// (minstd_rand0: x <- 16807 x mod 2^31 - 1; a canonical double takes two outputs).
//
// On the GPU:
//   - mt19937 runs in one CTA: each 624-word twist in three dependency phases (words 0..226 from the
//     old state, 227..453 from the first phase, 454..623 from the second), then tempering.  The
//     stream is bit-identical to the host generator.
//   - The polar method's attempts are independent given their position in the minstd stream: thread
//     t finds its four engine outputs by jump-ahead (16807^(4t) mod m), tests acceptance, and a block
//     scan of the accepted flags assigns each accepted attempt its generation index g, hence the
//     particle pair (2 (g / 3), 2 (g / 3) + 1) and axis (z, y, x for g % 3 = 0, 1, 2): the first
//     particle of the pair takes y * mult, the second the cached x * mult.
//   - The CSV round trip (printf %g, 6 significant digits, then strtod) is reproduced exactly: the
//     scaled value v * 10^k is formed with its FMA residual, so the rounding to an integer sees the
//     exact product (ties to even), and the integer / 10^k is one correctly rounded division.
// The polar method's mult = sqrt(-2 log(r2) / r2) uses the device log, which can differ from the
// host library's in the last bit; after the 6-digit rounding the positions agree unless a value lies
// within an ulp of a decimal rounding boundary.
#include <cuda_runtime.h>
#include <stdint.h>

#include "tbmd_internal.cuh"

namespace tbmd {

namespace {

constexpr int MT_N = 624, MT_M = 397;
constexpr uint32_t MT_MATRIX = 0x9908b0dfu, MT_UPPER = 0x80000000u, MT_LOWER = 0x7fffffffu;

__device__ __forceinline__ uint32_t mt_next(uint32_t cur, uint32_t nxt, uint32_t far)
{
    const uint32_t y = (cur & MT_UPPER) | (nxt & MT_LOWER);
    return far ^ (y >> 1) ^ ((y & 1u) ? MT_MATRIX : 0u);
}

__device__ __forceinline__ uint32_t mt_temper(uint32_t y)
{
    y ^= y >> 11;
    y ^= (y << 7) & 0x9d2c5680u;
    y ^= (y << 15) & 0xefc60000u;
    y ^= y >> 18;
    return y;
}

// nwords outputs of std::mt19937(seed), in order.
__global__ void __launch_bounds__(640) k_mt19937(uint32_t seed, int64_t nwords, uint32_t *__restrict__ out)
{
    __shared__ uint32_t mt[MT_N];
    const int i = threadIdx.x;
    if (i == 0) {
        mt[0] = seed;
        for (int k = 1; k < MT_N; ++k) mt[k] = 1812433253u * (mt[k - 1] ^ (mt[k - 1] >> 30)) + (uint32_t)k;
    }
    __syncthreads();
    for (int64_t base = 0; base < nwords; base += MT_N) {
        // phase 1: words 0..226 (inputs: old state)
        uint32_t v = 0;
        if (i < MT_N - MT_M) v = mt_next(mt[i], mt[i + 1], mt[i + MT_M]);
        __syncthreads();
        if (i < MT_N - MT_M) mt[i] = v;
        __syncthreads();
        // phase 2: words 227..453 (far input: new words 0..226)
        const int j = i + (MT_N - MT_M);
        if (i < MT_N - MT_M) v = mt_next(mt[j], mt[j + 1], mt[j - (MT_N - MT_M)]);
        __syncthreads();
        if (i < MT_N - MT_M) mt[j] = v;
        __syncthreads();
        // phase 3: words 454..623 (far input: new words 227..396; word 623 also reads the new word 0)
        const int k = i + 2 * (MT_N - MT_M);
        if (k < MT_N) v = mt_next(mt[k], mt[(k + 1) % MT_N], mt[k - (MT_N - MT_M)]);
        __syncthreads();
        if (k < MT_N) mt[k] = v;
        __syncthreads();
        if (i < MT_N && base + i < nwords) out[base + i] = mt_temper(mt[i]);
        __syncthreads();
    }
}

// libstdc++ generate_canonical<double, 53> from two mt19937 outputs
__device__ __forceinline__ double canonical_mt(uint32_t lo, uint32_t hi)
{
    const double s = __dadd_rn((double)lo, __dmul_rn((double)hi, 4294967296.0));
    const double r = s * 0x1p-64;                // exact
    return r >= 1.0 ? 0x1.fffffffffffffp-1 : r;  // nextafter(1, 0)
}

// positions of n uniform particles (or cluster centres) from 6 n mt19937 words
__global__ void k_uniform_positions(int64_t n, const uint32_t *__restrict__ w, double cx, double cy, double cz,
                                    double bx, double by, double bz, double *x, double *y, double *z)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t *p = w + 6 * i;  // draws z, y, x
    z[i] = __dadd_rn(cz, __dmul_rn(canonical_mt(p[0], p[1]), bz));
    y[i] = __dadd_rn(cy, __dmul_rn(canonical_mt(p[2], p[3]), by));
    x[i] = __dadd_rn(cx, __dmul_rn(canonical_mt(p[4], p[5]), bx));
}

constexpr uint64_t MINSTD_M = 2147483647ull, MINSTD_A = 16807ull;

__device__ __forceinline__ uint64_t mulmod(uint64_t a, uint64_t b) { return (a * b) % MINSTD_M; }

__device__ __forceinline__ uint64_t powmod(uint64_t a, uint64_t e)
{
    uint64_t r = 1;
    while (e) {
        if (e & 1ull) r = mulmod(r, a);
        a = mulmod(a, a);
        e >>= 1;
    }
    return r;
}

// libstdc++ generate_canonical<double, 53> from two minstd_rand0 outputs (range 1 .. 2^31 - 2)
__device__ __forceinline__ double canonical_minstd(uint64_t o1, uint64_t o2)
{
    const double r = 2147483646.0;
    const double s = __dadd_rn((double)(o1 - 1), __dmul_rn((double)(o2 - 1), r));
    const double v = __ddiv_rn(s, __dmul_rn(r, r));
    return v >= 1.0 ? 0x1.fffffffffffffp-1 : v;
}

struct Attempt {
    double x, y, r2;
    bool ok;
};

// polar-method attempt t: engine outputs 4t+1 .. 4t+4 after the seed state x0
__device__ __forceinline__ Attempt attempt(uint64_t x0, uint64_t t)
{
    uint64_t s = mulmod(powmod(MINSTD_A, 4 * t), x0);
    const uint64_t o1 = s = mulmod(s, MINSTD_A);
    const uint64_t o2 = s = mulmod(s, MINSTD_A);
    const uint64_t o3 = s = mulmod(s, MINSTD_A);
    const uint64_t o4 = mulmod(s, MINSTD_A);
    Attempt a;
    a.x = __dsub_rn(2.0 * canonical_minstd(o1, o2), 1.0);
    a.y = __dsub_rn(2.0 * canonical_minstd(o3, o4), 1.0);
    a.r2 = __dadd_rn(__dmul_rn(a.x, a.x), __dmul_rn(a.y, a.y));
    a.ok = !(a.r2 > 1.0 || a.r2 == 0.0);
    return a;
}

constexpr int GEN_BLOCK = 1024;

// accepted attempts per block of GEN_BLOCK attempts starting at t0
__global__ void __launch_bounds__(GEN_BLOCK) k_polar_count(uint64_t x0, uint64_t t0, int64_t T,
                                                           unsigned int *__restrict__ block_count)
{
    __shared__ unsigned int wsum[GEN_BLOCK / 32];
    const int64_t t = (int64_t)blockIdx.x * GEN_BLOCK + threadIdx.x;
    const bool ok = t < T && attempt(x0, t0 + (uint64_t)t).ok;
    const unsigned m = __ballot_sync(0xffffffffu, ok);
    if ((threadIdx.x & 31) == 0) wsum[threadIdx.x >> 5] = __popc(m);
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned int s = 0;
        for (int k = 0; k < GEN_BLOCK / 32; ++k) s += wsum[k];
        block_count[blockIdx.x] = s;
    }
}

// exclusive scan of the block counts (one block; nb <= GEN_BLOCK * 64), generation index after the
// pass at [nb]
__global__ void __launch_bounds__(GEN_BLOCK) k_polar_scan(int nb, unsigned long long g0,
                                                          const unsigned int *__restrict__ count,
                                                          unsigned long long *__restrict__ start)
{
    __shared__ unsigned long long part[GEN_BLOCK];
    const int tid = threadIdx.x;
    const int chunk = (nb + GEN_BLOCK - 1) / GEN_BLOCK;
    const int b = tid * chunk, e = min(b + chunk, nb);
    unsigned long long s = 0;
    for (int k = b; k < e; ++k) s += count[k];
    part[tid] = s;
    __syncthreads();
    for (int off = 1; off < GEN_BLOCK; off <<= 1) {
        const unsigned long long v = tid >= off ? part[tid - off] : 0ull;
        __syncthreads();
        part[tid] += v;
        __syncthreads();
    }
    unsigned long long run = g0 + part[tid] - s;
    for (int k = b; k < e; ++k) {
        start[k] = run;
        run += count[k];
    }
    if (tid == GEN_BLOCK - 1) start[nb] = g0 + part[GEN_BLOCK - 1];
}

// accepted attempt with generation index g < G: the Gaussian pair of particles 2 (g / 3) and
// 2 (g / 3) + 1 on axis z, y, x (g % 3 = 0, 1, 2), added to their cluster centre
__global__ void __launch_bounds__(GEN_BLOCK) k_polar_place(uint64_t x0, uint64_t t0, int64_t T,
                                                           const unsigned long long *__restrict__ start,
                                                           unsigned long long G, int64_t m, int64_t per,
                                                           const double *__restrict__ cxs,
                                                           const double *__restrict__ cys,
                                                           const double *__restrict__ czs, double mean,
                                                           double stddev, double *x, double *y, double *z)
{
    __shared__ unsigned int wpre[GEN_BLOCK / 32];
    const int64_t t = (int64_t)blockIdx.x * GEN_BLOCK + threadIdx.x;
    const Attempt a = t < T ? attempt(x0, t0 + (uint64_t)t) : Attempt{0.0, 0.0, 0.0, false};
    const unsigned msk = __ballot_sync(0xffffffffu, a.ok);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) wpre[warp] = __popc(msk);
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned int s = 0;
        for (int k = 0; k < GEN_BLOCK / 32; ++k) {
            const unsigned int c = wpre[k];
            wpre[k] = s;
            s += c;
        }
    }
    __syncthreads();
    if (!a.ok) return;
    const unsigned long long g = start[blockIdx.x] + wpre[warp] + __popc(msk & ((1u << lane) - 1u));
    if (g >= G) return;
    const double mult = sqrt(__ddiv_rn(-2.0 * log(a.r2), a.r2));
    const int axis = 2 - (int)(g % 3);  // z, y, x
    const int64_t q0 = 2 * (int64_t)(g / 3);
    double *dst = axis == 0 ? x : (axis == 1 ? y : z);
    const double *cen = axis == 0 ? cxs : (axis == 1 ? cys : czs);
    const double v0 = __dadd_rn(__dmul_rn(__dmul_rn(a.y, mult), stddev), mean);
    const int64_t ncen = (m + per - 1) / per;
    dst[TBMD_IX(q0, m, BS_GEN)] = __dadd_rn(cen[TBMD_IX(q0 / per, ncen, BS_GEN)], v0);
    if (q0 + 1 < m) {
        const double v1 = __dadd_rn(__dmul_rn(__dmul_rn(a.x, mult), stddev), mean);
        dst[q0 + 1] = __dadd_rn(cen[TBMD_IX((q0 + 1) / per, ncen, BS_GEN)], v1);
    }
}

// 10^k, exact for 0 <= k <= 22
__device__ __forceinline__ double pow10_exact(int k)
{
    double p = 1.0;
    for (int i = 0; i < k; ++i) p *= 10.0;
    return p;
}

// Value of printf("%.6g", v) read back by strtod: v rounded to 6 significant decimal digits (ties to
// even on the exact binary value), then the nearest double.  Exact for 1e-17 <= |v| < 1e15.
__device__ double round_sig6(double v)
{
    if (v == 0.0 || !isfinite(v)) return v;
    const double a = fabs(v);
    int e = (int)floor(log10(a));
    for (int iter = 0; iter < 3; ++iter) {
        const int k = 5 - e;  // scale so that 1e5 <= a * 10^k < 1e6
        double p, err;
        if (k >= 0) {
            const double P = pow10_exact(k < 22 ? k : 22);
            p = a * P;
            err = fma(a, P, -p);  // a * P = p + err exactly
        } else {
            const double D = pow10_exact(-k);
            p = a / D;
            err = fma(-p, D, a);  // sign of the remainder a - p D
        }
        if (p < 1e5 || (p == 1e5 && err < 0)) {
            --e;
            continue;
        }
        if (p > 1e6 || (p == 1e6 && err >= 0)) {
            ++e;
            continue;
        }
        double n = rint(p);
        const double f = p - n;  // exact
        if (f == 0.5 && err > 0) n += 1.0;
        if (f == -0.5 && err < 0) n -= 1.0;
        const double r = k >= 0 ? n / pow10_exact(k < 22 ? k : 22) : n * pow10_exact(-k);
        return v < 0 ? -r : r;
    }
    return v;
}

__global__ void k_round_sig6(int64_t n, double *a)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) a[i] = round_sig6(a[i]);
}

__global__ void k_fill(int64_t n, double v, double *a)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) a[i] = v;
}

}  // namespace

cudaError_t launch_round_sig6(int64_t n, double *a, cudaStream_t st)
{
    if (n <= 0) return cudaSuccess;
    k_round_sig6<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(n, a);
    return cudaGetLastError();
}

cudaError_t launch_fill(int64_t n, double v, double *a, cudaStream_t st)
{
    if (n <= 0) return cudaSuccess;
    k_fill<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(n, v, a);
    return cudaGetLastError();
}

cudaError_t launch_mt19937(uint32_t seed, int64_t nwords, uint32_t *out, cudaStream_t st)
{
    k_mt19937<<<1, 640, 0, st>>>(seed, nwords, out);
    return cudaGetLastError();
}

cudaError_t launch_uniform_positions(int64_t n, const uint32_t *words, const double corner[3], const double box[3],
                                     double *x, double *y, double *z, cudaStream_t st)
{
    if (n <= 0) return cudaSuccess;
    k_uniform_positions<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(n, words, corner[0], corner[1], corner[2], box[0],
                                                                     box[1], box[2], x, y, z);
    return cudaGetLastError();
}

size_t polar_scratch_bytes(int64_t attempts)
{
    const int64_t nb = (attempts + GEN_BLOCK - 1) / GEN_BLOCK;
    return (size_t)nb * sizeof(unsigned int) + (size_t)(nb + 1) * sizeof(unsigned long long) + 64;
}

int64_t polar_attempts_per_pass() { return (int64_t)GEN_BLOCK * GEN_BLOCK * 64; }

cudaError_t launch_polar_pass(uint64_t x0, uint64_t t0, int64_t T, unsigned long long g0, unsigned long long G,
                              int64_t m, int64_t per, const double *const centres[3], double mean, double stddev,
                              double *x, double *y, double *z, void *scratch, unsigned long long *accepted_end,
                              cudaStream_t st)
{
    const int64_t nb = (T + GEN_BLOCK - 1) / GEN_BLOCK;
    unsigned int *count = (unsigned int *)scratch;
    unsigned long long *start =
        (unsigned long long *)((char *)scratch + ((nb * sizeof(unsigned int) + 15) / 16) * 16);
    k_polar_count<<<(unsigned)nb, GEN_BLOCK, 0, st>>>(x0, t0, T, count);
    k_polar_scan<<<1, GEN_BLOCK, 0, st>>>((int)nb, g0, count, start);
    k_polar_place<<<(unsigned)nb, GEN_BLOCK, 0, st>>>(x0, t0, T, start, G, m, per, centres[0], centres[1], centres[2],
                                                      mean, stddev, x, y, z);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    return cudaMemcpyAsync(accepted_end, start + nb, sizeof(unsigned long long), cudaMemcpyDeviceToHost, st);
}


// The bounds-check record of this translation unit (see TBMD_IX), read and cleared; zero when the
// library was built without the checks.
cudaError_t bounds_read_gen(BoundsRecord *out)
{
#ifdef TBMD_BOUNDS_CHECK
    cudaError_t e = cudaMemcpyFromSymbol(out, g_bounds_record, sizeof(BoundsRecord));
    if (e != cudaSuccess) return e;
    const BoundsRecord zero{};
    return cudaMemcpyToSymbol(g_bounds_record, &zero, sizeof(BoundsRecord));
#else
    *out = BoundsRecord{};
    return cudaSuccess;
#endif
}

}  // namespace tbmd
