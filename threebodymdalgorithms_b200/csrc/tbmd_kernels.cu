// CUDA kernels (sm_100a) of the Axilrod-Teller three-body path.
//
//   k_auta       AUTA: every unique triplet i < j < k once (Algorithm.cpp:72-141 with one owner).
//                A warp takes a work item (block of 32*R consecutive j, one i): lanes own the j
//                (register accumulators), k sweeps the rest of the system in tiles of 32 staged in
//                shared memory.  The k-side contributions travel with a rotating accumulator (one
//                shuffle per tile step) so that after 32 steps lane l holds the complete sum for
//                k = tile + l and writes it with one FP64 atomic.  i's force is -(sum of the j- and
//                k-side totals) by translation invariance, so it costs nothing per triplet.
//   k_nata       NATA: all triplets seen from each particle i; only grad_i is accumulated (in the
//                well-conditioned (u, w) or (v, w) form of at_self), no atomics; per-(i, j-block)
//                partial sums are reduced in a fixed order (deterministic).
//   k_cell_*     P3BCA cell grid: wrap-and-bin (FP64, same arithmetic as the oracle), counting sort
//                by cell, stable within a cell.
//   k_neighbors  half neighbour lists (sorted index t > s) with the reference's exact FP64
//                periodic cutoff test (structs.hpp:106-115; d == cutoff is inside).
//   k_p3bca      warp per particle s: all pairs (a < b) of its half list, guarded cutoff test of the
//                third edge (exact decision), triplet math, per-slot accumulation in shared memory,
//                one FP64 atomic per list slot.
//   k_predictor / k_update   the reference's integrator (structs.hpp:40-99), FP64.
//
// Precision: S = double is the FP64 drop-in.  S = float is the mixed form: displacements are
// formed in FP64 from FP64 positions and rounded once (relative to particle i, so they are small
// and accurate), the triplet geometry and coefficients are FP32, short FP32 partial sums (at
// most one 32-wide tile) are flushed into FP64 accumulators, and all global accumulation is FP64.
// S = Dual<T> is the adjoint: the same kernels carry a tangent (the cotangent on the forces as a
// direction) and return H * direction alongside the forces.
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <cstring>
#include <type_traits>

#include "tbmd_internal.cuh"

namespace tbmd {

// One k entry staged in shared memory: edge v from i (hi part), b = v.v, and for the mixed form
// the lo part of v.
template <class S>
struct Tile {
    S vx, vy, vz, b;
    __device__ __forceinline__ V3<S> lo() const { return vzero<S>(); }
    __device__ __forceinline__ void set_lo(V3<S>) {}
};
template <>
struct Tile<float> {
    float vx, vy, vz, b, lx, ly, lz, pad;
    __device__ __forceinline__ V3<float> lo() const { return {lx, ly, lz}; }
    __device__ __forceinline__ void set_lo(V3<float> l)
    {
        lx = l.x;
        ly = l.y;
        lz = l.z;
    }
};
template <>
struct Tile<Dual<float>> {
    Dual<float> vx, vy, vz, b, lx, ly, lz, pad;
    __device__ __forceinline__ V3<Dual<float>> lo() const { return {lx, ly, lz}; }
    __device__ __forceinline__ void set_lo(V3<Dual<float>> l)
    {
        lx = l.x;
        ly = l.y;
        lz = l.z;
    }
};

template <class S>
__device__ __forceinline__ V3<typename Traits<S>::Acc> widen(V3<S> a)
{
    return {to_acc(a.x), to_acc(a.y), to_acc(a.z)};
}

template <class A>
__device__ __forceinline__ V3<A> warp_sum3(V3<A> v)
{
    return {warp_sum(v.x), warp_sum(v.y), warp_sum(v.z)};
}

// Edge x_j - x_i: FP64 subtraction, then hi/lo split (see split); the tangent carries d_j - d_i.
template <class S>
__device__ __forceinline__ void edge(const Pos &p, int64_t j, double xi, double yi, double zi, double dxi, double dyi,
                                     double dzi, V3<S> &h, V3<S> &l)
{
    const bool dual = Traits<S>::dual;
    split<S>(p.x[j] - xi, dual ? p.dx[j] - dxi : 0.0, h.x, l.x);
    split<S>(p.y[j] - yi, dual ? p.dy[j] - dyi : 0.0, h.y, l.y);
    split<S>(p.z[j] - zi, dual ? p.dz[j] - dzi : 0.0, h.z, l.z);
}

// The six scalars of a triplet from the edges u, v (hi/lo) of vertex i; c, q and s come from the
// third edge w itself (returned for the gradients), so no scalar is a difference of nearly equal
// numbers.
template <bool ENERGY, class S>
__device__ __forceinline__ ATCoef<S> triplet(V3<S> uh, V3<S> ul, S a, V3<S> vh, V3<S> vl, S b, S nu, S nu3, S nu15,
                                             bool valid, S &e, V3<S> &w)
{
    w = third_edge(uh, ul, vh, vl);
    return at_coef<ENERGY>(a, b, dot3(w, w), dot_uv(uh, ul, vh, vl, w), dot3(uh, w), dot3(vh, w), nu, nu3, nu15,
                           valid, e);
}

// Decode a sweep work item: block b with prefix[b] <= w < prefix[b+1], i = w - prefix[b].
__device__ __forceinline__ int find_block(const int64_t *prefix, int nblocks, int64_t w)
{
    int lo = 0, hi = nblocks;
    while (hi - lo > 1) {
        int mid = (lo + hi) >> 1;
        if (__ldg(prefix + mid) <= w)
            lo = mid;
        else
            hi = mid;
    }
    return lo;
}

// value part as FP64
__device__ __forceinline__ double to_double(double v) { return v; }
__device__ __forceinline__ double to_double(float v) { return (double)v; }
template <class T>
__device__ __forceinline__ double to_double(Dual<T> v) { return (double)v.v; }

// value part as FP32 (comparisons that only choose between equivalent forms)
template <class S>
__device__ __forceinline__ float to_float(S v);
template <>
__device__ __forceinline__ float to_float<float>(float v) { return v; }
template <>
__device__ __forceinline__ float to_float<double>(double v) { return (float)v; }
template <>
__device__ __forceinline__ float to_float<Dual<double>>(Dual<double> v) { return (float)v.v; }
template <>
__device__ __forceinline__ float to_float<Dual<float>>(Dual<float> v) { return v.v; }

// ---------------------------------------------------------------------------------------------
// AUTA sweep

// Register bound of the sweeps: the mixed form at R = 4 must fit two blocks of 8 warps per SM (128
// registers); left free, its energy variant took 174 and ran 8% slower on the batched C5 systems.
// The other forms keep the compiler's own choice.
template <class S, int R>
struct SweepMinBlocks {
    static constexpr int value = 1;
};
template <>
struct SweepMinBlocks<float, 4> {
    static constexpr int value = 2;
};

template <class S, int R, bool ENERGY, int WARPS>
__global__ void __launch_bounds__(WARPS * 32, (SweepMinBlocks<S, R>::value))
    k_auta(int64_t n, Pos pos, Out out, double *energy_out, double nu_d, SweepWork work)
{
    using Acc = typename Traits<S>::Acc;
    constexpr int JB = 32 * R;
    __shared__ Tile<S> tile[WARPS][32];
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    const S nu = constant<S>(nu_d), nu3 = constant<S>(-3.0 * nu_d), nu15 = constant<S>(15.0 * nu_d);

    unsigned int w = 0;
    if (lane == 0) w = atomicAdd(work.counter, 1u);
    w = __shfl_sync(0xffffffffu, w, 0);
    while ((int64_t)w < work.total) {
        unsigned int wn = 0;
        if (lane == 0) wn = atomicAdd(work.counter, 1u);
        // system, then (block, i) inside it
        const int sys = (int)TBMD_IX(work.nsys > 1 ? find_block(work.sys_items, work.nsys, (int64_t)w) : 0, work.nsys,
                                     BS_SYSTEM);
        const int64_t wl = (int64_t)w - work.sys_items[sys];
        const int64_t off = work.sys_off[sys], hi = work.sys_off[sys + 1];
        const int64_t *prefix = work.prefix + work.sys_prefix[sys];
        const int b = find_block(prefix, work.sys_nblocks[sys], wl);
        // item -> (i, k range): the whole sweep from the block, or one segment of it
        int64_t i = off + wl - prefix[b], kbeg = off + (int64_t)b * JB, kend = hi;
        if (work.kseg > 0) {
            const int64_t r = wl - prefix[b], nseg = (hi - kbeg + work.kseg - 1) / work.kseg;
            i = off + r / nseg;
            kbeg += (r % nseg) * work.kseg;
            kend = min(hi, kbeg + work.kseg);
        }
        i = TBMD_IX(i, n, BS_SWEEP);
        const double xi = pos.x[i], yi = pos.y[i], zi = pos.z[i];
        double dxi = 0.0, dyi = 0.0, dzi = 0.0;
        if (Traits<S>::dual) {
            dxi = pos.dx[i];
            dyi = pos.dy[i];
            dzi = pos.dz[i];
        }
        V3<S> u[R], ul[R];
        S aa[R];
        int64_t jj[R];
        bool jv[R];
        V3<Acc> fj[R];
#pragma unroll
        for (int r = 0; r < R; ++r) {
            jj[r] = off + (int64_t)b * JB + r * 32 + lane;
            jv[r] = jj[r] > i && jj[r] < hi;
            u[r] = vzero<S>();
            ul[r] = vzero<S>();
            if (jv[r]) edge<S>(pos, jj[r], xi, yi, zi, dxi, dyi, dzi, u[r], ul[r]);
            aa[r] = dot3(u[r], u[r]);
            fj[r] = widen(vzero<S>());
        }
        V3<Acc> fi = widen(vzero<S>());
        Acc en_item = to_acc(szero<S>());
        for (int64_t kt = kbeg; kt < kend; kt += 32) {
            const int64_t k = kt + lane;
            const bool kv = k < kend;
            V3<S> vk = vzero<S>(), vkl = vzero<S>();
            if (kv) edge<S>(pos, k, xi, yi, zi, dxi, dyi, dzi, vk, vkl);
            {
                Tile<S> tl;
                tl.vx = vk.x;
                tl.vy = vk.y;
                tl.vz = vk.z;
                tl.b = dot3(vk, vk);
                tl.set_lo(vkl);
                tile[wib][lane] = tl;
            }
            __syncwarp();
            S al[R];
            V3<S> gv[R];
#pragma unroll
            for (int r = 0; r < R; ++r) {
                al[r] = szero<S>();
                gv[r] = vzero<S>();
            }
            S bsum = szero<S>();
            V3<S> gw = vzero<S>();
            S en = szero<S>();
#pragma unroll 2
            for (int t = 0; t < 32; ++t) {
                const int kk = (lane + t) & 31;
                const Tile<S> e = tile[wib][kk];
                const V3<S> v = {e.vx, e.vy, e.vz};
                const V3<S> vl = e.lo();
                const int64_t kidx = kt + kk;
#pragma unroll
                for (int r = 0; r < R; ++r) {
                    const bool valid = jv[r] && kidx > jj[r] && kidx < kend;
                    V3<S> ec;  // third edge x_k - x_j
                    const ATCoef<S> cf = triplet<ENERGY>(u[r], ul[r], aa[r], v, vl, e.b, nu, nu3, nu15, valid, en, ec);
                    al[r] = al[r] + cf.alpha;
                    gv[r] = fma3(ec, cf.gamma, gv[r]);
                    bsum = bsum + cf.beta;
                    gw = fma3(ec, -cf.gamma, gw);
                }
                const int src = (lane + 1) & 31;
                bsum = shfl_idx(bsum, src);
                gw = shfl_idx(gw, src);
            }
            // After the full rotation lane l holds the k-side sums of k = kt + l.
            const V3<Acc> fk = widen(fma3(vk, bsum, gw));
            if (kv) atomic_out(out, k, fk);
            fi = fi - fk;
#pragma unroll
            for (int r = 0; r < R; ++r) {
                const V3<Acc> f = widen(fma3(u[r], al[r], gv[r]));
                fj[r] = fj[r] + f;
                fi = fi - f;
            }
            if (ENERGY) en_item = en_item + to_acc(en);
            __syncwarp();
        }
#pragma unroll
        for (int r = 0; r < R; ++r)
            if (jv[r]) atomic_out(out, jj[r], fj[r]);
        fi = warp_sum3(fi);
        if (lane == 0) atomic_out(out, i, fi);
        if (ENERGY) {
            en_item = warp_sum(en_item);
            if (lane == 0) atomicAdd(energy_out + sys, acc_value(en_item));
        }
        w = __shfl_sync(0xffffffffu, wn, 0);
    }
}

// ---------------------------------------------------------------------------------------------
// NATA sweep: item (j-block b, particle i) sums grad_i over all pairs j < k (j in block b, both
// different from i).  Energy is counted only for i < j < k, so each triplet's energy once.

template <class S, int R, bool ENERGY, int WARPS>
__global__ void __launch_bounds__(WARPS * 32) k_nata(int64_t n, Pos pos, double *partial, double *energy_out,
                                                    double nu_d, SweepWork work)
{
    using Acc = typename Traits<S>::Acc;
    constexpr int JB = 32 * R;
    __shared__ Tile<S> tile[WARPS][32];
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    const S nu = constant<S>(nu_d), nu3 = constant<S>(-3.0 * nu_d), nu15 = constant<S>(15.0 * nu_d);
    Acc en_acc = to_acc(szero<S>());
    const int nb = work.nblocks;

    unsigned int w = 0;
    if (lane == 0) w = atomicAdd(work.counter, 1u);
    w = __shfl_sync(0xffffffffu, w, 0);
    while ((int64_t)w < work.total) {
        unsigned int wn = 0;
        if (lane == 0) wn = atomicAdd(work.counter, 1u);
        const int b = (int)((int64_t)w / n);
        const int64_t i = TBMD_IX((int64_t)w - (int64_t)b * n, n, BS_SWEEP);
        const double xi = pos.x[i], yi = pos.y[i], zi = pos.z[i];
        V3<S> u[R], ul[R];
        S aa[R];
        int64_t jj[R];
        bool jv[R];
#pragma unroll
        for (int r = 0; r < R; ++r) {
            jj[r] = (int64_t)b * JB + r * 32 + lane;
            jv[r] = jj[r] < n && jj[r] != i;
            u[r] = vzero<S>();
            ul[r] = vzero<S>();
            if (jv[r]) edge<S>(pos, jj[r], xi, yi, zi, 0.0, 0.0, 0.0, u[r], ul[r]);
            aa[r] = dot3(u[r], u[r]);
        }
        V3<Acc> g = widen(vzero<S>());
        for (int64_t kt = (int64_t)b * JB; kt < n; kt += 32) {
            const int64_t k = kt + lane;
            V3<S> vk = vzero<S>(), vkl = vzero<S>();
            if (k < n) edge<S>(pos, k, xi, yi, zi, 0.0, 0.0, 0.0, vk, vkl);
            {
                Tile<S> tl;
                tl.vx = vk.x;
                tl.vy = vk.y;
                tl.vz = vk.z;
                tl.b = dot3(vk, vk);
                tl.set_lo(vkl);
                tile[wib][lane] = tl;
            }
            __syncwarp();
            S A[R];
#pragma unroll
            for (int r = 0; r < R; ++r) A[r] = szero<S>();
            V3<S> Tw = vzero<S>();
            S en = szero<S>();
#pragma unroll 2
            for (int t = 0; t < 32; ++t) {
                const Tile<S> e = tile[wib][t];
                const V3<S> v = {e.vx, e.vy, e.vz};
                const V3<S> vl = e.lo();
                const int64_t kidx = kt + t;
                const bool kv = kidx < n && kidx != i;
                S sv = szero<S>();  // sigma of the pairs taken in the (v, w) basis, for this k
#pragma unroll
                for (int r = 0; r < R; ++r) {
                    const bool valid = jv[r] && kv && kidx > jj[r];
                    S e_r = szero<S>();
                    const V3<S> w = third_edge(u[r], ul[r], v, vl);
                    // basis (u, w) when |u| <= |v|, else (v, w): see at_self
                    const bool ub = to_float(aa[r]) <= to_float(e.b);
                    const ATSelf<S> cf = at_self<ENERGY>(aa[r], e.b, dot3(w, w), dot_uv(u[r], ul[r], v, vl, w), dot3(u[r], w),
                                                         dot3(v, w), nu, nu3, nu15, valid, ub, e_r);
                    if (ENERGY && i < jj[r]) en = en + e_r;
                    if (ub)
                        A[r] = A[r] + cf.sigma;
                    else
                        sv = sv + cf.sigma;
                    Tw = fma3(w, cf.kappa, Tw);
                }
                Tw = fma3(v, sv, Tw);
            }
            V3<S> gt = Tw;
#pragma unroll
            for (int r = 0; r < R; ++r) gt = fma3(u[r], A[r], gt);
            g = g + widen(gt);
            if (ENERGY) en_acc = en_acc + to_acc(en);
            __syncwarp();
        }
        g = warp_sum3(g);
        if (lane == 0) {
            double *dst = partial + TBMD_IX(((int64_t)i * nb + b) * 3, n * nb * 3, BS_PARTIAL);
            dst[0] = -acc_value(g.x);
            dst[1] = -acc_value(g.y);
            dst[2] = -acc_value(g.z);
        }
        w = __shfl_sync(0xffffffffu, wn, 0);
    }
    if (ENERGY) {
        en_acc = warp_sum(en_acc);
        if (lane == 0) atomicAdd(energy_out, acc_value(en_acc));
    }
}

// f_i = sum over blocks b of partial[i][b], in block order.
__global__ void k_nata_reduce(int64_t n, int nb, const double *__restrict__ partial, Out out)
{
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double sx = 0.0, sy = 0.0, sz = 0.0;
    const double *p = partial + i * nb * 3;
    for (int b = 0; b < nb; ++b) {
        sx += p[3 * b + 0];
        sy += p[3 * b + 1];
        sz += p[3 * b + 2];
    }
    out.fx[i] = sx;
    out.fy[i] = sy;
    out.fz[i] = sz;
}

// ---------------------------------------------------------------------------------------------
// Work lists and launch helpers for the sweeps.

constexpr int SWEEP_WARPS = 8;

int64_t sweep_items(int algorithm, int64_t n, int JB, int64_t *prefix, int64_t kseg)
{
    // AUTA (algorithm 2): block b = [b*JB, (b+1)*JB) needs j <= n-2 and i < j, so it has
    // min((b+1)*JB - 1, n - 2) values i = 0 ..; NATA (0): every block with j <= n-2 pairs with all n i.
    // With kseg > 0 (AUTA) each (block, i) is split into ceil((n - b*JB) / kseg) items by k range.
    int64_t nb = n >= 3 ? (n - 2 + JB) / JB : 0;  // blocks holding some j <= n - 2
    int64_t total = 0;
    if (prefix) prefix[0] = 0;
    for (int64_t b = 0; b < nb; ++b) {
        int64_t cnt = algorithm == 0 ? n : std::min<int64_t>((b + 1) * JB - 1, n - 2);
        if (cnt < 0) cnt = 0;
        if (algorithm != 0 && kseg > 0) cnt *= (n - b * JB + kseg - 1) / kseg;
        total += cnt;
        if (prefix) prefix[b + 1] = total;
    }
    return total;
}

int sweep_block_size(int, bool, bool, int) { return SWEEP_WARPS * 32; }

template <class S, int R>
static cudaError_t launch_auta_t(bool energy, int64_t n, Pos pos, Out out, double *eo, double nu, SweepWork work,
                                 int grid, cudaStream_t st)
{
    if (work.total <= 0) return cudaSuccess;
    if (energy)
        k_auta<S, R, true, SWEEP_WARPS><<<grid, SWEEP_WARPS * 32, 0, st>>>(n, pos, out, eo, nu, work);
    else
        k_auta<S, R, false, SWEEP_WARPS><<<grid, SWEEP_WARPS * 32, 0, st>>>(n, pos, out, eo, nu, work);
    return cudaGetLastError();
}

cudaError_t launch_auta(bool mixed, bool dual, int R, bool energy, int64_t n, Pos pos, Out out, double *eo, double nu,
                        SweepWork work, int grid, cudaStream_t st)
{
    if (dual) {
        if (mixed) return launch_auta_t<Dual<float>, 2>(energy, n, pos, out, eo, nu, work, grid, st);
        return launch_auta_t<Dual<double>, 1>(energy, n, pos, out, eo, nu, work, grid, st);
    }
    if (mixed) {
        switch (R) {
            case 1: return launch_auta_t<float, 1>(energy, n, pos, out, eo, nu, work, grid, st);
            case 2: return launch_auta_t<float, 2>(energy, n, pos, out, eo, nu, work, grid, st);
            default: return launch_auta_t<float, 4>(energy, n, pos, out, eo, nu, work, grid, st);
        }
    }
    switch (R) {
        case 1: return launch_auta_t<double, 1>(energy, n, pos, out, eo, nu, work, grid, st);
        case 4: return launch_auta_t<double, 4>(energy, n, pos, out, eo, nu, work, grid, st);
        default: return launch_auta_t<double, 2>(energy, n, pos, out, eo, nu, work, grid, st);
    }
}

template <class S, int R>
static cudaError_t launch_nata_t(bool energy, int64_t n, Pos pos, double *partial, double *eo, double nu,
                                 SweepWork work, int grid, cudaStream_t st)
{
    if (work.total <= 0) return cudaSuccess;
    if (energy)
        k_nata<S, R, true, SWEEP_WARPS><<<grid, SWEEP_WARPS * 32, 0, st>>>(n, pos, partial, eo, nu, work);
    else
        k_nata<S, R, false, SWEEP_WARPS><<<grid, SWEEP_WARPS * 32, 0, st>>>(n, pos, partial, eo, nu, work);
    return cudaGetLastError();
}

cudaError_t launch_nata(bool mixed, bool dual, int R, bool energy, int64_t n, Pos pos, Out, double *eo, double nu,
                        SweepWork work, double *partial, int grid, cudaStream_t st)
{
    if (dual) return cudaErrorInvalidValue;  // the adjoint of NATA uses the AUTA sweep (same triplet set)
    if (mixed) {
        switch (R) {
            case 1: return launch_nata_t<float, 1>(energy, n, pos, partial, eo, nu, work, grid, st);
            case 2: return launch_nata_t<float, 2>(energy, n, pos, partial, eo, nu, work, grid, st);
            default: return launch_nata_t<float, 4>(energy, n, pos, partial, eo, nu, work, grid, st);
        }
    }
    switch (R) {
        case 1: return launch_nata_t<double, 1>(energy, n, pos, partial, eo, nu, work, grid, st);
        case 4: return launch_nata_t<double, 4>(energy, n, pos, partial, eo, nu, work, grid, st);
        default: return launch_nata_t<double, 2>(energy, n, pos, partial, eo, nu, work, grid, st);
    }
}

cudaError_t launch_nata_reduce(bool, int64_t n, int nblocks, const double *partial, Out out, cudaStream_t st)
{
    if (n <= 0) return cudaSuccess;
    k_nata_reduce<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(n, nblocks, partial, out);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------------------------
// P3BCA cell grid.  Arithmetic without FMA contraction so that it equals the oracle's C code.

// A non-finite coordinate (a run that blew up) lands in cell 0, never outside the grid.
__device__ __forceinline__ int cell_coord(double x, double lo, double w, int nd)
{
    double t = floor(__ddiv_rn(__dsub_rn(x, lo), w));
    double m = fmod(t, (double)nd);
    if (m < 0) m = __dadd_rn(m, (double)nd);
    if (!(m >= 0.0 && m < (double)nd)) return 0;
    return (int)m;
}

// Cell coordinate as cell_coord, and whether it was reached by wrapping: the raw coordinate lies
// outside the box (or is not a number).
__device__ __forceinline__ int cell_coord_w(double x, double lo, double w, int nd, bool &outside)
{
    const double t = floor(__ddiv_rn(__dsub_rn(x, lo), w));
    outside = outside || !(t >= 0.0 && t < (double)nd);
    double m = fmod(t, (double)nd);
    if (m < 0) m = __dadd_rn(m, (double)nd);
    if (!(m >= 0.0 && m < (double)nd)) return 0;
    return (int)m;
}

// Particle::GetSqrDistPeriodic (structs.hpp:106-115), evaluated in the reference's order.
__device__ __forceinline__ double sqdist_periodic(double xa, double ya, double za, double xb, double yb, double zb,
                                                  const Grid &g)
{
    double ax = fabs(__dsub_rn(xb, xa)), ay = fabs(__dsub_rn(yb, ya)), az = fabs(__dsub_rn(zb, za));
    double mx = fmin(ax, __dsub_rn(g.L[0], ax)), my = fmin(ay, __dsub_rn(g.L[1], ay)),
           mz = fmin(az, __dsub_rn(g.L[2], az));
    return __dadd_rn(__dadd_rn(__dmul_rn(mx, mx), __dmul_rn(my, my)), __dmul_rn(mz, mz));
}

// index of the system owning item idx (sys_off has nsys + 1 entries)
__device__ __forceinline__ int system_of(const int64_t *sys_off, int nsys, int64_t idx)
{
    return nsys > 1 ? find_block(sys_off, nsys, idx) : 0;
}

__global__ void k_cell_assign(int64_t n, const double *__restrict__ x, const double *__restrict__ y,
                              const double *__restrict__ z, const __grid_constant__ Grid g, GridSet set,
                              int32_t *__restrict__ cell_of, int32_t *__restrict__ cell_rank,
                              int32_t *__restrict__ cell_count, int32_t *__restrict__ cell_out)
{
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int sys = system_of(set.sys_off, set.nsys, i);
    const Grid &G = set.nsys > 1 ? set.grids[sys] : g;
    bool out = false;
    int cx = cell_coord_w(x[i], G.lo[0], G.w[0], G.dims[0], out);
    int cy = cell_coord_w(y[i], G.lo[1], G.w[1], G.dims[1], out);
    int cz = cell_coord_w(z[i], G.lo[2], G.w[2], G.dims[2], out);
    int c = (int)(set.nsys > 1 ? set.cell_off[sys] : 0) + (cz * G.dims[1] + cy) * G.dims[0] + cx;
    c = (int)TBMD_IX(c, g.ncells, BS_CELL_OF);
    cell_of[i] = c;
    cell_rank[i] = atomicAdd(cell_count + c, 1);  // the particle's slot within its cell
    if (out) cell_out[c] = 1;
}

// Exclusive scan of cell counts: one block of 1024 threads over tiles of 8192 cells.  A tile is read
// into shared memory with coalesced loads (all issued before the first is used), each thread scans
// its 8 contiguous cells there, the thread totals are scanned with warp shuffles and across the 32
// warps, and the starts go back out with coalesced stores.  A carry links the tiles.
constexpr int SCAN_PER_THREAD = 8;

__global__ void __launch_bounds__(1024) k_cell_scan(int64_t ncells, const int32_t *__restrict__ count,
                                                    int32_t *__restrict__ start)
{
    constexpr int TILE = 1024 * SCAN_PER_THREAD;
    __shared__ __align__(16) int32_t tile[TILE];
    __shared__ int32_t wsum[32];
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    int32_t carry = 0;
    for (int64_t base = 0; base < ncells; base += TILE) {
        const int m = (int)(ncells - base < TILE ? ncells - base : TILE);
#pragma unroll
        for (int k = 0; k < SCAN_PER_THREAD; ++k) {
            const int i = k * 1024 + t;
            tile[i] = i < m ? count[base + i] : 0;
        }
        __syncthreads();
        const int4 *own = (const int4 *)(tile + t * SCAN_PER_THREAD);
        const int4 p = own[0], q = own[1];
        const int32_t v[SCAN_PER_THREAD] = {p.x, p.y, p.z, p.w, q.x, q.y, q.z, q.w};
        int32_t s = 0;
#pragma unroll
        for (int k = 0; k < SCAN_PER_THREAD; ++k) s += v[k];
        int32_t inc = s;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int32_t x = __shfl_up_sync(0xffffffffu, inc, o);
            if (lane >= o) inc += x;
        }
        if (lane == 31) wsum[warp] = inc;
        __syncthreads();
        if (warp == 0) {
            int32_t w = wsum[lane];
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int32_t x = __shfl_up_sync(0xffffffffu, w, o);
                if (lane >= o) w += x;
            }
            wsum[lane] = w;  // inclusive over warps
        }
        __syncthreads();
        int32_t run = carry + (warp > 0 ? wsum[warp - 1] : 0) + inc - s;
        int32_t ex[SCAN_PER_THREAD];
#pragma unroll
        for (int k = 0; k < SCAN_PER_THREAD; ++k) {
            ex[k] = run;
            run += v[k];
        }
        int4 *own_w = (int4 *)(tile + t * SCAN_PER_THREAD);
        own_w[0] = make_int4(ex[0], ex[1], ex[2], ex[3]);
        own_w[1] = make_int4(ex[4], ex[5], ex[6], ex[7]);
        carry += wsum[31];
        __syncthreads();
#pragma unroll
        for (int k = 0; k < SCAN_PER_THREAD; ++k) {
            const int i = k * 1024 + t;
            if (i < m) start[base + i] = tile[i];
        }
        __syncthreads();  // the tile and wsum are reused by the next tile
    }
    if (t == 0) start[ncells] = carry;
}

__global__ void k_cell_scatter(int64_t n, const int32_t *__restrict__ cell_of, const int32_t *__restrict__ start,
                               const int32_t *__restrict__ cell_rank, int32_t *__restrict__ sorted)
{
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    sorted[TBMD_IX(start[cell_of[i]] + cell_rank[i], n, BS_CELL_SLOT)] = (int32_t)i;
}

// Positions (and the adjoint direction) in sorted order, plus the FP32 hi/lo copy relative to the
// system's box corner.
__global__ void k_gather(int64_t n, const int32_t *__restrict__ sorted, Pos pos, const __grid_constant__ Grid g,
                         GridSet set, double *xs, double *ys, double *zs, float4 *qhi, float4 *qlo, double *dxs,
                         double *dys, double *dzs)
{
    int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    int32_t i = (int32_t)TBMD_IX(sorted[s], n, BS_SORTED);
    const double x = pos.x[i], y = pos.y[i], z = pos.z[i];
    xs[s] = x;
    ys[s] = y;
    zs[s] = z;
    const Grid &G = set.nsys > 1 ? set.grids[system_of(set.sys_off, set.nsys, s)] : g;
    float hx, hy, hz, lx, ly, lz;
    split<float>(x - G.lo[0], 0.0, hx, lx);
    split<float>(y - G.lo[1], 0.0, hy, ly);
    split<float>(z - G.lo[2], 0.0, hz, lz);
    qhi[s] = make_float4(hx, hy, hz, 0.f);
    qlo[s] = make_float4(lx, ly, lz, 0.f);
    if (dxs) {
        dxs[s] = pos.dx[i];
        dys[s] = pos.dy[i];
        dzs[s] = pos.dz[i];
    }
}

// Counting sort by cell.  The order inside a cell is the order of the scatter's atomics; nothing
// depends on it (counts are order-independent, forces are accumulated with atomics anyway).
cudaError_t launch_cell_build(int64_t n, Pos pos, const Grid &g, const GridSet &set, CellBufs &cb, bool with_dir,
                              cudaStream_t st, int *launches)
{
    const unsigned nb = (unsigned)((n + 255) / 256);
    cudaError_t e;
    // cell_count and cell_out are adjacent: one memset
    if ((e = cudaMemsetAsync(cb.cell_count, 0, sizeof(int32_t) * 2 * g.ncells, st)) != cudaSuccess) return e;
    k_cell_assign<<<nb, 256, 0, st>>>(n, pos.x, pos.y, pos.z, g, set, cb.cell_of, cb.cell_rank, cb.cell_count,
                                      cb.cell_out);
    k_cell_scan<<<1, 1024, 0, st>>>(g.ncells, cb.cell_count, cb.cell_start);
    k_cell_scatter<<<nb, 256, 0, st>>>(n, cb.cell_of, cb.cell_start, cb.cell_rank, cb.sorted);
    k_gather<<<nb, 256, 0, st>>>(n, cb.sorted, pos, g, set, cb.xs, cb.ys, cb.zs, cb.qhi, cb.qlo,
                                 with_dir ? cb.dxs : nullptr, with_dir ? cb.dys : nullptr, with_dir ? cb.dzs : nullptr);
    if (launches) *launches += 4;
    return cudaGetLastError();
}

// The Simulation step of one system fuses the integrator into the cell build and the unsort:
//   k_predict_assign  predictor (structs.hpp:40-55), the cell of the moved particle and its rank in
//                     the cell (the old count its atomic increment returns)
//   k_scatter_gather  slot in the counting sort (cell start + rank), and the particle's positions
//                     written to that slot
//   k_update_record   unsort (a gather of the particle's force from its sorted slot), update
//                     (structs.hpp:57-99) and the step's count record
// The arithmetic per particle is that of k_predictor / k_cell_assign / k_gather / k_update, so the
// results are identical; the step needs fewer launches and passes over memory.
__global__ void k_predict_assign(int64_t n, double *x, double *y, double *z, const double *vx, const double *vy,
                                 const double *vz, const double *ax, double dt, const __grid_constant__ Grid g,
                                 int32_t *__restrict__ cell_of, int32_t *__restrict__ cell_rank,
                                 int32_t *__restrict__ cell_count, int32_t *__restrict__ cell_out)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double h = __dmul_rn(__dmul_rn(dt, dt), 0.5);
    const double ah = __dmul_rn(ax[i], h);
    const double px = __dadd_rn(__dadd_rn(x[i], __dmul_rn(vx[i], dt)), ah);
    const double py = __dadd_rn(__dadd_rn(y[i], __dmul_rn(vy[i], dt)), ah);
    const double pz = __dadd_rn(__dadd_rn(z[i], __dmul_rn(vz[i], dt)), ah);
    x[i] = px;
    y[i] = py;
    z[i] = pz;
    bool out = false;
    const int cx = cell_coord_w(px, g.lo[0], g.w[0], g.dims[0], out);
    const int cy = cell_coord_w(py, g.lo[1], g.w[1], g.dims[1], out);
    const int cz = cell_coord_w(pz, g.lo[2], g.w[2], g.dims[2], out);
    const int c = (int)TBMD_IX((cz * g.dims[1] + cy) * g.dims[0] + cx, g.ncells, BS_CELL_OF);
    cell_of[i] = c;
    cell_rank[i] = atomicAdd(cell_count + c, 1);  // the particle's slot within its cell
    if (out) cell_out[c] = 1;
}

__global__ void k_scatter_gather(int64_t n, const int32_t *__restrict__ cell_of, const int32_t *__restrict__ start,
                                 int32_t *__restrict__ cell_rank, int32_t *__restrict__ sorted,
                                 const double *__restrict__ x, const double *__restrict__ y,
                                 const double *__restrict__ z, const __grid_constant__ Grid g, double *xs, double *ys,
                                 double *zs, float4 *qhi, float4 *qlo)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int c = cell_of[i];
    const int slot = (int)TBMD_IX(start[c] + cell_rank[i], n, BS_CELL_SLOT);
    sorted[slot] = (int32_t)i;
    cell_rank[i] = slot;  // from here on the particle's sorted slot, for the update's force gather
    const double px = x[i], py = y[i], pz = z[i];
    xs[slot] = px;
    ys[slot] = py;
    zs[slot] = pz;
    float hx, hy, hz, lx, ly, lz;
    split<float>(px - g.lo[0], 0.0, hx, lx);
    split<float>(py - g.lo[1], 0.0, hy, ly);
    split<float>(pz - g.lo[2], 0.0, hz, lz);
    qhi[slot] = make_float4(hx, hy, hz, 0.f);
    qlo[slot] = make_float4(lx, ly, lz, 0.f);
}

__global__ void k_unsort(int64_t n, const int32_t *__restrict__ sorted, const double *__restrict__ f0,
                         const double *__restrict__ f1, const double *__restrict__ f2, double *o0, double *o1,
                         double *o2);

// unsort, update (structs.hpp:57-99) and the step's triplet count record, in input order: particle i
// gathers its force from its sorted slot (recorded by k_scatter_gather), stores it in the state's
// force arrays and updates its velocity and acceleration, so every state array is read and written
// coalesced and only the three force loads are scattered
__global__ void k_update_record(int64_t n, const int32_t *__restrict__ slot_of, const double *__restrict__ f0,
                                const double *__restrict__ f1, const double *__restrict__ f2, double *vx, double *vy,
                                double *vz, double *ax, double *ay, double *az, double *fxo, double *fyo,
                                double *fzo, const double *__restrict__ m, double dt, double gx, double gy, double gz,
                                unsigned long long *cur, unsigned long long *per_step, unsigned int *step)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i == 0) {  // the step's triplet count (the triplet kernel has finished)
        const unsigned int k = *step;
        per_step[k] = *cur;
        *step = k + 1;
        *cur = 0ull;
    }
    if (i >= n) return;
    const int64_t slot = TBMD_IX(slot_of[i], n, BS_SORTED);
    const double fx = f0[slot], fy = f1[slot], fz = f2[slot];
    fxo[i] = fx;
    fyo[i] = fy;
    fzo[i] = fz;
    const double h = __dmul_rn(dt, 0.5);
    const double mi = m[i];
    const double nx = __dsub_rn(gx, __ddiv_rn(fx, mi));
    const double ny = __dsub_rn(gy, __ddiv_rn(fy, mi));
    const double nz = __dsub_rn(gz, __ddiv_rn(fz, mi));
    vx[i] = __dadd_rn(vx[i], __dmul_rn(nx, h));
    vy[i] = __dadd_rn(vy[i], __dmul_rn(ny, h));
    vz[i] = __dadd_rn(vz[i], __dmul_rn(nz, h));
    ax[i] = nx;
    ay[i] = ny;
    az[i] = nz;
}

cudaError_t launch_step_cells(int64_t n, double *const st13[13], double dt, const Grid &g, CellBufs &cb,
                              cudaStream_t st, int *launches)
{
    const unsigned nb = (unsigned)((n + 255) / 256);
    cudaError_t e;
    if ((e = cudaMemsetAsync(cb.cell_count, 0, sizeof(int32_t) * 2 * g.ncells, st)) != cudaSuccess) return e;
    k_predict_assign<<<nb, 256, 0, st>>>(n, st13[0], st13[1], st13[2], st13[3], st13[4], st13[5], st13[6], dt, g,
                                          cb.cell_of, cb.cell_rank, cb.cell_count, cb.cell_out);
    k_cell_scan<<<1, 1024, 0, st>>>(g.ncells, cb.cell_count, cb.cell_start);
    k_scatter_gather<<<nb, 256, 0, st>>>(n, cb.cell_of, cb.cell_start, cb.cell_rank, cb.sorted, st13[0], st13[1],
                                          st13[2], g, cb.xs, cb.ys, cb.zs, cb.qhi, cb.qlo);
    if (launches) *launches += 3;
    return cudaGetLastError();
}

cudaError_t launch_unsort_update(int64_t n, const CellBufs &cb, double *const st13[13], double dt, const double g3[3],
                                 unsigned long long *cur, unsigned long long *per_step, unsigned int *step,
                                 cudaStream_t st)
{
    const unsigned nb = (unsigned)((n + 255) / 256);
    k_update_record<<<nb, 256, 0, st>>>(n, cb.cell_rank, cb.fs[0], cb.fs[1], cb.fs[2], st13[3], st13[4], st13[5],
                                         st13[6], st13[7], st13[8], st13[10], st13[11], st13[12], st13[9], dt, g3[0],
                                         g3[1], g3[2], cur, per_step, step);
    return cudaGetLastError();
}

// Half neighbour lists: for sorted particle s, every t > s in the 27 (fewer on one-cell axes)
// neighbouring cells with periodic d^2 <= cutoff^2 (the reference's test, structs.hpp:106-115,
// d == cutoff inside).
//
// Block per cell c.  Particles are counting-sorted by cell id, so the candidates t > s of a
// particle s in c are: the particles of c after s, and all particles of the neighbour cells with
// id > c.  nbr_cells (built on the host with the grid) lists, per cell, its neighbour cells with
// id >= c in increasing id order (-1 padded to 27).  The block scans their sizes and stages their
// particles (FP32 hi/lo positions relative to the box corner, with the sorted index in the hi
// record's spare w) in shared memory in that order - cell by cell, so every copy is coalesced - and
// the candidates of the i-th particle of c are the suffix after i.  Warps take the particles of c in
// turn and sweep their suffix 32 candidates at a time, writing survivors compacted by ballot.  A
// cell whose candidates exceed the staging capacity reads them from global memory instead.  Lists
// longer than cap are truncated; the largest length is recorded so the host can enlarge cap and
// recompute.
//
// The test runs in FP32 on d = (hi_t - hi_s) + (lo_t - lo_s), which is within 2^-24 (|d| + L) of
// the FP64 difference per component, inside the bound e = 16 eps32 (L + cutoff) of the guard band
// (the triplet kernel's).  Outside the band around cutoff^2 the FP32 value decides; inside it the
// exact FP64 test on the FP64 positions does, so the lists are exactly the reference's.
// Positions are not wrapped into the box, so a particle that drifted out of it sits in a cell it
// reached by wrapping, with a raw offset near a multiple of L; the cell build flags such cells
// (cell_out).  A cell that is interior (at least 4 cells per axis, not on the boundary) and whose
// candidate cells carry no flag has every coordinate inside the box and every candidate within
// 2 cells <= L / 2 per axis: there the periodic form equals the raw distance and the hi parts alone
// are accurate to 2^-24 L, so the cheaper test is used.  Elsewhere min(|d|, L - |d|) on hi + lo.
constexpr int NB_THREADS = 128;
// Start value of the triplet kernel's work counters that leaves it nothing to do: above every particle
// and item index (both below 2^31), with room for one increment per warp.
constexpr unsigned int P3_NO_WORK = 0x80000000u;
constexpr size_t NB_STAGE_BYTES = 2 * sizeof(float4);  // per staged candidate (hi with the index in w, lo)

__global__ void __launch_bounds__(NB_THREADS, 10) k_neighbors(int64_t n, const __grid_constant__ Grid g, GridSet set,
                                                          const int32_t *__restrict__ nbr_cells,
                                                          const float4 *__restrict__ qhi,
                                                          const float4 *__restrict__ qlo,
                                                          const double *__restrict__ xs,
                                                          const double *__restrict__ ys,
                                                          const double *__restrict__ zs,
                                                          const int32_t *__restrict__ cell_start,
                                                          const int32_t *__restrict__ cell_out, int32_t *nbr,
                                                          int32_t *nbr_count, int32_t *max_count, int cap,
                                                          int max_stage, unsigned long long *long_items,
                                                          unsigned int long_cap, unsigned int *long_count,
                                                          unsigned int *long_max, unsigned int *work_counter)
{
    // Arm the triplet kernel's two work counters (it runs next on the stream).  After a list or
    // chunk-pair overflow in an earlier step of the same call (the flags are cleared per call and
    // only grow) the host re-runs the call with larger capacities and drops what the steps compute,
    // so the counters start past every item and the triplet kernel of this step does no work.
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        const bool over = *(volatile int32_t *)max_count > cap || *(volatile unsigned int *)long_max > long_cap;
        work_counter[0] = over ? P3_NO_WORK : 0u;
        work_counter[1] = over ? P3_NO_WORK : 0u;
    }
    extern __shared__ __align__(16) unsigned char smraw[];
    float4 *shi = (float4 *)smraw;
    float4 *slo = shi + max_stage;
    __shared__ int cstart[32], cpre[33], raw_cell;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    constexpr int NW = NB_THREADS / 32;
    int warp_max = 0;  // longest list this warp produced (one atomic per warp at the end)
    for (int64_t c = blockIdx.x; c < g.ncells; c += gridDim.x) {
        const int b0 = cell_start[c], e0 = cell_start[c + 1];
        if (b0 == e0) continue;
        const int sys = system_of(set.cell_off, set.nsys, c);
        const Grid &G = set.nsys > 1 ? set.grids[sys] : g;
        const float Lx = (float)G.L[0], Ly = (float)G.L[1], Lz = (float)G.L[2];
        const float sq_lo = (float)G.sqcut - G.band, sq_hi = (float)G.sqcut + G.band;
        if (warp == 0) {
            int nc = lane < 27 ? nbr_cells[c * 27 + lane] : -1;
            if (nc >= 0) nc = (int)TBMD_IX(nc, g.ncells, BS_NBR_CELL);
            const int cs = nc >= 0 ? cell_start[nc] : 0;
            const int len = nc >= 0 ? cell_start[nc + 1] - cs : 0;
            // raw test: an interior cell (at least 4 cells per axis, not on the boundary, so no
            // candidate cell wraps) whose candidate cells hold only particles inside the box
            const bool any_out = __any_sync(0xffffffffu, nc >= 0 && cell_out[nc] != 0);
            if (lane == 0) {
                const int64_t lc = c - (set.nsys > 1 ? set.cell_off[sys] : 0);
                const int cx = (int)(lc % G.dims[0]), cy = (int)((lc / G.dims[0]) % G.dims[1]),
                          cz = (int)(lc / ((int64_t)G.dims[0] * G.dims[1]));
                const bool interior = G.dims[0] >= 4 && G.dims[1] >= 4 && G.dims[2] >= 4 && cx > 0 && cy > 0 &&
                                      cz > 0 && cx < G.dims[0] - 1 && cy < G.dims[1] - 1 && cz < G.dims[2] - 1;
                raw_cell = interior && !any_out;
            }
            int incl = len;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int v = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= o) incl += v;
            }
            cstart[lane] = cs;
            cpre[lane] = incl - len;
            if (lane == 31) cpre[32] = incl;
        }
        __syncthreads();
        const int T = cpre[32];
        // staged: the candidates and, after them, 32 far-away sentinels, so that a warp's scan
        // needs no bounds test (a lane past T reads a sentinel, which fails the cutoff)
        const bool staged = T + 32 <= max_stage;
        // candidate q lies in table entry k: the largest k with cpre[k] <= q (empty entries have
        // cpre[k] == cpre[k + 1] and are skipped by taking the largest)
        auto entry_of = [&](int q) {
            int k = 0;
#pragma unroll
            for (int step = 16; step > 0; step >>= 1)
                if (k + step < 27 && cpre[k + step] <= q) k += step;
            return k;
        };
        // read before the barrier below: warp 0 rewrites raw_cell for its next cell once past it
        const bool raw = raw_cell != 0;
        if (staged) {
            for (int q = threadIdx.x; q < T + 32; q += NB_THREADS) {
                if (q < T) {
                    const int k = entry_of(q);
                    const int t = (int)TBMD_IX(cstart[k] + (q - cpre[k]), n, BS_CANDIDATE);
                    (void)TBMD_IX(q, max_stage, BS_STAGE);
                    float4 h = qhi[t];
                    h.w = __int_as_float(t);  // the sorted index rides in the unused w
                    shi[q] = h;
                    slo[q] = qlo[t];
                } else {
                    shi[q] = make_float4(1e18f, 1e18f, 1e18f, __int_as_float(-1));
                    slo[q] = make_float4(0.f, 0.f, 0.f, 0.f);
                }
            }
        }
        __syncthreads();
        // particle sl scans the candidates after it, so earlier particles have longer scans: the warps
        // take them in a snake order (0 1 2 3 3 2 1 0 0 1 ...) so that their totals even out before the
        // barrier at the end of the cell
        for (int it = 0; it * NW < e0 - b0; ++it) {
            const int sl = it * NW + ((it & 1) ? NW - 1 - warp : warp);
            if (sl >= e0 - b0) continue;
            const int s = b0 + sl;  // cell c comes first in the candidate order: q = sl
            const float4 oh = staged ? shi[sl] : qhi[s], ol = staged ? slo[sl] : qlo[s];
            int cnt = 0;
            int32_t *dst = nbr + (int64_t)s * cap;
            // one candidate per lane and iteration; the pass mask compacts the list in order
            auto emit = [&](bool pass, int t) {
                const unsigned m = __ballot_sync(0xffffffffu, pass);
                const int off = cnt + __popc(m & ((1u << lane) - 1u));
                if (pass && off < cap) dst[off] = t;
                cnt += __popc(m);
            };
            auto exact = [&](int t) {
                return sqdist_periodic(xs[s], ys[s], zs[s], xs[t], ys[t], zs[t], G) <= G.sqcut;
            };
            if (staged && raw) {
                // every coordinate lies in the box: the hi parts alone are within 2^-24 L, and the
                // periodic form is the raw distance (each axis under 2 cells <= L / 2).  Two
                // iterations per trip let the next candidate's loads and test overlap this one's
                // compaction (1% faster than one).
#pragma unroll 2
                for (int q0 = sl + 1; q0 < T; q0 += 32) {
                    const int q = q0 + lane;
                    const float4 h = shi[q];
                    const int t = __float_as_int(h.w);
                    const float dx = h.x - oh.x, dy = h.y - oh.y, dz = h.z - oh.z;
                    const float d2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
                    bool pass = d2 <= sq_lo;
                    if (!pass && d2 <= sq_hi) pass = exact(t);
                    emit(pass, t);
                }
            } else if (staged) {
#pragma unroll 2
                for (int q0 = sl + 1; q0 < T; q0 += 32) {
                    const int q = q0 + lane;
                    const float4 h = shi[q], l = slo[q];
                    const int t = __float_as_int(h.w);
                    const float dx = (h.x - oh.x) + (l.x - ol.x), dy = (h.y - oh.y) + (l.y - ol.y),
                                dz = (h.z - oh.z) + (l.z - ol.z);
                    const float ax = fabsf(dx), ay = fabsf(dy), az = fabsf(dz);
                    const float mx = fminf(ax, Lx - ax), my = fminf(ay, Ly - ay), mz = fminf(az, Lz - az);
                    const float d2 = fmaf(mx, mx, fmaf(my, my, mz * mz));
                    bool pass = d2 <= sq_lo;
                    if (!pass && d2 <= sq_hi) pass = exact(t);
                    emit(pass, t);
                }
            } else {
                // more candidates than the staging holds: read them from global memory
                for (int q0 = sl + 1; q0 < T; q0 += 32) {
                    const int q = q0 + lane;
                    bool pass = false;
                    int t = 0;
                    if (q < T) {
                        const int k = entry_of(q);
                        t = (int)TBMD_IX(cstart[k] + (q - cpre[k]), n, BS_CANDIDATE);
                        const float4 h = qhi[t];
                        float d2;
                        if (raw) {
                            const float dx = h.x - oh.x, dy = h.y - oh.y, dz = h.z - oh.z;
                            d2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
                        } else {
                            const float4 l = qlo[t];
                            const float dx = (h.x - oh.x) + (l.x - ol.x), dy = (h.y - oh.y) + (l.y - ol.y),
                                        dz = (h.z - oh.z) + (l.z - ol.z);
                            const float ax = fabsf(dx), ay = fabsf(dy), az = fabsf(dz);
                            const float mx = fminf(ax, Lx - ax), my = fminf(ay, Ly - ay),
                                        mz = fminf(az, Lz - az);
                            d2 = fmaf(mx, mx, fmaf(my, my, mz * mz));
                        }
                        pass = d2 <= sq_lo;
                        if (!pass && d2 <= sq_hi) pass = exact(t);
                    }
                    emit(pass, t);
                }
            }
            if (lane == 0) nbr_count[s] = cnt;
            warp_max = cnt > warp_max ? cnt : warp_max;
            // a list longer than one chunk: queue its chunk pairs (I <= J) for the triplet kernel
            const int M = cnt < cap ? cnt : cap;
            if (M > P3_CHUNK) {
                const unsigned int nch = (unsigned int)((M + P3_CHUNK - 1) / P3_CHUNK);
                const unsigned int nitems = nch * (nch + 1) / 2;
                unsigned int base = 0;
                if (lane == 0) {
                    base = atomicAdd(long_count, nitems);
                    atomicMax(long_max, base + nitems);
                }
                base = __shfl_sync(0xffffffffu, base, 0);
                for (unsigned int k = lane; k < nitems; k += 32) {
                    unsigned int I = 0, r = k;
                    while (r >= nch - I) {
                        r -= nch - I;
                        ++I;
                    }
                    if (base + k < long_cap)
                        long_items[base + k] = ((unsigned long long)(unsigned int)s << 32) | (I << 16) | (I + r);
                }
            }
        }
        __syncthreads();
    }
    if (lane == 0 && warp_max > 0) atomicMax(max_count, warp_max);
}

// Staging capacity: 1.6 times the expected candidate count (14 of the 27 cells have id >= c on
// average), at least 256, at most 4096 (144 KiB).
int neighbor_stage_cap(const Grid &g, int64_t n)
{
    const double mean = (double)n / (double)g.ncells;
    const int cells = (g.dims[0] == 1 ? 1 : 3) * (g.dims[1] == 1 ? 1 : 3) * (g.dims[2] == 1 ? 1 : 3);
    int want = (int)(1.6 * mean * (cells / 2 + 1)) + 128;
    want = (want + 31) / 32 * 32;
    return want < 256 ? 256 : (want > 4096 ? 4096 : want);
}

// Per cell of grid g (cells numbered from cell0), its neighbour cells with id >= its own id in
// increasing order, -1 padded to 27 entries.
void neighbor_cell_table(const Grid &g, int64_t cell0, int32_t *out)
{
    const int ox = g.dims[0] == 1 ? 0 : 1, oy = g.dims[1] == 1 ? 0 : 1, oz = g.dims[2] == 1 ? 0 : 1;
    for (int64_t lc = 0; lc < g.ncells; ++lc) {
        const int cx = (int)(lc % g.dims[0]), cy = (int)((lc / g.dims[0]) % g.dims[1]),
                  cz = (int)(lc / ((int64_t)g.dims[0] * g.dims[1]));
        int32_t ids[27];
        int K = 0;
        for (int dz = -oz; dz <= oz; ++dz)
            for (int dy = -oy; dy <= oy; ++dy)
                for (int dx = -ox; dx <= ox; ++dx) {
                    const int nx = (cx + dx + g.dims[0]) % g.dims[0];
                    const int ny = (cy + dy + g.dims[1]) % g.dims[1];
                    const int nz = (cz + dz + g.dims[2]) % g.dims[2];
                    const int64_t nc = (int64_t)(nz * g.dims[1] + ny) * g.dims[0] + nx;
                    if (nc < lc) continue;
                    int q = K++;
                    while (q > 0 && ids[q - 1] > nc + cell0) {
                        ids[q] = ids[q - 1];
                        --q;
                    }
                    ids[q] = (int32_t)(nc + cell0);
                }
        int32_t *row = out + (cell0 + lc) * 27;
        for (int k = 0; k < 27; ++k) row[k] = k < K ? ids[k] : -1;
    }
}

cudaError_t launch_neighbors(int64_t n, const Grid &g, const GridSet &set, const int32_t *nbr_cells, int max_stage,
                             CellBufs &cb, cudaStream_t st)
{
    const size_t smem = (size_t)max_stage * NB_STAGE_BYTES;
    int64_t blocks = g.ncells < 65535 * 16 ? g.ncells : 65535 * 16;
    cudaError_t e = cudaMemsetAsync(cb.long_count, 0, sizeof(unsigned int), st);
    if (e != cudaSuccess) return e;
    k_neighbors<<<(unsigned)blocks, NB_THREADS, smem, st>>>(n, g, set, nbr_cells, cb.qhi, cb.qlo, cb.xs, cb.ys, cb.zs,
                                                            cb.cell_start, cb.cell_out, cb.nbr, cb.nbr_count,
                                                            cb.max_count, cb.cap,
                                                            max_stage, cb.long_items, (unsigned int)cb.long_cap,
                                                            cb.long_count, cb.long_max, cb.work_counter);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------------------------
// P3BCA triplets.  A warp takes work items from two dynamic counters.  An item is a particle s
// whose half list has at most P3_CHUNK (64) entries, or, for a longer list, a pair of its chunks
// (I <= J) queued by the neighbour kernel; long lists are thus spread over many warps and the
// shared memory of a warp is fixed (two chunks) whatever the list length.  The item's entries are
// staged as slots in the warp's shared memory: edge from s (hi, its square, and the lo part for the
// mixed form), an S gradient accumulator per slot and the neighbour index.
//
// Every unordered slot pair of the item (all pairs of one chunk, or all pairs across two chunks)
// is visited once, block by block (blocks of 32 slots).  For own block A
// lane x owns slot A+x: its edge and its gradient accumulator live in registers.
//   - pairs inside A: circular diagonals, pair (x, (x + d) mod m_A), d = 1 .. m_A/2 (on the half
//     diagonal of an even m_A only x < m_A/2);
//   - pairs A x B with a later block B: a full B by a rotation, pair (x, (x + t) & 31),
//     t = 0..31.  A short B: lanes in groups of m_B, lane j of each group meets (j + t) mod m_B at
//     step t = 0..m_B-1; groups after the first add their partner shares to per-warp copies, summed
//     into B's slots at the end.
// In every warp step the partner slots (and copies) are distinct, so partner gradients are added with
// a plain shared-memory read-modify-write (one __syncwarp per step, no atomics).  The own-slot
// gradient stays in registers.  At the end of an item each slot is flushed with one FP64 atomic.
//
// Cutoff test of the third edge: the reference's periodic formula (structs.hpp:106-115) on the third
// edge the triplet math uses (FP32 in the mixed form, FP64 in the FP64 forms), or, when no list
// entry of s wraps around the box and the box is at least 4 cutoffs wide, the raw squared distance,
// which the formula then equals.  Outside a guard band around cutoff^2 that bounds the difference
// to the reference's own FP64 value the computed distance decides; inside it the reference's exact
// test on the two neighbours' FP64 positions.  Counts are therefore exact in both forms.

template <class S>
struct alignas(4 * sizeof(S)) Slot4 {
    S x, y, z, w;
};

// Gradient accumulator of a slot: three components, padded to a power of two for float and double
// so that the per-step update is whole vector loads and stores (the dual forms stay unpadded).
template <class S>
struct Grad {
    S x, y, z;
};
template <>
struct alignas(16) Grad<float> {
    float x, y, z, w;
};
// FP64: padded to 32 bytes as well, so that a slot's read-modify-write is two 16-byte accesses
// that do not straddle banks of the neighbouring slots (24-byte slots gave 24 M bank conflicts per
// C3 launch)
template <>
struct alignas(32) Grad<double> {
    double x, y, z, w;
};
template <class S>
__device__ __forceinline__ Grad<S> grad_zero()
{
    Grad<S> g;
    g.x = szero<S>();
    g.y = szero<S>();
    g.z = szero<S>();
    return g;
}
template <>
__device__ __forceinline__ Grad<float> grad_zero<float>()
{
    return Grad<float>{0.f, 0.f, 0.f, 0.f};
}
template <>
__device__ __forceinline__ Grad<double> grad_zero<double>()
{
    return Grad<double>{0.0, 0.0, 0.0, 0.0};
}
// dst += src, component-wise (the mixed form's accumulators, whose w is the factored scalar)
template <class S>
__device__ __forceinline__ void grad_merge(Grad<S> &dst, const Grad<S> &src)
{
    dst.x += src.x;
    dst.y += src.y;
    dst.z += src.z;
    dst.w += src.w;
}
template <class S>
__device__ __forceinline__ Grad<S> grad_shfl_down(const Grad<S> &v, int off)
{
    return Grad<S>{__shfl_down_sync(0xffffffffu, v.x, off), __shfl_down_sync(0xffffffffu, v.y, off),
                   __shfl_down_sync(0xffffffffu, v.z, off), __shfl_down_sync(0xffffffffu, v.w, off)};
}
template <>
__device__ __forceinline__ Grad<double> grad_shfl_down<double>(const Grad<double> &v, int off)
{
    // w is padding in the FP64 accumulators
    return Grad<double>{__shfl_down_sync(0xffffffffu, v.x, off), __shfl_down_sync(0xffffffffu, v.y, off),
                        __shfl_down_sync(0xffffffffu, v.z, off), 0.0};
}
// the dual forms' accumulators: three dual components
template <class T>
__device__ __forceinline__ void grad_merge(Grad<Dual<T>> &dst, const Grad<Dual<T>> &src)
{
    dst.x = dst.x + src.x;
    dst.y = dst.y + src.y;
    dst.z = dst.z + src.z;
}
template <class T>
__device__ __forceinline__ Dual<T> shfl_down_s(Dual<T> v, int off)
{
    return {__shfl_down_sync(0xffffffffu, v.v, off), __shfl_down_sync(0xffffffffu, v.d, off)};
}
template <class T>
__device__ __forceinline__ Grad<Dual<T>> grad_shfl_down(const Grad<Dual<T>> &v, int off)
{
    return Grad<Dual<T>>{shfl_down_s(v.x, off), shfl_down_s(v.y, off), shfl_down_s(v.z, off)};
}
template <class S>
__device__ __forceinline__ void slot_add(Grad<S> &slot, V3<S> g)
{
    Grad<S> v = slot;
    v.x = v.x + g.x;
    v.y = v.y + g.y;
    v.z = v.z + g.z;
    slot = v;
}

// Factored accumulation.  A slot's edge e (hi part) is fixed during an item, so every gradient it
// receives is (scalar) * e + (vector): as the own slot of a lane it gets alpha u + gamma w (e = u),
// as a partner beta v - gamma w (e = v), w the pair's third edge.  The mixed form keeps the scalar
// in the slot's spare fourth float and the vector in x, y, z, and forms scalar * e + vector once,
// at the flush: 4 instead of 9 FP32 operations per triplet and side.  The other forms accumulate
// the gradient itself.
template <class S>
struct PGrad {  // a partner's share of one triplet
    V3<S> g;
};
template <>
struct PGrad<float> {
    float beta, ngamma;  // beta and -gamma
    V3<float> w;
};
template <class S>
__device__ __forceinline__ PGrad<S> make_pgrad(const ATCoef<S> &cf, V3<S> v, V3<S> w)
{
    return PGrad<S>{fma3(v, cf.beta, w * (-cf.gamma))};
}
template <>
__device__ __forceinline__ PGrad<float> make_pgrad<float>(const ATCoef<float> &cf, V3<float>, V3<float> w)
{
    return PGrad<float>{cf.beta, -cf.gamma, w};
}
template <class S>
__device__ __forceinline__ void pgrad_add(Grad<S> &slot, const PGrad<S> &pg)
{
    slot_add(slot, pg.g);
}
template <>
__device__ __forceinline__ void pgrad_add<float>(Grad<float> &slot, const PGrad<float> &pg)
{
    Grad<float> v = slot;
    v.x = fmaf(pg.ngamma, pg.w.x, v.x);
    v.y = fmaf(pg.ngamma, pg.w.y, v.y);
    v.z = fmaf(pg.ngamma, pg.w.z, v.z);
    v.w = v.w + pg.beta;
    slot = v;
}
// own-slot accumulator of a lane
template <class S>
struct OwnAcc {
    V3<S> g;
    __device__ __forceinline__ void zero() { g = vzero<S>(); }
    __device__ __forceinline__ void add(const ATCoef<S> &cf, V3<S> u, V3<S> w) { g = g + fma3(u, cf.alpha, w * cf.gamma); }
    __device__ __forceinline__ void merge(Grad<S> &slot) const { slot_add(slot, g); }
};
template <>
struct OwnAcc<float> {
    V3<float> g;
    float alpha;
    __device__ __forceinline__ void zero()
    {
        g = {0.f, 0.f, 0.f};
        alpha = 0.f;
    }
    __device__ __forceinline__ void add(const ATCoef<float> &cf, V3<float>, V3<float> w)
    {
        alpha += cf.alpha;
        g = fma3(w, cf.gamma, g);
    }
    __device__ __forceinline__ void merge(Grad<float> &slot) const
    {
        Grad<float> v = slot;
        v.x += g.x;
        v.y += g.y;
        v.z += g.z;
        v.w += alpha;
        slot = v;
    }
};
// slot gradient at the flush, widened to the accumulator type (e = the slot's edge, hi part)
template <class S, class A>
__device__ __forceinline__ V3<A> slot_gradient(const Grad<S> &g, const Slot4<S> &)
{
    return widen(V3<S>{g.x, g.y, g.z});
}
template <>
__device__ __forceinline__ V3<double> slot_gradient<float, double>(const Grad<float> &g, const Slot4<float> &e)
{
    const double w = (double)g.w;
    return V3<double>{fma(w, (double)e.x, (double)g.x), fma(w, (double)e.y, (double)g.y),
                      fma(w, (double)e.z, (double)g.z)};
}

// Partner accumulators of the lane groups g >= 1 of a short block B (see the item loops): (g - 1) m_B + y
// < 32 entries.
constexpr int P3_COPIES = 32;

// The mixed forces kernel keeps a slot's neighbour index in the unused w of its lo-edge record (the
// bits of an int32 in a float), so that the P3_COPIES accumulators of the group form of short blocks
// take no more shared memory than the index array did (26.6 KB per CTA of 4 warps).  The FP64 and
// dual forms, whose occupancy their registers bound, keep their index array and add the copies.
template <class S>
struct IdxInLo {
    static constexpr bool value = false;
};
template <>
struct IdxInLo<float> {
    static constexpr bool value = true;
};
template <class S>
struct SlotLayout {
    // per-warp shared memory, [2 * P3_CHUNK] of each: edge hi + b (Slot4), edge lo (Slot4, mixed only),
    // gradient accumulator (Grad), neighbour index (unless IdxInLo); then P3_COPIES gradient
    // accumulators
    static constexpr bool mixed = HasLo<S>::value;
    static constexpr int nlo = mixed ? 1 : 0;
    static constexpr size_t bytes_per_slot =
        (1 + nlo) * sizeof(Slot4<S>) + sizeof(Grad<S>) + (IdxInLo<S>::value ? 0 : sizeof(int32_t));
    static constexpr size_t bytes_per_warp =
        2 * P3_CHUNK * bytes_per_slot + P3_COPIES * sizeof(Grad<S>);
};


template <class S>
struct P3Warp {
    Slot4<S> *sd;  // hi edge + b
    Slot4<S> *sl;  // lo edge (mixed)
    Grad<S> *gr;   // gradient accumulators
    int32_t *idx;  // neighbour indices (unless IdxInLo)
    Grad<S> *cp;   // [P3_COPIES] partner accumulators of lane groups >= 1
    __device__ __forceinline__ int32_t index(int i) const
    {
        if constexpr (IdxInLo<S>::value)
            return __float_as_int(sl[i].w);
        else
            return idx[i];
    }
    // stage slot i's lo edge and neighbour index
    __device__ __forceinline__ void set_lo_index(int i, const V3<S> &l, int32_t t) const
    {
        if constexpr (IdxInLo<S>::value) {
            sl[i] = Slot4<S>{l.x, l.y, l.z, __int_as_float(t)};
        } else {
            idx[i] = t;
            if constexpr (HasLo<S>::value) sl[i] = Slot4<S>{l.x, l.y, l.z, szero<S>()};
        }
    }
    __device__ __forceinline__ Slot4<S> slot(int i) const { return sd[i]; }
    __device__ __forceinline__ void set_slot(int i, const Slot4<S> &v) const { sd[i] = v; }
    __device__ __forceinline__ Grad<S> grad(int i) const { return gr[i]; }
    __device__ __forceinline__ void set_grad(int i, const Grad<S> &v) const { gr[i] = v; }
    __device__ __forceinline__ Grad<S> copy(int i) const { return cp[i]; }
    __device__ __forceinline__ void set_copy(int i, const Grad<S> &v) const { cp[i] = v; }
};
// FP64: the 32-byte slot and accumulator records are stored as two arrays of 16-byte halves, (x, y)
// for all slots and then (z, w), so that the 16-byte accesses of a warp to consecutive slots are free
// of bank conflicts (32-byte records read as two halves conflict two ways: 73 M of 160 M shared
// wavefronts of a C3 launch).
template <>
struct P3Warp<double> {
    static constexpr int SL = 2 * P3_CHUNK;
    Slot4<double> *sd;  // [SL] (x, y), then [SL] (z, w), as double2
    Slot4<double> *sl;  // unused
    Grad<double> *gr;   // [SL] (x, y), then [SL] (z, w), as double2
    int32_t *idx;
    Grad<double> *cp;   // [P3_COPIES] (x, y), then [P3_COPIES] (z, w), as double2
    __device__ __forceinline__ int32_t index(int i) const { return idx[i]; }
    __device__ __forceinline__ Grad<double> copy(int i) const
    {
        const double2 a = ((const double2 *)cp)[i], b = ((const double2 *)cp)[P3_COPIES + i];
        return Grad<double>{a.x, a.y, b.x, b.y};
    }
    __device__ __forceinline__ void set_copy(int i, const Grad<double> &v) const
    {
        ((double2 *)cp)[i] = make_double2(v.x, v.y);
        ((double2 *)cp)[P3_COPIES + i] = make_double2(v.z, v.w);
    }
    __device__ __forceinline__ void set_lo_index(int i, const V3<double> &, int32_t t) const { idx[i] = t; }
    __device__ __forceinline__ Slot4<double> slot(int i) const
    {
        const double2 a = ((const double2 *)sd)[i], b = ((const double2 *)sd)[SL + i];
        return Slot4<double>{a.x, a.y, b.x, b.y};
    }
    __device__ __forceinline__ void set_slot(int i, const Slot4<double> &v) const
    {
        ((double2 *)sd)[i] = make_double2(v.x, v.y);
        ((double2 *)sd)[SL + i] = make_double2(v.z, v.w);
    }
    __device__ __forceinline__ Grad<double> grad(int i) const
    {
        const double2 a = ((const double2 *)gr)[i], b = ((const double2 *)gr)[SL + i];
        return Grad<double>{a.x, a.y, b.x, b.y};
    }
    __device__ __forceinline__ void set_grad(int i, const Grad<double> &v) const
    {
        ((double2 *)gr)[i] = make_double2(v.x, v.y);
        ((double2 *)gr)[SL + i] = make_double2(v.z, v.w);
    }
};
// read-modify-write of slot i's accumulator (or of copy i) with a partner share
template <class S>
__device__ __forceinline__ void pgrad_add_at(const P3Warp<S> &W, int i, const PGrad<S> &pg)
{
    Grad<S> g = W.grad(i);
    pgrad_add(g, pg);
    W.set_grad(i, g);
}
template <class S>
__device__ __forceinline__ void pgrad_add_copy(const P3Warp<S> &W, int i, const PGrad<S> &pg)
{
    Grad<S> g = W.copy(i);
    pgrad_add(g, pg);
    W.set_copy(i, g);
}

// Third-edge cutoff decision for slots a (own) and b (partner) with third edge w (cww = w.w).
// sq_lo / sq_hi: the FP32 thresholds (cutoff^2 minus / plus the band of the item's test form),
// hoisted out of the pair loop by the caller (FP32 geometry: the mixed forces and the mixed
// adjoint).  Outside the band the computed edge decides; inside it the reference's own test on the
// FP64 positions of the two neighbours.
template <class S>
__device__ __forceinline__ bool cut_inside(const P3Warp<S> &W, const CellBufs &cb, const Grid &g, int a, int b,
                                           V3<S> w, S cww, bool rawok, float sq_lo, float sq_hi, float Lx, float Ly,
                                           float Lz)
{
    // g is the system's grid (L and cutoff of the exact test)
    if (std::is_same<typename Traits<S>::T, float>::value) {
        float d2;
        if (rawok) {
            d2 = to_float(cww);
        } else {
            const float ax = fabsf(to_float(w.x)), ay = fabsf(to_float(w.y)), az = fabsf(to_float(w.z));
            const float mx = fminf(ax, Lx - ax), my = fminf(ay, Ly - ay), mz = fminf(az, Lz - az);
            d2 = fmaf(mx, mx, fmaf(my, my, mz * mz));
        }
        if (d2 <= sq_lo) return true;
        if (d2 > sq_hi) return false;
        const int32_t ta = W.index(a), tb = W.index(b);
        return sqdist_periodic(cb.xs[ta], cb.ys[ta], cb.zs[ta], cb.xs[tb], cb.ys[tb], cb.zs[tb], g) <= g.sqcut;
    }
    // FP64 forms: the same guarded test in FP64 on the FP64 third edge, with the FP64 band
    double d2;
    if (rawok) {
        d2 = to_double(cww);
    } else {
        const double ax = fabs(to_double(w.x)), ay = fabs(to_double(w.y)), az = fabs(to_double(w.z));
        const double mx = fmin(ax, g.L[0] - ax), my = fmin(ay, g.L[1] - ay), mz = fmin(az, g.L[2] - az);
        d2 = mx * mx + my * my + mz * mz;
    }
    if (d2 <= g.sqcut - g.band64) return true;
    if (d2 > g.sqcut + g.band64) return false;
    const int32_t ta = W.index(a), tb = W.index(b);
    return sqdist_periodic(cb.xs[ta], cb.ys[ta], cb.zs[ta], cb.xs[tb], cb.ys[tb], cb.zs[tb], g) <= g.sqcut;
}

// Register cap of the triplet kernel per form.  The mixed forces kernel runs at 72 registers (28
// resident warps per SM at 4 warps per block): with the short-block lane groups, 72 took C3 from 0.444
// to 0.430 ms and C4 from 30.1 to 28.2 ms against 64 (32 warps), and 80 gave 0.437 ms.  The others
// keep about what they need unconstrained.
template <class S, bool ENERGY>
struct P3MaxReg {
    static constexpr int value = 128;
};
template <>
struct P3MaxReg<float, false> {
    static constexpr int value = 72;
};
template <>
struct P3MaxReg<float, true> {
    static constexpr int value = 72;
};
template <bool E>
struct P3MaxReg<double, E> {  // 96 with the group form (0.701 ms at C3; 88 spills 96 B, 104 is 0.733 ms)
    static constexpr int value = 96;
};
template <bool E>
struct P3MaxReg<Dual<float>, E> {
    static constexpr int value = E ? 96 : 80;
};
template <bool E>
struct P3MaxReg<Dual<double>, E> {
    static constexpr int value = E ? 168 : 128;
};

template <class S, bool ENERGY>
__global__ void __maxnreg__((P3MaxReg<S, ENERGY>::value))
    k_p3bca(int64_t n, const __grid_constant__ Grid g, GridSet set, CellBufs cb, double nu_d, double *energy_out,
            unsigned long long *count_out)
{
    using Acc = typename Traits<S>::Acc;
    using L = SlotLayout<S>;
    constexpr int SL = 2 * P3_CHUNK;  // staged slots per warp: one or two chunks of a half list
    extern __shared__ __align__(16) unsigned char smem[];
    const int cap = cb.cap;
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    unsigned char *base = smem + (size_t)wib * L::bytes_per_warp;
    P3Warp<S> W;
    W.sd = (Slot4<S> *)base;
    W.sl = W.sd + SL;
    W.gr = (Grad<S> *)(W.sl + (L::nlo ? SL : 0));
    W.idx = IdxInLo<S>::value ? nullptr : (int32_t *)(W.gr + SL);
    W.cp = IdxInLo<S>::value ? W.gr + SL : (Grad<S> *)(W.idx + SL);
    W.set_copy(lane, grad_zero<S>());
    __syncwarp();

    const S nu = constant<S>(nu_d), nu3 = constant<S>(-3.0 * nu_d), nu15 = constant<S>(15.0 * nu_d);
    const Out outs = {cb.fs[0], cb.fs[1], cb.fs[2], cb.hs[0], cb.hs[1], cb.hs[2]};
    const bool dual = Traits<S>::dual;
    const double cwrap = sqrt(g.sqcut) * 1.0000001;
    unsigned int cnt = 0;
    Acc en_acc = to_acc(szero<S>());
    int cur_sys = 0;
    // per-system count and energy, flushed when this warp moves on to another system
    auto flush = [&](int sys) {
        unsigned long long c64 = warp_sum_u64((unsigned long long)cnt);
        if (lane == 0 && count_out && c64) atomicAdd(count_out + sys, c64);
        cnt = 0;
        if (ENERGY) {
            Acc e = warp_sum(en_acc);
            if (lane == 0) atomicAdd(energy_out + sys, acc_value(e));
            en_acc = to_acc(szero<S>());
        }
    };

    // One work item of particle s: list entries [offI, offI + mI) staged as slots [0, mI) and, for
    // a pair of chunks, entries [offJ, offJ + mJ) as slots [mI, mI + mJ).  mJ == 0: every slot pair
    // inside [0, mI); mJ > 0: every pair (a in [0, mI), b in [mI, mI + mJ)).  The item's gradients
    // go out with one FP64 atomic per slot; s's share is minus their sum (translation invariance,
    // per triplet, so per item).
    auto item = [&](int s, int offI, int mI, int offJ, int mJ) {
        const int sys = system_of(set.sys_off, set.nsys, s);
        if (sys != cur_sys) {
            flush(cur_sys);
            cur_sys = sys;
        }
        const Grid &G = set.nsys > 1 ? set.grids[sys] : g;
        const float Lx = (float)G.L[0], Ly = (float)G.L[1], Lz = (float)G.L[2];
        const int Ms = mI + mJ;
        const double xi = cb.xs[s], yi = cb.ys[s], zi = cb.zs[s];
        const double dxi = dual ? cb.dxs[s] : 0.0, dyi = dual ? cb.dys[s] : 0.0, dzi = dual ? cb.dzs[s] : 0.0;
        bool nowrap = true;
        for (int e = lane; e < Ms; e += 32) {
            const int pos_in_list = e < mI ? offI + e : offJ + (e - mI);
            const int32_t t = (int32_t)TBMD_IX(cb.nbr[(int64_t)s * cap + pos_in_list], n, BS_LIST);
            const double x = cb.xs[t], y = cb.ys[t], z = cb.zs[t];
            const double ddx = x - xi, ddy = y - yi, ddz = z - zi;
            nowrap = nowrap && fabs(ddx) <= cwrap && fabs(ddy) <= cwrap && fabs(ddz) <= cwrap;
            V3<S> v, l;
            split<S>(ddx, dual ? cb.dxs[t] - dxi : 0.0, v.x, l.x);
            split<S>(ddy, dual ? cb.dys[t] - dyi : 0.0, v.y, l.y);
            split<S>(ddz, dual ? cb.dzs[t] - dzi : 0.0, v.z, l.z);
            W.set_slot(e, Slot4<S>{v.x, v.y, v.z, dot3(v, v)});
            W.set_lo_index(e, l, t);
            W.set_grad(e, grad_zero<S>());
        }
        const bool rawok = G.raw_ok && __all_sync(0xffffffffu, nowrap);
        // FP32 thresholds: the narrow band of hi + lo edges that do not wrap (mixed forces), else
        // the band of FP32 geometry with wrapping (the mixed adjoint always keeps this wide band)
        const bool narrow = rawok && std::is_same<S, float>::value;
        const float sq_lo = narrow ? G.raw_lo : (float)G.sqcut - G.band;
        const float sq_hi = narrow ? G.raw_hi : (float)G.sqcut + G.band;
        __syncwarp();
        S en = szero<S>();
        const unsigned int cnt0 = cnt;
        using T = typename Traits<S>::T;
        const float f_mid = (float)G.sqcut;
        // held in registers: G may live in global memory (batched systems), and the pair loops
        // store to shared memory, so a field read inside them would be read again every step
        const double d_mid = G.sqcut, d_lo = G.sqcut - G.band64, d_hi = G.sqcut + G.band64;
        // The pair loops.  FAST (items that do not wrap): one compare with cutoff^2 decides every
        // third edge, and `amb` records whether one fell inside the guard band, where the compare
        // may differ from the reference's test.  Outside the band both decide alike, so an item
        // without such an edge has exactly the results of the exact form.
        auto sweep = [&](auto fast_tag) -> bool {
            constexpr bool FAST = decltype(fast_tag)::value;
            bool amb = false;
            for (int A0 = 0; A0 < mI; A0 += 32) {
                const int mA = min(32, mI - A0);
                const bool own = lane < mA;
                const int a = A0 + (own ? lane : 0);
                const Slot4<S> od = W.slot(a);
                const V3<S> u = {od.x, od.y, od.z};
                V3<S> ul = vzero<S>();
                if (L::nlo) {
                    const Slot4<S> ol = W.sl[a];
                    ul = {ol.x, ol.y, ol.z};
                }
                const S aa = od.w;
                OwnAcc<S> acc;
                acc.zero();

                // evaluate own slot a against partner slot b; returns the partner's share
                auto pair = [&](bool act, int b) -> PGrad<S> {
                    const Slot4<S> pd = W.slot(b);
                    const V3<S> v = {pd.x, pd.y, pd.z};
                    V3<S> vl = vzero<S>();
                    if (L::nlo) {
                        const Slot4<S> pl = W.sl[b];
                        vl = {pl.x, pl.y, pl.z};
                    }
                    const V3<S> wv = third_edge(u, ul, v, vl);
                    const S cww = dot3(wv, wv);
                    bool inside = false;
                    if constexpr (FAST) {
                        if constexpr (std::is_same<T, float>::value) {
                            const float d2 = to_float(cww);
                            inside = act && d2 <= f_mid;
                            amb = amb || (act && d2 > sq_lo && d2 <= sq_hi);
                        } else {
                            const double d2 = to_double(cww);
                            inside = act && d2 <= d_mid;
                            amb = amb || (act && d2 > d_lo && d2 <= d_hi);
                        }
                    } else {
                        if (act) inside = cut_inside(W, cb, G, a, b, wv, cww, rawok, sq_lo, sq_hi, Lx, Ly, Lz);
                    }
                    cnt += inside ? 1u : 0u;
                    const ATCoef<S> cf =
                        at_coef<ENERGY>(aa, pd.w, cww, dot_uv(u, ul, v, vl, wv), dot3(u, wv), dot3(v, wv), nu, nu3, nu15, inside, en);
                    acc.add(cf, u, wv);
                    return make_pgrad(cf, v, wv);
                };

                if (mJ == 0) {
                    // pairs inside block A: circular diagonals; y = (lane + d) mod mA advances by one per
                    // diagonal (lanes past the block cycle through valid slots and are masked)
                    int y = own ? lane : 0;
                    for (int d = 1; 2 * d <= mA; ++d) {
                        y = y + 1 == mA ? 0 : y + 1;
                        const bool act = own && (2 * d < mA || lane < d);
                        const int b = A0 + y;
                        const PGrad<S> gb = pair(act, b);
                        if (act) pgrad_add_at(W, b, gb);
                        __syncwarp();
                    }
                }
                // pairs A x B with every later block B (of the same chunk, or of the second chunk)
                for (int B0 = (mJ == 0 ? A0 + 32 : mI); B0 < Ms; B0 += 32) {
                    const int mB = min(32, Ms - B0);
                    // a full block: 32 steps of distinct partners; a short block: mB steps in lane
                    // groups
                    if (mB == 32) {
                        for (int t = 0; t < 32; ++t) {
                            const int y = (lane + t) & 31;
                            const bool act = own && y < mB;
                            const int b = B0 + (y < mB ? y : 0);
                            const PGrad<S> gb = pair(act, b);
                            if (act) pgrad_add_at(W, b, gb);
                            __syncwarp();
                        }
                    } else {
                        // a short block: lanes form groups of mB, and lane j of group g meets partner
                        // (j + t) mod mB at step t, so the partners of one group are distinct.  Group 0
                        // adds to B's slots and group g >= 1 to copy (g - 1) mB + y.  Then lane l takes
                        // copy l (partner l mod mB), and the copies of a partner sum down the lanes
                        // l, l + mB, l + 2 mB, ... into lane l < mB.
                        const int g = lane / mB, j = lane - g * mB;
                        int y = j;
                        for (int t = 0; t < mB; ++t) {
                            const int b = B0 + y;
                            const PGrad<S> gb = pair(own, b);
                            if (own) {
                                if (g == 0)
                                    pgrad_add_at(W, b, gb);
                                else
                                    pgrad_add_copy(W, (int)TBMD_IX((g - 1) * mB + y, P3_COPIES, BS_SLOT), gb);
                            }
                            __syncwarp();
                            y = y + 1 == mB ? 0 : y + 1;
                        }
                        Grad<S> c = W.copy(lane);
                        W.set_copy(lane, grad_zero<S>());
                        for (int off = mB; off < 32; off *= 2) {
                            const Grad<S> o = grad_shfl_down(c, off);
                            if (lane + off < 32) grad_merge(c, o);
                        }
                        if (lane < mB) {
                            Grad<S> gl = W.grad(B0 + lane);
                            grad_merge(gl, c);
                            W.set_grad(B0 + lane, gl);
                        }
                        __syncwarp();
                    }
                }
                // merge the own accumulator into its slot
                if (own) {
                    Grad<S> ga = W.grad(a);
                    acc.merge(ga);
                    W.set_grad(a, ga);
                }
                __syncwarp();
            }
            return amb;
        };
        bool exact_form = !rawok;
        if (rawok && __any_sync(0xffffffffu, sweep(std::true_type{}))) {
            // a third edge inside the guard band: drop the item's partial sums and run it again
            // with the exact test
            cnt = cnt0;
            en = szero<S>();
            for (int e = lane; e < Ms; e += 32) W.set_grad(e, grad_zero<S>());
            __syncwarp();
            exact_form = true;
        }
        if (exact_form) sweep(std::false_type{});

        // flush the slots; s's gradient is minus the sum of all slot gradients
        V3<Acc> gia = widen(vzero<S>());
        for (int e = lane; e < Ms; e += 32) {
            const V3<Acc> ge = slot_gradient<S, Acc>(W.grad(e), W.slot(e));
            atomic_out(outs, W.index(e), ge);
            gia = gia + ge;
        }
        gia = warp_sum3(gia);
        if (lane == 0) atomic_out(outs, s, V3<Acc>{-gia.x, -gia.y, -gia.z});
        if (ENERGY) en_acc = en_acc + to_acc(en);
        __syncwarp();
    };

    if constexpr (!std::is_same<S, float>::value) {
        // Both kinds of item through one call site.  The dual forms need it to get the item body
        // inlined (two call sites left it out of line, with a stack frame of 620-710 bytes); the FP64
        // forces kernel gains 0.8% at C3 and C4 from it, and the mixed forces kernel loses 3.5%, so it
        // keeps the two loops below.
        for (int kind = 0; kind < 2; ++kind) {
            const unsigned int lim = kind == 0 ? (unsigned int)n : min(*cb.long_count, (unsigned int)cb.long_cap);
            unsigned int w = 0;
            if (lane == 0) w = atomicAdd(cb.work_counter + kind, 1u);
            w = __shfl_sync(0xffffffffu, w, 0);
            while (w < lim) {
                unsigned int wn = 0;
                if (lane == 0) wn = atomicAdd(cb.work_counter + kind, 1u);
                int s, offI = 0, mI, offJ = 0, mJ = 0;
                if (kind == 0) {
                    s = (int)w;
                    mI = min(cb.nbr_count[s], cap);
                    if (mI > P3_CHUNK) mI = 0;  // a long list: its chunk pairs come as items of kind 1
                } else {
                    const unsigned long long it = cb.long_items[w];
                    s = (int)TBMD_IX((int64_t)(it >> 32), n, BS_LONG_ITEM);
                    const int I = (int)((it >> 16) & 0xffffu), J = (int)(it & 0xffffu);
                    const int M = min(cb.nbr_count[s], cap);
                    offI = I * P3_CHUNK;
                    mI = min(P3_CHUNK, M - offI);
                    if (J != I) {
                        offJ = J * P3_CHUNK;
                        mJ = min(P3_CHUNK, M - offJ);
                    }
                }
                if (mI + mJ > 1) item(s, offI, mI, offJ, mJ);
                w = __shfl_sync(0xffffffffu, wn, 0);
            }
        }
    } else {
        // lists of at most one chunk: one item per particle
        unsigned int w = 0;
        if (lane == 0) w = atomicAdd(cb.work_counter, 1u);
        w = __shfl_sync(0xffffffffu, w, 0);
        while ((int64_t)w < n) {
            unsigned int wn = 0;
            if (lane == 0) wn = atomicAdd(cb.work_counter, 1u);
            const int s = (int)w;
            const int M = min(cb.nbr_count[s], cap);
            if (M <= P3_CHUNK && M > 1) item(s, 0, M, 0, 0);
            w = __shfl_sync(0xffffffffu, wn, 0);
        }
        // longer lists: the chunk-pair items the neighbour kernel queued
        const unsigned int nlong = min(*cb.long_count, (unsigned int)cb.long_cap);
        if (lane == 0) w = atomicAdd(cb.work_counter + 1, 1u);
        w = __shfl_sync(0xffffffffu, w, 0);
        while (w < nlong) {
            unsigned int wn = 0;
            if (lane == 0) wn = atomicAdd(cb.work_counter + 1, 1u);
            const unsigned long long it = cb.long_items[w];
            const int s = (int)TBMD_IX((int64_t)(it >> 32), n, BS_LONG_ITEM), I = (int)((it >> 16) & 0xffffu),
                      J = (int)(it & 0xffffu);
            const int M = min(cb.nbr_count[s], cap);
            const int mI = min(P3_CHUNK, M - I * P3_CHUNK);
            const int mJ = J != I ? min(P3_CHUNK, M - J * P3_CHUNK) : 0;
            item(s, I * P3_CHUNK, mI, J * P3_CHUNK, mJ);
            w = __shfl_sync(0xffffffffu, wn, 0);
        }
    }
    flush(cur_sys);
}

void fill_grid_test_params(Grid &g);

// Half-width of the uncertainty band around cutoff^2 of the guarded third-edge test, for unit
// roundoff eps.  Mixed (eps32): each FP32 component of the third edge (two-float difference of edges
// from i, then L - |d|) is within e = 16 eps (max L + cutoff) of the FP64 value.  FP64 forms
// (eps64): the third edge is the FP64 difference of two FP64 edges from i, each within eps / 2 of
// its at most L + cutoff long exact value, so it and the reference's own x_k - x_j (and L - |d|)
// differ by a few eps (L + cutoff) per component, inside the same e.  The squared periodic
// distance is then within 2 sqrt(3) c e + 3 e^2 plus its own rounding (8 eps c^2) of the
// reference's.  Four times that is used.
static double guard_band(const Grid &g, double eps)
{
    const double c = sqrt(g.sqcut);
    const double Lm = fmax(g.L[0], fmax(g.L[1], g.L[2]));
    const double e = 16.0 * eps * (Lm + c);
    return 4.0 * (2.0 * 1.7320508075688772 * c * e + 3.0 * e * e + 8.0 * eps * g.sqcut);
}

// The raw squared distance equals the periodic formula for two neighbours of s that do not wrap
// (each within the cutoff of s per axis, so within 2 cutoffs of each other) when every box length
// is at least 4 cutoffs: then min(|d|, L - |d|) = |d| exactly.
static int raw_test_ok(const Grid &g)
{
    const double c = sqrt(g.sqcut) * 1.0000001;
    return (g.L[0] >= 4.0 * c && g.L[1] >= 4.0 * c && g.L[2] >= 4.0 * c) ? 1 : 0;
}

// Half-width of the band of the FP32 third-edge test of an item whose neighbours do not wrap, with
// hi + lo edges (mixed forces).  Each edge from s is formed in FP64 (components within the cutoff
// c) and split into hi + lo floats, exact to 2^-48 c.  A third-edge component
// w = (v_hi - u_hi) + (v_lo - u_lo) is then within 2^-23 |w| + 2^-45 c of the difference of the FP64
// edges: the hi difference rounds to within 2^-24 of itself and lies within 2^-23 c of w (the lo
// parts), the lo difference to within 2^-47 c, and the sum rounds once.  The squared length (one
// product and two FMAs over positive terms, three roundings) is then within
// (2^-22 + 3 * 2^-24) |w|^2 + 2^-42 c^2 of the squared FP64 difference, which is within 2^-46 c^2 of
// the reference's sum of squares of x_k - x_j (raw here: |w| <= 2 c <= L / 2).  Near cutoff^2 all of
// that is below 8 * 2^-24 c^2, and the thresholds themselves round to within 2^-24 c^2 in FP32.
// Four times the sum, 36 * 2^-24 c^2, is used.  It is independent of the box length, unlike the
// band of the wrapped form, whose L - |d| carries errors of order 2^-24 L.
static double raw_band(const Grid &g) { return 36.0 / 16777216.0 * g.sqcut; }  // 2^-24

void fill_grid_test_params(Grid &g)
{
    g.band = (float)guard_band(g, 1.0 / 8388608.0);      // 2^-23
    g.band64 = guard_band(g, 1.0 / 4503599627370496.0);  // 2^-52
    g.raw_lo = (float)(g.sqcut - raw_band(g));
    g.raw_hi = (float)(g.sqcut + raw_band(g));
    g.raw_ok = raw_test_ok(g);
}

template <class S>
static cudaError_t plan_p3bca_t(bool energy, int cap, int warps, P3Plan *plan)
{
    int dev = 0, num_sms = 0;
    cudaError_t e;
    if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
    if ((e = cudaDeviceGetAttribute(&num_sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
    (void)cap;
    const size_t per_warp = SlotLayout<S>::bytes_per_warp;
    const size_t smem_cap = 220 * 1024;
    if (warps < 1) warps = 1;
    if (warps > 8) warps = 8;
    while (warps > 1 && per_warp * warps > smem_cap) --warps;
    if (per_warp * warps > smem_cap) return cudaErrorInvalidValue;
    const size_t smem = per_warp * warps;
    auto kern = energy ? k_p3bca<S, true> : k_p3bca<S, false>;
    if ((e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)) != cudaSuccess)
        return e;
    int per_sm = 0;
    if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, warps * 32, smem)) != cudaSuccess) return e;
    if (per_sm < 1) per_sm = 1;
    plan->warps = warps;
    plan->smem = smem;
    plan->grid = num_sms * per_sm;
    return cudaSuccess;
}

cudaError_t plan_p3bca(bool mixed, bool dual, bool energy, int cap, int warps, P3Plan *plan)
{
    // the neighbour kernel's largest staging size (4096 candidates), set once outside any capture
    cudaError_t e0 = cudaFuncSetAttribute(k_neighbors, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)(4096 * NB_STAGE_BYTES));
    if (e0 != cudaSuccess) return e0;
    if (dual) {
        if (mixed) return plan_p3bca_t<Dual<float>>(energy, cap, warps, plan);
        return plan_p3bca_t<Dual<double>>(energy, cap, warps, plan);
    }
    if (mixed) return plan_p3bca_t<float>(energy, cap, warps, plan);
    return plan_p3bca_t<double>(energy, cap, warps, plan);
}

template <class S>
static cudaError_t launch_p3bca_t(bool energy, int64_t n, const Grid &g, const GridSet &set, CellBufs &cb, double nu,
                                  double *eo, unsigned long long *co, const P3Plan &plan, cudaStream_t st)
{
    // the work counters were armed by the neighbour kernel of the same step
    auto kern = energy ? k_p3bca<S, true> : k_p3bca<S, false>;
    kern<<<plan.grid, plan.warps * 32, plan.smem, st>>>(n, g, set, cb, nu, eo, co);
    return cudaGetLastError();
}

cudaError_t launch_p3bca(bool mixed, bool dual, bool energy, int64_t n, const Grid &g, const GridSet &set,
                         CellBufs &cb, double nu, double *eo, unsigned long long *co, const P3Plan &plan,
                         cudaStream_t st)
{
    if (n <= 0) return cudaSuccess;
    if (dual) {
        if (mixed) return launch_p3bca_t<Dual<float>>(energy, n, g, set, cb, nu, eo, co, plan, st);
        return launch_p3bca_t<Dual<double>>(energy, n, g, set, cb, nu, eo, co, plan, st);
    }
    if (mixed) return launch_p3bca_t<float>(energy, n, g, set, cb, nu, eo, co, plan, st);
    return launch_p3bca_t<double>(energy, n, g, set, cb, nu, eo, co, plan, st);
}

__global__ void k_unsort(int64_t n, const int32_t *__restrict__ sorted, const double *__restrict__ f0,
                         const double *__restrict__ f1, const double *__restrict__ f2, double *o0, double *o1,
                         double *o2)
{
    int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    int32_t i = (int32_t)TBMD_IX(sorted[s], n, BS_SORTED);
    o0[i] = f0[s];
    o1[i] = f1[s];
    o2[i] = f2[s];
}

cudaError_t launch_unsort(int64_t n, const CellBufs &cb, Out out, bool dual, cudaStream_t st)
{
    unsigned nb = (unsigned)((n + 255) / 256);
    k_unsort<<<nb, 256, 0, st>>>(n, cb.sorted, cb.fs[0], cb.fs[1], cb.fs[2], out.fx, out.fy, out.fz);
    if (dual) k_unsort<<<nb, 256, 0, st>>>(n, cb.sorted, cb.hs[0], cb.hs[1], cb.hs[2], out.hx, out.hy, out.hz);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------------------------
// Integrator (structs.hpp:40-99), FP64, in input order.  No FMA contraction, matching the
// reference's evaluation order: x = (x + v*dt) + aX*h with h = dt*dt*0.5 (the aX quirk: the
// acceleration vector is (aX, aX, aX)); a = g - f/m; v = v + a*(dt*0.5).

__global__ void k_predictor(int64_t n, double *x, double *y, double *z, const double *vx, const double *vy,
                            const double *vz, const double *ax, double dt)
{
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double h = __dmul_rn(__dmul_rn(dt, dt), 0.5);
    const double a = ax[i];
    const double ah = __dmul_rn(a, h);
    x[i] = __dadd_rn(__dadd_rn(x[i], __dmul_rn(vx[i], dt)), ah);
    y[i] = __dadd_rn(__dadd_rn(y[i], __dmul_rn(vy[i], dt)), ah);
    z[i] = __dadd_rn(__dadd_rn(z[i], __dmul_rn(vz[i], dt)), ah);
}

__global__ void k_update(int64_t n, double *vx, double *vy, double *vz, double *ax, double *ay, double *az,
                         const double *fx, const double *fy, const double *fz, const double *m, double dt, double gx,
                         double gy, double gz)
{
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double h = __dmul_rn(dt, 0.5);
    const double mi = m[i];
    const double nx = __dsub_rn(gx, __ddiv_rn(fx[i], mi));
    const double ny = __dsub_rn(gy, __ddiv_rn(fy[i], mi));
    const double nz = __dsub_rn(gz, __ddiv_rn(fz[i], mi));
    vx[i] = __dadd_rn(vx[i], __dmul_rn(nx, h));
    vy[i] = __dadd_rn(vy[i], __dmul_rn(ny, h));
    vz[i] = __dadd_rn(vz[i], __dmul_rn(nz, h));
    ax[i] = nx;
    ay[i] = ny;
    az[i] = nz;
}

cudaError_t launch_predictor(int64_t n, double *x, double *y, double *z, const double *vx, const double *vy,
                             const double *vz, const double *ax, double dt, cudaStream_t st)
{
    k_predictor<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(n, x, y, z, vx, vy, vz, ax, dt);
    return cudaGetLastError();
}

cudaError_t launch_update(int64_t n, double *vx, double *vy, double *vz, double *ax, double *ay, double *az,
                          const double *fx, const double *fy, const double *fz, const double *m, double dt, double gx,
                          double gy, double gz, cudaStream_t st)
{
    k_update<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(n, vx, vy, vz, ax, ay, az, fx, fy, fz, m, dt, gx, gy, gz);
    return cudaGetLastError();
}

// per_step[*step] = *cur + constant_count; ++*step; *cur = 0   (graph-replay safe step bookkeeping)
__global__ void k_record_count(unsigned long long *cur, unsigned long long *per_step, unsigned int *step,
                               unsigned long long constant_count)
{
    unsigned int s = *step;
    per_step[s] = *cur + constant_count;
    *step = s + 1;
    *cur = 0ull;
}

cudaError_t launch_record_count(unsigned long long *cur, unsigned long long *per_step, unsigned int *step,
                                unsigned long long constant_count, cudaStream_t st)
{
    k_record_count<<<1, 1, 0, st>>>(cur, per_step, step, constant_count);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------------------------
// Input check of tbmd_set_particles on the device: the particle arrays (x y z vx vy vz ax ay az m,
// n each, back to back) are checked for non-finite values and non-positive masses, and the
// extremes of x, y, z are reduced for the domain size.  Extremes travel as order-preserving
// integer keys (exact), so the domain equals the one a host loop over the same values gives.
__device__ __forceinline__ unsigned long long order_key(double d)
{
    const unsigned long long b = (unsigned long long)__double_as_longlong(d);
    return (b >> 63) ? ~b : (b | 0x8000000000000000ull);
}

__global__ void __launch_bounds__(256) k_validate(int64_t n, const double *__restrict__ a, ValidateResult *res)
{
    // per warp, then per block (shared memory), then one set of atomics per block: the result's
    // fields share one L2 slice, where same-address atomics from every warp serialise
    __shared__ unsigned int s_bad[8];
    __shared__ unsigned long long s_bm[8], s_mn[8][3], s_mx[8][3];
    unsigned int bad = 0;
    unsigned long long bad_mass = ~0ull;
    unsigned long long mn[3] = {~0ull, ~0ull, ~0ull}, mx[3] = {0ull, 0ull, 0ull};
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
#pragma unroll
        for (int k = 0; k < 10; ++k) {
            const double v = a[(int64_t)k * n + i];
            if (!isfinite(v)) bad |= 1u << k;
            if (k < 3) {
                const unsigned long long key = order_key(v);
                mn[k] = key < mn[k] ? key : mn[k];
                mx[k] = key > mx[k] ? key : mx[k];
            }
            if (k == 9 && !(v > 0.0) && (unsigned long long)i < bad_mass) bad_mass = (unsigned long long)i;
        }
    }
    auto warp_reduce = [&]() {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            bad |= __shfl_xor_sync(0xffffffffu, bad, o);
            const unsigned long long bm = __shfl_xor_sync(0xffffffffu, bad_mass, o);
            bad_mass = bm < bad_mass ? bm : bad_mass;
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                const unsigned long long lo = __shfl_xor_sync(0xffffffffu, mn[k], o);
                const unsigned long long hi = __shfl_xor_sync(0xffffffffu, mx[k], o);
                mn[k] = lo < mn[k] ? lo : mn[k];
                mx[k] = hi > mx[k] ? hi : mx[k];
            }
        }
    };
    warp_reduce();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) {
        s_bad[warp] = bad;
        s_bm[warp] = bad_mass;
        for (int k = 0; k < 3; ++k) {
            s_mn[warp][k] = mn[k];
            s_mx[warp][k] = mx[k];
        }
    }
    __syncthreads();
    if (warp == 0) {
        const bool has = lane < (int)(blockDim.x >> 5);
        bad = has ? s_bad[lane] : 0u;
        bad_mass = has ? s_bm[lane] : ~0ull;
        for (int k = 0; k < 3; ++k) {
            mn[k] = has ? s_mn[lane][k] : ~0ull;
            mx[k] = has ? s_mx[lane][k] : 0ull;
        }
        warp_reduce();
        if (lane == 0) {
            if (bad) atomicOr(&res->bad_arrays, bad);
            if (bad_mass != ~0ull) atomicMin(&res->bad_mass, bad_mass);
            for (int k = 0; k < 3; ++k) {
                atomicMin(&res->min_key[k], mn[k]);
                atomicMax(&res->max_key[k], mx[k]);
            }
        }
    }
}

cudaError_t launch_validate(int64_t n, const double *arrays, ValidateResult *res, int grid, cudaStream_t st)
{
    cudaError_t e;
    if ((e = cudaMemsetAsync(res, 0, sizeof(ValidateResult), st)) != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(&res->bad_mass, 0xff, 4 * sizeof(unsigned long long), st)) != cudaSuccess) return e;
    const int64_t need = (n + 255) / 256;
    k_validate<<<(unsigned)(need < grid ? need : grid), 256, 0, st>>>(n, arrays, res);
    return cudaGetLastError();
}

// Per-system input check of a batch: non-finite positions (flag) and the extremes of x, y, z of each
// system (order keys, keys[6 s + 0..2] minima, keys[6 s + 3..5] maxima; preset to ~0 / 0).
__global__ void __launch_bounds__(256) k_batch_extents(int64_t n, const double *__restrict__ x,
                                                       const double *__restrict__ y, const double *__restrict__ z,
                                                       const int64_t *__restrict__ sys_off, int nsys,
                                                       unsigned int *bad, unsigned long long *keys)
{
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    const int lane = threadIdx.x & 31;
    for (int64_t i0 = (int64_t)blockIdx.x * blockDim.x; i0 < n; i0 += stride) {
        const int64_t i = i0 + threadIdx.x;
        const bool in = i < n;
        const double v[3] = {in ? x[i] : 0.0, in ? y[i] : 0.0, in ? z[i] : 0.0};
        const int sys = in ? system_of(sys_off, nsys, i) : -1;
        if (in && !(isfinite(v[0]) && isfinite(v[1]) && isfinite(v[2]))) atomicOr(bad, 1u);
        // a warp whose lanes all belong to one system reduces first (systems are contiguous)
        const int s0 = __shfl_sync(0xffffffffu, sys, 0);
        if (__all_sync(0xffffffffu, sys == s0) && s0 >= 0) {
            for (int d = 0; d < 3; ++d) {
                unsigned long long lo = order_key(v[d]), hi = lo;
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) {
                    const unsigned long long a = __shfl_xor_sync(0xffffffffu, lo, o);
                    const unsigned long long b = __shfl_xor_sync(0xffffffffu, hi, o);
                    lo = a < lo ? a : lo;
                    hi = b > hi ? b : hi;
                }
                if (lane == 0) {
                    atomicMin(keys + 6 * s0 + d, lo);
                    atomicMax(keys + 6 * s0 + 3 + d, hi);
                }
            }
        } else if (in) {
            for (int d = 0; d < 3; ++d) {
                atomicMin(keys + 6 * sys + d, order_key(v[d]));
                atomicMax(keys + 6 * sys + 3 + d, order_key(v[d]));
            }
        }
    }
}

__global__ void k_init_extents(int nsys, unsigned int *bad, unsigned long long *keys)
{
    for (int k = threadIdx.x; k < 6 * nsys; k += blockDim.x) keys[k] = (k % 6) < 3 ? ~0ull : 0ull;
    if (threadIdx.x == 0) *bad = 0u;
}

cudaError_t launch_batch_extents(int64_t n, const double *x, const double *y, const double *z, const int64_t *sys_off,
                                 int nsys, unsigned int *bad, unsigned long long *keys, int grid, cudaStream_t st)
{
    k_init_extents<<<1, 256, 0, st>>>(nsys, bad, keys);
    const int64_t need = (n + 255) / 256;
    k_batch_extents<<<(unsigned)(need < grid ? need : grid), 256, 0, st>>>(n, x, y, z, sys_off, nsys, bad, keys);
    return cudaGetLastError();
}

double key_to_double(unsigned long long key)
{
    const unsigned long long b = (key >> 63) ? (key & 0x7fffffffffffffffull) : ~key;
    double d;
    std::memcpy(&d, &b, sizeof d);
    return d;
}


// The bounds-check record of this translation unit (see TBMD_IX), read and cleared; zero when the
// library was built without the checks.
cudaError_t bounds_read_kernels(BoundsRecord *out)
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
