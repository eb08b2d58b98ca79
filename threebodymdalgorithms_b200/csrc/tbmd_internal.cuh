// Internal declarations shared by the kernels (tbmd_kernels.cu) and the C ABI (tbmd_api.cu).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "at_math.cuh"

namespace tbmd {

// ---------------------------------------------------------------------------------------------
// Scalar plumbing for the generic triplet kernels.  S is the arithmetic type of the triplet math:
// double (FP64 drop-in), float (mixed precision), or Dual<double>/Dual<float> (the adjoint, whose
// tangent part carries the Hessian-vector product).  Acc is the matching FP64 accumulator.

template <class S>
struct Traits;
template <>
struct Traits<double> {
    using T = double;
    using Acc = double;
    static constexpr bool dual = false;
};
template <>
struct Traits<float> {
    using T = float;
    using Acc = double;
    static constexpr bool dual = false;
};
template <>
struct Traits<Dual<double>> {
    using T = double;
    using Acc = Dual<double>;
    static constexpr bool dual = true;
};
template <>
struct Traits<Dual<float>> {
    using T = float;
    using Acc = Dual<double>;
    static constexpr bool dual = true;
};

template <class S>
struct V3 {
    S x, y, z;
};
template <class S>
__device__ __forceinline__ V3<S> operator+(V3<S> a, V3<S> b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
template <class S>
__device__ __forceinline__ V3<S> operator-(V3<S> a, V3<S> b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
template <class S>
__device__ __forceinline__ V3<S> operator*(V3<S> a, S s) { return {a.x * s, a.y * s, a.z * s}; }
template <class S>
__device__ __forceinline__ S dot3(V3<S> a, V3<S> b) { return fma_(a.x, b.x, fma_(a.y, b.y, a.z * b.z)); }
// acc + a * s, component-wise fused
template <class S>
__device__ __forceinline__ V3<S> fma3(V3<S> a, S s, V3<S> acc)
{
    return {fma_(a.x, s, acc.x), fma_(a.y, s, acc.y), fma_(a.z, s, acc.z)};
}

template <class S>
__device__ __forceinline__ S szero() { return S(0); }
template <>
__device__ __forceinline__ Dual<double> szero<Dual<double>>() { return {0.0, 0.0}; }
template <>
__device__ __forceinline__ Dual<float> szero<Dual<float>>() { return {0.f, 0.f}; }
template <class S>
__device__ __forceinline__ V3<S> vzero() { return {szero<S>(), szero<S>(), szero<S>()}; }

// A scalar of type S from an FP64 value and an FP64 tangent (ignored by non-dual types).
template <class S>
__device__ __forceinline__ S make_s(double v, double d);
template <>
__device__ __forceinline__ double make_s<double>(double v, double) { return v; }
template <>
__device__ __forceinline__ float make_s<float>(double v, double) { return (float)v; }
template <>
__device__ __forceinline__ Dual<double> make_s<Dual<double>>(double v, double d) { return {v, d}; }
template <>
__device__ __forceinline__ Dual<float> make_s<Dual<float>>(double v, double d) { return {(float)v, (float)d}; }

template <class S>
__device__ __forceinline__ S constant(double c) { return make_s<S>(c, 0.0); }

// Widen to the FP64 accumulator type.
__device__ __forceinline__ double to_acc(double v) { return v; }
__device__ __forceinline__ double to_acc(float v) { return (double)v; }
__device__ __forceinline__ Dual<double> to_acc(Dual<double> v) { return v; }
__device__ __forceinline__ Dual<double> to_acc(Dual<float> v) { return {(double)v.v, (double)v.d}; }

__device__ __forceinline__ double shfl_idx(double v, int src) { return __shfl_sync(0xffffffffu, v, src); }
__device__ __forceinline__ float shfl_idx(float v, int src) { return __shfl_sync(0xffffffffu, v, src); }
template <class T>
__device__ __forceinline__ Dual<T> shfl_idx(Dual<T> v, int src)
{
    return {shfl_idx(v.v, src), shfl_idx(v.d, src)};
}
template <class S>
__device__ __forceinline__ V3<S> shfl_idx(V3<S> v, int src)
{
    return {shfl_idx(v.x, src), shfl_idx(v.y, src), shfl_idx(v.z, src)};
}
__device__ __forceinline__ double shfl_xor_(double v, int m) { return __shfl_xor_sync(0xffffffffu, v, m); }
template <class T>
__device__ __forceinline__ Dual<T> shfl_xor_(Dual<T> v, int m)
{
    return {shfl_xor_(v.v, m), shfl_xor_(v.d, m)};
}
template <class A>
__device__ __forceinline__ A warp_sum(A v)
{
#pragma unroll
    for (int m = 16; m > 0; m >>= 1) v = v + shfl_xor_(v, m);
    return v;
}
__device__ __forceinline__ unsigned long long warp_sum_u64(unsigned long long v)
{
#pragma unroll
    for (int m = 16; m > 0; m >>= 1) v += __shfl_xor_sync(0xffffffffu, v, m);
    return v;
}

// Output of a triplet kernel: forces (the value part) and, for the adjoint, H * direction (the
// tangent part), both accumulated in FP64.
struct Out {
    double *fx, *fy, *fz;
    double *hx, *hy, *hz;
};
__device__ __forceinline__ void atomic_out(const Out &o, int64_t idx, V3<double> a)
{
    atomicAdd(o.fx + idx, a.x);
    atomicAdd(o.fy + idx, a.y);
    atomicAdd(o.fz + idx, a.z);
}
__device__ __forceinline__ void atomic_out(const Out &o, int64_t idx, V3<Dual<double>> a)
{
    atomicAdd(o.fx + idx, a.x.v);
    atomicAdd(o.fy + idx, a.y.v);
    atomicAdd(o.fz + idx, a.z.v);
    atomicAdd(o.hx + idx, a.x.d);
    atomicAdd(o.hy + idx, a.y.d);
    atomicAdd(o.hz + idx, a.z.d);
}
__device__ __forceinline__ double acc_value(double a) { return a; }
__device__ __forceinline__ double acc_value(Dual<double> a) { return a.v; }
__device__ __forceinline__ double dual_tangent(double) { return 0.0; }
__device__ __forceinline__ double dual_tangent(Dual<double> a) { return a.d; }

// ---------------------------------------------------------------------------------------------
// Edge vectors.  A displacement from vertex i is formed in FP64 and rounded once to S.  For the
// mixed form (S = float) the rounding remainder is kept as a second float ("lo"), so that the third
// edge w = v - u = (v_hi - u_hi) + (v_lo - u_lo) is accurate to a relative FP32 epsilon even when
// j and k are close to each other and far from i (v_hi - u_hi is then exact by Sterbenz's lemma).
// The mixed adjoint (Dual<float>) splits the value and its tangent the same way.  For double and
// Dual<double> the lo part is identically zero and compiled away.

template <class S>
struct HasLo {
    static constexpr bool value = false;
};
template <>
struct HasLo<float> {
    static constexpr bool value = true;
};
// The mixed adjoint splits the value and the tangent into hi + lo parts too (see dot_uv).
template <>
struct HasLo<Dual<float>> {
    static constexpr bool value = true;
};

// hi and lo parts of one FP64 displacement component (plus its tangent for dual types)
template <class S>
__device__ __forceinline__ void split(double d, double t, S &hi, S &lo)
{
    hi = make_s<S>(d, t);
    lo = szero<S>();
}
template <>
__device__ __forceinline__ void split<float>(double d, double, float &hi, float &lo)
{
    hi = (float)d;
    lo = (float)(d - (double)hi);
}
template <>
__device__ __forceinline__ void split<Dual<float>>(double d, double t, Dual<float> &hi, Dual<float> &lo)
{
    hi = {(float)d, (float)t};
    lo = {(float)(d - (double)hi.v), (float)(t - (double)hi.d)};
}

template <class S>
__device__ __forceinline__ V3<S> third_edge(V3<S> uh, V3<S> ul, V3<S> vh, V3<S> vl)
{
    if (HasLo<S>::value) return (vh - uh) + (vl - ul);
    return vh - uh;
}

// p = u.v of the triplet math, from the edges u, v from i (hi and lo parts) and the third edge w.
// For the mixed adjoint the tangent u'.v + u.v' is formed as u'.w + (u' + v').u (v = u + w): for a
// close pair j, k with large, nearly opposite cotangents (a force-matching cotangent of a close pair
// is one), u' and v' nearly cancel, and u'.v + u.v' in FP32 would lose about log2(|u| / |w|) bits.
// u' + v' is summed from the hi and the lo parts of both tangents (the hi sum is exact where they
// cancel), so every term left is free of cancellation.
template <class S>
__device__ __forceinline__ S dot_uv(V3<S> uh, V3<S>, V3<S> vh, V3<S>, V3<S>)
{
    return dot3(uh, vh);
}
template <>
__device__ __forceinline__ Dual<float> dot_uv<Dual<float>>(V3<Dual<float>> uh, V3<Dual<float>> ul, V3<Dual<float>> vh,
                                                          V3<Dual<float>> vl, V3<Dual<float>> w)
{
    const float val = fmaf(uh.x.v, vh.x.v, fmaf(uh.y.v, vh.y.v, uh.z.v * vh.z.v));
    const float sx = (uh.x.d + vh.x.d) + (ul.x.d + vl.x.d);
    const float sy = (uh.y.d + vh.y.d) + (ul.y.d + vl.y.d);
    const float sz = (uh.z.d + vh.z.d) + (ul.z.d + vl.z.d);
    const float tan = fmaf(uh.x.d, w.x.v, fmaf(uh.y.d, w.y.v, uh.z.d * w.z.v)) +
                      fmaf(sx, uh.x.v, fmaf(sy, uh.y.v, sz * uh.z.v));
    return {val, tan};
}

// ---------------------------------------------------------------------------------------------
// Debug-build index checks.  Compiled with -DTBMD_BOUNDS_CHECK (libtbmd_checked.so),
// TBMD_IX(i, size, site) passes an index i inside [0, size) through and otherwise records it (the
// first violation's site, index and size, and a count) in a device-side record of its translation
// unit and yields 0, so the access stays inside the array and the kernel runs on: nothing traps and
// no wait is involved.  The host reads and clears the records with tbmd_bounds_report.  In the
// normal build TBMD_IX(i, size, site) is i.  Sites are numbered in BoundsSite.
struct BoundsRecord {
    unsigned int count;
    int site;
    long long index, size;
};
enum BoundsSite : int {
    BS_CELL_OF = 1,       // cell of a particle (assign, predictor-assign)
    BS_CELL_SLOT,         // sorted slot of a particle (scatter)
    BS_SORTED,            // sorted index -> input index (gather, unsort)
    BS_NBR_CELL,          // neighbour-cell table entry
    BS_STAGE,             // neighbour kernel staging place
    BS_CANDIDATE,         // neighbour kernel candidate particle
    BS_LIST,              // half-list entry (sorted index)
    BS_LONG_ITEM,         // chunk-pair item
    BS_SLOT,              // staged slot of a triplet item
    BS_SWEEP,             // AUTA / NATA particle index
    BS_PARTIAL,           // NATA partial-sum slot
    BS_SYSTEM,            // system of a batched item
    BS_GEN,               // generator word / particle
};
#ifdef TBMD_BOUNDS_CHECK
static __device__ BoundsRecord g_bounds_record;
__device__ __forceinline__ long long tbmd_ix(long long i, long long size, int site)
{
    if (i >= 0 && i < size) return i;
    if (atomicAdd(&g_bounds_record.count, 1u) == 0u) {
        g_bounds_record.site = site;
        g_bounds_record.index = i;
        g_bounds_record.size = size;
    }
    return 0;
}
#define TBMD_IX(i, size, site) tbmd_ix((long long)(i), (long long)(size), (site))
#else
#define TBMD_IX(i, size, site) (i)
#endif
// Host side: this translation unit's record (a zero record in the normal build), cleared after reading.
cudaError_t bounds_read_kernels(BoundsRecord *out);
cudaError_t bounds_read_gen(BoundsRecord *out);

// ---------------------------------------------------------------------------------------------
// Kernel argument blocks.

// Positions (FP64 SoA) and, for the adjoint, the direction vector (cotangent on the forces).
struct Pos {
    const double *x, *y, *z;
    const double *dx, *dy, *dz;
};

// Static work list of the no-cutoff sweeps.  A work item is (system, block b of JB consecutive j,
// i).  Systems are packed back to back (particles sys_off[s] .. sys_off[s+1]-1); a single system
// is nsys = 1.  NATA uses only nblocks/total/counter (its items are b * n + i).
struct SweepWork {
    const int64_t *prefix;       // per system: items of blocks < b (nblocks_s + 1 entries each)
    int nblocks;                 // single-system NATA: number of j-blocks
    int64_t total;               // items over all systems
    unsigned int *counter;       // dynamic item counter, zeroed before the launch
    int nsys;
    const int64_t *sys_items;    // [nsys + 1] first item of each system
    const int64_t *sys_off;      // [nsys + 1] first particle of each system
    const int64_t *sys_prefix;   // [nsys] start of each system's block prefix in `prefix`
    const int32_t *sys_nblocks;  // [nsys]
    int64_t kseg;                // AUTA: k range of one item (a multiple of 32), 0 = to the system's end
};

// Cell grid of the P3BCA path (one per system).  band, band64, raw_lo / raw_hi and raw_ok
// parametrise the guarded cutoff tests of the list and triplet kernels.
struct Grid {
    double L[3], lo[3], w[3];
    int dims[3];
    int64_t ncells;
    double sqcut;
    double band64;  // half-width of the FP64 uncertainty band around cutoff^2 (FP64 forms)
    float band;     // half-width of the FP32 uncertainty band around cutoff^2 (FP32 geometry)
    float raw_lo;   // FP32 third-edge test without wrapping, hi + lo edges: d2 <= raw_lo is inside,
    float raw_hi;   // d2 > raw_hi outside, the exact test in between
    int raw_ok;     // every box length >= 4 cutoffs: raw distance = periodic formula for non-wrapping pairs
};

// Several independent systems packed back to back: system s owns particles (and sorted slots)
// sys_off[s] .. sys_off[s+1]-1 and cells cell_off[s] .. cell_off[s+1]-1 of the concatenated grid.
// nsys = 1 is the single-system case (the kernels then use the Grid passed by value).
struct GridSet {
    const Grid *grids;       // [nsys] device
    const int64_t *cell_off;  // [nsys + 1] device
    const int64_t *sys_off;   // [nsys + 1] device
    int nsys;
};
void fill_grid_test_params(Grid &g);

// ---------------------------------------------------------------------------------------------
// Launchers (tbmd_kernels.cu).  All take the stream they run on and return the launch error.

int sweep_block_size(int algorithm, bool mixed, bool dual, int R);
int64_t sweep_items(int algorithm, int64_t n, int JB, int64_t *prefix_host /* nb+1 or NULL */, int64_t kseg = 0);
// energy_out: one accumulator per system (index = system)

cudaError_t launch_auta(bool mixed, bool dual, int R, bool energy, int64_t n, Pos pos, Out out, double *energy_out,
                        double nu, SweepWork work, int grid, cudaStream_t st);
cudaError_t launch_nata(bool mixed, bool dual, int R, bool energy, int64_t n, Pos pos, Out out, double *energy_out,
                        double nu, SweepWork work, double *partial, int grid, cudaStream_t st);
cudaError_t launch_nata_reduce(bool dual, int64_t n, int nblocks, const double *partial, Out out, cudaStream_t st);

// P3BCA pipeline
// Half-list chunk of the P3BCA triplet kernel: lists of at most P3_CHUNK entries are one work item,
// longer ones are split into chunk pairs.
constexpr int P3_CHUNK = 64;

struct CellBufs {
    int32_t *cell_of;      // [n] cell of each particle (input order)
    int32_t *cell_rank;    // [n] its rank within the cell (the old count its increment returned); the
                           //     step's scatter replaces it by the particle's sorted slot
    int32_t *cell_count;   // [ncells]
    int32_t *cell_start;   // [ncells + 1]
    int32_t *cell_out;     // [ncells] 1 if the cell holds a particle whose raw coordinates lie outside the
                           //          box (binned by wrapping); follows cell_count in memory
    int32_t *sorted;       // [n] sorted slot -> original index
    double *xs, *ys, *zs;  // [n] positions in sorted order
    float4 *qhi, *qlo;     // [n] sorted positions relative to the system's box corner lo, as FP32
                           //     hi + lo parts (x, y, z, unused): the neighbour kernel's FP32 test
    double *dxs, *dys, *dzs;  // [n] adjoint direction in sorted order (or NULL)
    int32_t *nbr;          // [n * cap] half neighbour lists (sorted indices)
    int32_t *nbr_count;    // [n]
    int32_t *max_count;    // [1] largest list length seen (overflow detection)
    unsigned int *work_counter;  // [2] dynamic item counters of the triplet kernel (particles, chunk pairs)
    int cap;
    // lists longer than P3_CHUNK: (s << 32 | I << 16 | J) chunk-pair items, queued by the neighbour kernel
    unsigned long long *long_items;  // [long_cap]
    int long_cap;
    unsigned int *long_count;  // [1] items queued by this evaluation (reset before the neighbour kernel)
    unsigned int *long_max;    // [1] largest item total requested (overflow detection)
    double *fs[3];         // [n] forces in sorted order
    double *hs[3];         // [n] H*direction in sorted order (adjoint)
};
// For a GridSet, g is the first system's grid with ncells = total cells over all systems.
cudaError_t launch_cell_build(int64_t n, Pos pos, const Grid &g, const GridSet &set, CellBufs &cb, bool with_dir,
                              cudaStream_t st, int *launches);
// The step of one system: predictor fused into the cell build; unsort, then the update fused with
// the step's count record (st13: the 13 state arrays x y z vx vy vz ax ay az m fx fy fz).
cudaError_t launch_step_cells(int64_t n, double *const st13[13], double dt, const Grid &g, CellBufs &cb,
                              cudaStream_t st, int *launches);
cudaError_t launch_unsort_update(int64_t n, const CellBufs &cb, double *const st13[13], double dt, const double g3[3],
                                 unsigned long long *cur, unsigned long long *per_step, unsigned int *step,
                                 cudaStream_t st);
cudaError_t launch_neighbors(int64_t n, const Grid &g, const GridSet &set, const int32_t *nbr_cells, int max_stage,
                             CellBufs &cb, cudaStream_t st);
int neighbor_stage_cap(const Grid &g, int64_t n);
// host: neighbour-cell table rows (27 ints per cell, ids >= the cell's own, ascending, -1 padded)
void neighbor_cell_table(const Grid &g, int64_t cell0, int32_t *out);
// Launch shape of the P3BCA triplet kernel for a list capacity; computed outside graph capture.
struct P3Plan {
    int warps = 0;
    size_t smem = 0;
    int grid = 0;
};
cudaError_t plan_p3bca(bool mixed, bool dual, bool energy, int cap, int warps_requested, P3Plan *plan);
// energy_out / count_out: one accumulator per system
cudaError_t launch_p3bca(bool mixed, bool dual, bool energy, int64_t n, const Grid &g, const GridSet &set,
                         CellBufs &cb, double nu, double *energy_out, unsigned long long *count_out,
                         const P3Plan &plan, cudaStream_t st);
// forces (and H*d) from sorted order back to input order
cudaError_t launch_unsort(int64_t n, const CellBufs &cb, Out out, bool dual, cudaStream_t st);

// integrator
cudaError_t launch_predictor(int64_t n, double *x, double *y, double *z, const double *vx, const double *vy,
                             const double *vz, const double *ax, double dt, cudaStream_t st);
cudaError_t launch_update(int64_t n, double *vx, double *vy, double *vz, double *ax, double *ay, double *az,
                          const double *fx, const double *fy, const double *fz, const double *m, double dt, double gx,
                          double gy, double gz, cudaStream_t st);
// Result of the device-side input check of tbmd_set_particles (k_validate).
struct ValidateResult {
    unsigned int bad_arrays;  // bit k: array k holds a non-finite value
    unsigned int pad;
    unsigned long long bad_mass;    // smallest index with mass <= 0 (or NaN), ~0 if none
    unsigned long long min_key[3];  // order-preserving keys of min / max of x, y, z
    unsigned long long max_key[3];
};
// arrays: x y z vx vy vz ax ay az m, n each, back to back
cudaError_t launch_validate(int64_t n, const double *arrays, ValidateResult *res, int grid, cudaStream_t st);
double key_to_double(unsigned long long key);
// Batched input check: *bad = 1 on a non-finite position; keys[6 s + d] / keys[6 s + 3 + d] the order
// keys of the minimum / maximum of coordinate d of system s.
cudaError_t launch_batch_extents(int64_t n, const double *x, const double *y, const double *z, const int64_t *sys_off,
                                 int nsys, unsigned int *bad, unsigned long long *keys, int grid, cudaStream_t st);

// Particle generation identical to the reference's particlegenerator (tbmd_gen.cu).
cudaError_t launch_mt19937(uint32_t seed, int64_t nwords, uint32_t *out, cudaStream_t st);
cudaError_t launch_uniform_positions(int64_t n, const uint32_t *words, const double corner[3], const double box[3],
                                     double *x, double *y, double *z, cudaStream_t st);
size_t polar_scratch_bytes(int64_t attempts);
int64_t polar_attempts_per_pass();
// One pass of T polar-method attempts from attempt t0 (generation indices from g0 on); writes the
// particles of generations < G and the generation count after the pass to *accepted_end (host).
cudaError_t launch_polar_pass(uint64_t x0, uint64_t t0, int64_t T, unsigned long long g0, unsigned long long G,
                              int64_t m, int64_t per, const double *const centres[3], double mean, double stddev,
                              double *x, double *y, double *z, void *scratch, unsigned long long *accepted_end,
                              cudaStream_t st);
cudaError_t launch_round_sig6(int64_t n, double *a, cudaStream_t st);
cudaError_t launch_fill(int64_t n, double v, double *a, cudaStream_t st);

cudaError_t launch_record_count(unsigned long long *cur, unsigned long long *per_step, unsigned int *step,
                                unsigned long long constant_count, cudaStream_t st);

}  // namespace tbmd
