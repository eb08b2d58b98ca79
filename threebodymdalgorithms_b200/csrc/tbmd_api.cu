// C ABI (include/tbmd.h): context, particle state, the Simulation step loop, forces, adjoint,
// device-pointer variants.  Host code in C++; every device operation is enqueued on the context
// stream.  Multi-step runs are captured once per configuration as a CUDA graph of one step and
// replayed; per-step triplet counts are recorded on the device and read back once per call.
#include <cuda_runtime.h>

#include <cfloat>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstddef>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <new>
#include <string>
#include <vector>

#include "../../include/tbmd.h"
#include "tbmd_internal.cuh"

using namespace tbmd;

namespace {

constexpr double kCellMargin = 1.000001;  // cell width >= cutoff * margin (same constant as the oracle)

struct DevBuf {
    void *p = nullptr;
    size_t bytes = 0;
    cudaError_t ensure(size_t b)
    {
        if (b <= bytes && p) return cudaSuccess;
        if (p) cudaFree(p);
        p = nullptr;
        bytes = 0;
        cudaError_t e = cudaMalloc(&p, b ? b : 16);
        if (e == cudaSuccess) bytes = b;
        return e;
    }
    void release()
    {
        if (p) cudaFree(p);
        p = nullptr;
        bytes = 0;
    }
    template <class T>
    T *as() const { return (T *)p; }
};

}  // namespace

struct tbmd_ctx {
    tbmd_config cfg{};
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    // tbmd_step_host: a second stream for the copies that overlap the step, and an event recorded
    // in every step once the predictor has written the positions (both made on first use)
    cudaStream_t copy_stream = nullptr;
    cudaEvent_t pos_event = nullptr;
    // pinned host words for the per-step counts and the overflow flags read after each step attempt
    // (a read into pageable memory would block the host until the whole step had finished)
    void *hstep = nullptr;
    size_t hstep_bytes = 0;
    std::string err;
    std::string tuning;
    uint64_t launches = 0;

    int64_t n = 0;
    std::vector<int32_t> id;

    // particle state, 13 FP64 arrays of n: x y z vx vy vz ax ay az m fx fy fz
    DevBuf state;
    double *s[13] = {};
    DevBuf snapshot;  // copy of x..az taken before a multi-step run (capacity retry)
    DevBuf staging;   // tbmd_set_particles: incoming arrays and their check result
    DevBuf gen_buf;   // tbmd_generate_particles: generator words, cluster centres, scan scratch

    // scalars: energy, count_cur, step counter, per-step counts
    DevBuf scalars;
    DevBuf step_counts;
    int64_t step_counts_cap = 0;

    // no-cutoff sweeps
    int R_auta = 4, R_nata = 2, R_fp64 = 2;
    DevBuf sweep_sys;  // single system: sys_items[2], sys_off[2], sys_prefix[1], sys_nblocks[1]
    DevBuf prefix;
    int prefix_JB = 0, prefix_alg = -1;
    int64_t prefix_kseg = 0;  // k range per AUTA item of the current work list (0: the whole sweep)
    int64_t prefix_n = -1;
    int nblocks = 0;
    int64_t total_items = 0;
    DevBuf partial;
    int sweep_grid = 0;

    // P3BCA
    bool domain_set = false;
    double L[3] = {0, 0, 0}, lo[3] = {0, 0, 0};
    Grid grid{};          // single system, or for a batch: first system's grid with ncells = all cells
    GridSet gset{};       // device tables of the systems being evaluated
    DevBuf gset_single;   // Grid[1] + cell_off[2] + sys_off[2] of the single-system case
    alignas(8) unsigned char gset_host[256] = {};  // host copy of what gset_single holds
    DevBuf ncell_tab;     // neighbour-cell table of the cells being evaluated (27 per cell)
    Grid ncell_grid{};    // grid the single-system table was built for
    bool ncell_single = false;
    std::vector<int32_t> ncell_batch_key;  // per-system dims the batched table was built for
    int max_stage = 256;  // neighbour staging capacity
    DevBuf cell_n, cell_c, nbr_buf;
    DevBuf long_buf;      // chunk-pair items of long half lists
    int long_cap = 0;     // capacity of long_buf in items
    int64_t cell_bufs_n = -1, cell_bufs_cells = -1;
    CellBufs cb{};
    int cap = 0;
    // list capacity of the last complete single-system P3BCA evaluation and its particle count: a
    // new particle set of the same size starts there instead of at the mean-density estimate, so a
    // clustered system that is reset and stepped again does not overflow and re-run every time
    int cap_used = 0;
    int64_t cap_used_n = -1;
    int p3_warps = 4;
    P3Plan plan{};
    int plan_key[5] = {-1, -1, -1, -1, -1};  // (mixed, dual, energy, cap, warps) the plan was made for

    // adjoint / device-variant scratch
    DevBuf dirs, hvp;

    // batched evaluation (tbmd_batch_*): packed positions/directions/outputs and system tables
    DevBuf bpos, bout, bsys, bprefix;
    DevBuf bext;  // batched input check: offsets, non-finite flag, per-system extremes
    void *hpin = nullptr;  // pinned host buffer of batched results
    size_t hpin_bytes = 0;

    // phase profiling (eager mode): marks recorded on the stream, resolved after each sync
    bool profiling = false;
    std::vector<cudaEvent_t> event_pool;
    std::vector<std::pair<int, cudaEvent_t>> marks;  // (phase that starts at this mark, event)
    double phase_ms[5] = {0, 0, 0, 0, 0};
    uint64_t phase_calls[5] = {0, 0, 0, 0, 0};
    uint64_t phase_launches[5] = {0, 0, 0, 0, 0};
    int cur_phase = -1;
    int cur_phase_launch0 = 0;

    // graph of one step
    cudaGraphExec_t gexec = nullptr;
    bool graph_valid = false;
    int graph_launches_per_step = 0;
};

// ---------------------------------------------------------------------------------------------
// helpers

static tbmd_status fail(tbmd_ctx *c, tbmd_status s, const char *fmt, ...)
{
    if (c) {
        char buf[512];
        va_list ap;
        va_start(ap, fmt);
        vsnprintf(buf, sizeof buf, fmt, ap);
        va_end(ap);
        c->err = buf;
    }
    return s;
}

#define CK(call)                                                                                             \
    do {                                                                                                     \
        cudaError_t e_ = (call);                                                                             \
        if (e_ != cudaSuccess) return fail(ctx, TBMD_CUDA_ERROR, "%s: %s (%s:%d)", #call, cudaGetErrorString(e_), \
                                           __FILE__, __LINE__);                                              \
    } while (0)

static bool is_p3bca_cut(const tbmd_ctx *ctx) { return ctx->cfg.algorithm == TBMD_P3BCA && ctx->cfg.cutoff > 0; }
static bool mixed(const tbmd_ctx *ctx) { return ctx->cfg.precision == TBMD_MIXED; }

static unsigned long long choose3(int64_t n)
{
    if (n < 3) return 0;
    unsigned __int128 v = (unsigned __int128)n * (unsigned __int128)(n - 1) * (unsigned __int128)(n - 2) / 6;
    return v > (unsigned __int128)UINT64_MAX ? UINT64_MAX : (unsigned long long)v;
}

static double *energy_ptr(tbmd_ctx *c) { return c->scalars.as<double>(); }
static unsigned long long *count_ptr(tbmd_ctx *c) { return (unsigned long long *)(c->scalars.as<char>() + 8); }
static unsigned int *step_ptr(tbmd_ctx *c) { return (unsigned int *)(c->scalars.as<char>() + 16); }
static unsigned int *sweep_counter(tbmd_ctx *c) { return (unsigned int *)(c->scalars.as<char>() + 24); }

static int sweep_R(const tbmd_ctx *ctx)
{
    if (!mixed(ctx)) return ctx->R_fp64;
    return ctx->cfg.algorithm == TBMD_NATA ? ctx->R_nata : ctx->R_auta;
}

static void invalidate_graph(tbmd_ctx *ctx)
{
    if (ctx->gexec) cudaGraphExecDestroy(ctx->gexec);
    ctx->gexec = nullptr;
    ctx->graph_valid = false;
}

enum Phase { PH_PREDICTOR = 0, PH_CELLS = 1, PH_NEIGHBORS = 2, PH_TRIPLETS = 3, PH_UPDATE = 4, PH_END = -1 };

// Start a profiling phase (or end the current one with PH_END).  nl = launches so far in this
// enqueue; the difference is attributed to the phase that ends.
static void phase_mark(tbmd_ctx *ctx, cudaStream_t st, int phase, int nl)
{
    if (!ctx->profiling) return;
    if (ctx->cur_phase >= 0) ctx->phase_launches[ctx->cur_phase] += (uint64_t)(nl - ctx->cur_phase_launch0);
    cudaEvent_t e;
    if (ctx->event_pool.empty()) {
        if (cudaEventCreate(&e) != cudaSuccess) return;
    } else {
        e = ctx->event_pool.back();
        ctx->event_pool.pop_back();
    }
    cudaEventRecord(e, st);
    ctx->marks.push_back({phase, e});
    ctx->cur_phase = phase;
    ctx->cur_phase_launch0 = nl;
    if (phase >= 0) ctx->phase_calls[phase] += 1;
}

// After a synchronisation: add the elapsed time between consecutive marks to their phases.
static void phase_resolve(tbmd_ctx *ctx)
{
    for (size_t k = 0; k + 1 < ctx->marks.size(); ++k) {
        int ph = ctx->marks[k].first;
        float ms = 0.f;
        if (ph >= 0 && cudaEventElapsedTime(&ms, ctx->marks[k].second, ctx->marks[k + 1].second) == cudaSuccess)
            ctx->phase_ms[ph] += ms;
    }
    for (auto &m : ctx->marks) ctx->event_pool.push_back(m.second);
    ctx->marks.clear();
    ctx->cur_phase = -1;
}

// Work list of the no-cutoff sweep for (algorithm, n, R).  A small AUTA system has fewer (block, i)
// items than the GPU has resident warps, and their k sweeps differ in length by the whole system, so
// the longest one sets the kernel time: its items are then split by k range (kseg particles each),
// the longest range that still gives every resident warp four items.
static tbmd_status ensure_sweep(tbmd_ctx *ctx, int alg, int64_t n, int R, bool dual)
{
    const int JB = 32 * R;
    int sms = 0;
    CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device));
    int per_sm = 2048 / sweep_block_size(alg, mixed(ctx), dual, R);  // resident blocks bounded below by registers
    if (per_sm < 1) per_sm = 1;
    ctx->sweep_grid = sms * per_sm;
    int64_t kseg = 0;
    if (alg == TBMD_AUTA) {
        const int64_t want = 4ll * ctx->sweep_grid * (sweep_block_size(alg, mixed(ctx), dual, R) / 32);
        if (sweep_items(alg, n, JB, nullptr) < want) {
            for (kseg = 256; kseg > 32 && sweep_items(alg, n, JB, nullptr, kseg) < want; kseg /= 2) {
            }
        }
    }
    if (ctx->prefix_n != n || ctx->prefix_JB != JB || ctx->prefix_alg != alg || ctx->prefix_kseg != kseg) {
        std::vector<int64_t> pre((size_t)(n / JB + 3), 0);
        int64_t total = sweep_items(alg, n, JB, pre.data(), kseg);
        int64_t nb = n >= 3 ? (n - 2 + JB) / JB : 0;
        if (total >= (int64_t)UINT32_MAX - 65536)
            return fail(ctx, TBMD_INVALID_ARG, "n = %lld gives too many sweep work items", (long long)n);
        CK(ctx->prefix.ensure(sizeof(int64_t) * (nb + 1)));
        CK(cudaMemcpyAsync(ctx->prefix.p, pre.data(), sizeof(int64_t) * (nb + 1), cudaMemcpyHostToDevice, ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
        ctx->prefix_n = n;
        ctx->prefix_JB = JB;
        ctx->prefix_alg = alg;
        ctx->prefix_kseg = kseg;
        ctx->nblocks = (int)nb;
        ctx->total_items = total;
        // one system: sys_items = {0, total}, sys_off = {0, n}, sys_prefix = {0}, sys_nblocks = {nb}
        struct {
            int64_t items[2], off[2], pre[1];
            int32_t nbl[2];
        } tab = {{0, total}, {0, n}, {0}, {(int32_t)nb, 0}};
        CK(ctx->sweep_sys.ensure(sizeof tab));
        CK(cudaMemcpyAsync(ctx->sweep_sys.p, &tab, sizeof tab, cudaMemcpyHostToDevice, ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
        if (alg == TBMD_NATA) CK(ctx->partial.ensure(sizeof(double) * 3 * (size_t)n * (size_t)(nb > 0 ? nb : 1)));
    }
    return TBMD_OK;
}

// Work list of the single system of the context (tables filled by ensure_sweep).
static SweepWork single_sweep(tbmd_ctx *ctx)
{
    const char *t = ctx->sweep_sys.as<char>();
    return SweepWork{ctx->prefix.as<int64_t>(), ctx->nblocks, ctx->total_items, sweep_counter(ctx), 1,
                     (const int64_t *)t, (const int64_t *)(t + 16), (const int64_t *)(t + 32),
                     (const int32_t *)(t + 40), ctx->prefix_kseg};
}

// Cell grid for the current domain and cutoff (oracle tbo_cell_dims).
static void make_grid(tbmd_ctx *ctx)
{
    Grid &g = ctx->grid;
    for (int d = 0; d < 3; ++d) {
        double m = std::floor(ctx->L[d] / (ctx->cfg.cutoff * kCellMargin));
        int nd = (m >= 3.0) ? (m > 1024.0 ? 1024 : (int)m) : 1;
        g.dims[d] = nd;
        g.L[d] = ctx->L[d];
        g.lo[d] = ctx->lo[d];
        g.w[d] = ctx->L[d] / (double)nd;
    }
    g.ncells = (int64_t)g.dims[0] * g.dims[1] * g.dims[2];
    g.sqcut = ctx->cfg.cutoff * ctx->cfg.cutoff;
    fill_grid_test_params(g);
}

// Grid of one system from its box (L, lo) and the context's cutoff (same rule as make_grid).
static Grid system_grid(const tbmd_ctx *ctx, const double *L, const double *lo)
{
    Grid g{};
    for (int d = 0; d < 3; ++d) {
        double m = std::floor(L[d] / (ctx->cfg.cutoff * kCellMargin));
        int nd = (m >= 3.0) ? (m > 1024.0 ? 1024 : (int)m) : 1;
        g.dims[d] = nd;
        g.L[d] = L[d];
        g.lo[d] = lo[d];
        g.w[d] = L[d] / (double)nd;
    }
    g.ncells = (int64_t)g.dims[0] * g.dims[1] * g.dims[2];
    g.sqcut = ctx->cfg.cutoff * ctx->cfg.cutoff;
    fill_grid_test_params(g);
    return g;
}

// Neighbour-list capacity estimate from the mean density: twice the expected half-list length
// plus slack, rounded to 32.  Clustered inputs are corrected by the overflow retry.
static int initial_cap(const tbmd_ctx *ctx, int64_t n)
{
    double vol = ctx->L[0] * ctx->L[1] * ctx->L[2];
    double rho = vol > 0 ? (double)n / vol : 0.0;
    double c = ctx->cfg.cutoff;
    double half = 4.18879020478639 * c * c * c * rho * 0.5;
    double want = 2.0 * half + 48.0;
    if (want > (double)n) want = (double)n + 32;
    int cap = ((int)want + 31) / 32 * 32;
    return cap < 32 ? 32 : cap;
}

// Cell-grid buffers for n particles and ncells cells (all systems), neighbour lists at ctx->cap,
// and the triplet kernel's launch plan.
static tbmd_status ensure_cell_bufs(tbmd_ctx *ctx, int64_t n, int64_t nc, bool dual, bool energy)
{
    if (ctx->cell_bufs_n != n || ctx->cell_bufs_cells != nc) {
        // per particle: float4 qhi qlo; FP64 xs ys zs dxs dys dzs fs[3] hs[3]; int32 cell_of, sorted,
        // nbr_count, cell_rank
        CK(ctx->cell_n.ensure((size_t)n * (2 * sizeof(float4) + 12 * sizeof(double) + 4 * sizeof(int32_t)) + 256));
        CK(ctx->cell_c.ensure((size_t)(3 * nc + 1) * sizeof(int32_t) + 256));
        CellBufs &cb = ctx->cb;
        cb.qhi = ctx->cell_n.as<float4>();
        cb.qlo = cb.qhi + n;
        double *d = (double *)(cb.qlo + n);
        cb.xs = d;
        cb.ys = d + n;
        cb.zs = d + 2 * n;
        cb.dxs = d + 3 * n;
        cb.dys = d + 4 * n;
        cb.dzs = d + 5 * n;
        for (int k = 0; k < 3; ++k) {
            cb.fs[k] = d + (6 + k) * n;
            cb.hs[k] = d + (9 + k) * n;
        }
        int32_t *q = (int32_t *)(d + 12 * n);
        cb.cell_of = q;
        cb.sorted = q + n;
        cb.nbr_count = q + 2 * n;
        cb.cell_rank = q + 3 * n;
        int32_t *r = ctx->cell_c.as<int32_t>();
        cb.cell_count = r;  // count, out: adjacent (zeroed by one memset)
        cb.cell_out = r + nc;
        cb.cell_start = r + 2 * nc;
        ctx->cell_bufs_n = n;
        ctx->cell_bufs_cells = nc;
    }
    CK(ctx->nbr_buf.ensure((size_t)n * ctx->cap * sizeof(int32_t) + 64));
    ctx->cb.nbr = ctx->nbr_buf.as<int32_t>();
    if (ctx->long_cap < 1024) ctx->long_cap = 1024;
    CK(ctx->long_buf.ensure((size_t)ctx->long_cap * sizeof(unsigned long long)));
    ctx->cb.long_items = ctx->long_buf.as<unsigned long long>();
    ctx->cb.long_cap = ctx->long_cap;
    ctx->cb.max_count = (int32_t *)(ctx->scalars.as<char>() + 28);
    ctx->cb.work_counter = (unsigned int *)(ctx->scalars.as<char>() + 32);  // and + 36
    ctx->cb.long_count = (unsigned int *)(ctx->scalars.as<char>() + 40);
    ctx->cb.long_max = (unsigned int *)(ctx->scalars.as<char>() + 44);
    ctx->cb.cap = ctx->cap;
    const int key[5] = {mixed(ctx) ? 1 : 0, dual ? 1 : 0, energy ? 1 : 0, ctx->cap, ctx->p3_warps};
    if (std::memcmp(key, ctx->plan_key, sizeof key) != 0) {
        CK(plan_p3bca(mixed(ctx), dual, energy, ctx->cap, ctx->p3_warps, &ctx->plan));
        std::memcpy(ctx->plan_key, key, sizeof key);
    }
    return TBMD_OK;
}

static tbmd_status ensure_cells(tbmd_ctx *ctx, int64_t n, bool dual, bool energy)
{
    if (!ctx->domain_set)
        return fail(ctx, TBMD_NOT_READY, "P3BCA needs a domain: set particles or call tbmd_set_domain");
    make_grid(ctx);
    if (ctx->cap == 0) {
        ctx->cap = initial_cap(ctx, n);
        if (ctx->cap_used_n == n && ctx->cap_used > ctx->cap) ctx->cap = ctx->cap_used;
    }
    // single-system tables: grids[0], cell_off = {0, ncells}, sys_off = {0, n}
    struct {
        Grid g;
        int64_t cell_off[2], sys_off[2];
    } tab;
    std::memset(&tab, 0, sizeof tab);  // padding too: the table is compared bytewise below
    tab.g = ctx->grid;
    tab.cell_off[1] = ctx->grid.ncells;
    tab.sys_off[1] = n;
    static_assert(sizeof tab <= sizeof ctx->gset_host, "single-system table size");
    if (!ctx->gset_single.p || std::memcmp(ctx->gset_host, &tab, sizeof tab) != 0) {
        CK(ctx->gset_single.ensure(sizeof tab));
        CK(cudaMemcpyAsync(ctx->gset_single.p, &tab, sizeof tab, cudaMemcpyHostToDevice, ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));  // tab lives on this stack frame
        std::memcpy(ctx->gset_host, &tab, sizeof tab);
    }
    char *base = ctx->gset_single.as<char>();
    ctx->gset = GridSet{(const Grid *)base, (const int64_t *)(base + offsetof(decltype(tab), cell_off)),
                        (const int64_t *)(base + offsetof(decltype(tab), sys_off)), 1};
    ctx->max_stage = neighbor_stage_cap(ctx->grid, n);
    if (!ctx->ncell_single || std::memcmp(&ctx->ncell_grid, &ctx->grid, sizeof(Grid)) != 0) {
        std::vector<int32_t> tab27((size_t)ctx->grid.ncells * 27);
        neighbor_cell_table(ctx->grid, 0, tab27.data());
        CK(ctx->ncell_tab.ensure(sizeof(int32_t) * tab27.size()));
        CK(cudaMemcpyAsync(ctx->ncell_tab.p, tab27.data(), sizeof(int32_t) * tab27.size(), cudaMemcpyHostToDevice,
                           ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
        ctx->ncell_grid = ctx->grid;
        ctx->ncell_single = true;
    }
    return ensure_cell_bufs(ctx, n, ctx->grid.ncells, dual, energy);
}

static tbmd_status ensure_scalars(tbmd_ctx *ctx)
{
    if (!ctx->scalars.p) {
        CK(ctx->scalars.ensure(64));
        CK(cudaMemsetAsync(ctx->scalars.p, 0, 64, ctx->stream));
    }
    return TBMD_OK;
}

// Prepare buffers for a forward (or adjoint) evaluation of n particles.
static tbmd_status prepare(tbmd_ctx *ctx, int64_t n, bool dual, bool energy)
{
    tbmd_status s = ensure_scalars(ctx);
    if (s != TBMD_OK) return s;
    if (is_p3bca_cut(ctx)) return ensure_cells(ctx, n, dual, energy);
    const int alg = dual ? TBMD_AUTA : (ctx->cfg.algorithm == TBMD_NATA ? TBMD_NATA : TBMD_AUTA);
    const int R = dual ? (mixed(ctx) ? 2 : 1) : sweep_R(ctx);
    return ensure_sweep(ctx, alg, n, R, dual);
}

__global__ void k_add_u64(unsigned long long *p, unsigned long long v) { *p += v; }

// Enqueue the triplet forces of n particles at `pos` into `out` (f, and H*d when dual).  The
// outputs are overwritten.  energy (may be NULL) and count accumulate on the device.
static tbmd_status enqueue_forces(tbmd_ctx *ctx, int64_t n, Pos pos, Out out, bool dual, double *energy,
                                  unsigned long long *count, cudaStream_t st, int *nl)
{
    const double nu = ctx->cfg.nu;
    const bool mx = mixed(ctx);
    if (n <= 0) return TBMD_OK;
    if (is_p3bca_cut(ctx)) {
        CellBufs &cb = ctx->cb;
        phase_mark(ctx, st, PH_CELLS, *nl);
        CK(launch_cell_build(n, pos, ctx->grid, ctx->gset, cb, dual, st, nl));
        phase_mark(ctx, st, PH_NEIGHBORS, *nl);
        CK(launch_neighbors(n, ctx->grid, ctx->gset, ctx->ncell_tab.as<int32_t>(), ctx->max_stage, cb, st));
        *nl += 1;
        CK(cudaMemsetAsync(cb.fs[0], 0, sizeof(double) * 3 * n, st));  // fs[0..2] are adjacent
        if (dual) CK(cudaMemsetAsync(cb.hs[0], 0, sizeof(double) * 3 * n, st));
        phase_mark(ctx, st, PH_TRIPLETS, *nl);
        CK(launch_p3bca(mx, dual, energy != nullptr, n, ctx->grid, ctx->gset, cb, nu, energy, count, ctx->plan, st));
        *nl += 1;
        phase_mark(ctx, st, PH_UPDATE, *nl);
        CK(launch_unsort(n, cb, out, dual, st));
        *nl += 1 + (dual ? 1 : 0);
        return TBMD_OK;
    }
    phase_mark(ctx, st, PH_TRIPLETS, *nl);
    SweepWork w = single_sweep(ctx);
    CK(cudaMemsetAsync(w.counter, 0, sizeof(unsigned int), st));
    if (ctx->cfg.algorithm == TBMD_NATA && !dual) {
        CK(launch_nata(mx, false, ctx->prefix_JB / 32, energy != nullptr, n, pos, out, energy, nu, w,
                       ctx->partial.as<double>(), ctx->sweep_grid, st));
        *nl += 1;
        phase_mark(ctx, st, PH_UPDATE, *nl);
        CK(launch_nata_reduce(false, n, ctx->nblocks, ctx->partial.as<double>(), out, st));
        *nl += 1;
    } else {
        CK(cudaMemsetAsync(out.fx, 0, sizeof(double) * n, st));
        CK(cudaMemsetAsync(out.fy, 0, sizeof(double) * n, st));
        CK(cudaMemsetAsync(out.fz, 0, sizeof(double) * n, st));
        if (dual) {
            CK(cudaMemsetAsync(out.hx, 0, sizeof(double) * n, st));
            CK(cudaMemsetAsync(out.hy, 0, sizeof(double) * n, st));
            CK(cudaMemsetAsync(out.hz, 0, sizeof(double) * n, st));
        }
        CK(launch_auta(mx, dual, ctx->prefix_JB / 32, energy != nullptr, n, pos, out, energy, nu, w, ctx->sweep_grid,
                       st));
        *nl += 1;
        phase_mark(ctx, st, PH_UPDATE, *nl);
    }
    if (count) {
        k_add_u64<<<1, 1, 0, st>>>(count, choose3(n));
        CK(cudaGetLastError());
        *nl += 1;
    }
    return TBMD_OK;
}

static Pos state_pos(tbmd_ctx *c) { return Pos{c->s[0], c->s[1], c->s[2], nullptr, nullptr, nullptr}; }
static Out state_out(tbmd_ctx *c) { return Out{c->s[10], c->s[11], c->s[12], nullptr, nullptr, nullptr}; }

// One Simulation::Start iteration: predictor, forces, update, per-step count.
static tbmd_status enqueue_step(tbmd_ctx *ctx, cudaStream_t st, int *nl)
{
    const int64_t n = ctx->n;
    double **s = ctx->s;
    if (is_p3bca_cut(ctx)) {
        // predictor + cell build, lists, triplets, then unsort + update + count in one kernel
        CellBufs &cb = ctx->cb;
        phase_mark(ctx, st, PH_CELLS, *nl);  // the predictor runs inside the cell build
        CK(launch_step_cells(n, s, ctx->cfg.dt, ctx->grid, cb, st, nl));
        if (ctx->pos_event) CK(cudaEventRecordWithFlags(ctx->pos_event, st, cudaEventRecordExternal));
        phase_mark(ctx, st, PH_NEIGHBORS, *nl);
        CK(launch_neighbors(n, ctx->grid, ctx->gset, ctx->ncell_tab.as<int32_t>(), ctx->max_stage, cb, st));
        *nl += 1;
        CK(cudaMemsetAsync(cb.fs[0], 0, sizeof(double) * 3 * n, st));  // fs[0..2] are adjacent
        phase_mark(ctx, st, PH_TRIPLETS, *nl);
        CK(launch_p3bca(mixed(ctx), false, false, n, ctx->grid, ctx->gset, cb, ctx->cfg.nu, nullptr, count_ptr(ctx),
                        ctx->plan, st));
        *nl += 1;
        phase_mark(ctx, st, PH_UPDATE, *nl);
        CK(launch_unsort_update(n, cb, s, ctx->cfg.dt, ctx->cfg.g, count_ptr(ctx),
                                ctx->step_counts.as<unsigned long long>(), step_ptr(ctx), st));
        *nl += 1;
        phase_mark(ctx, st, PH_END, *nl);
        return TBMD_OK;
    }
    phase_mark(ctx, st, PH_PREDICTOR, *nl);
    CK(launch_predictor(n, s[0], s[1], s[2], s[3], s[4], s[5], s[6], ctx->cfg.dt, st));
    *nl += 1;
    if (ctx->pos_event) CK(cudaEventRecordWithFlags(ctx->pos_event, st, cudaEventRecordExternal));
    // forces of the step's count go to count_cur; the no-cutoff count C(n,3) is added by k_add_u64
    tbmd_status r = enqueue_forces(ctx, n, state_pos(ctx), state_out(ctx), false, nullptr, count_ptr(ctx), st, nl);
    if (r != TBMD_OK) return r;
    CK(launch_update(n, s[3], s[4], s[5], s[6], s[7], s[8], s[10], s[11], s[12], s[9], ctx->cfg.dt, ctx->cfg.g[0],
                     ctx->cfg.g[1], ctx->cfg.g[2], st));
    CK(launch_record_count(count_ptr(ctx), ctx->step_counts.as<unsigned long long>(), step_ptr(ctx), 0ull, st));
    *nl += 2;
    phase_mark(ctx, st, PH_END, *nl);
    return TBMD_OK;
}

static tbmd_status build_graph(tbmd_ctx *ctx)
{
    invalidate_graph(ctx);
    cudaGraph_t g = nullptr;
    int nl = 0;
    CK(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
    tbmd_status r = enqueue_step(ctx, ctx->stream, &nl);
    cudaError_t e = cudaStreamEndCapture(ctx->stream, &g);
    if (r != TBMD_OK) {
        if (g) cudaGraphDestroy(g);
        return r;
    }
    if (e != cudaSuccess) return fail(ctx, TBMD_CUDA_ERROR, "graph capture: %s", cudaGetErrorString(e));
    e = cudaGraphInstantiate(&ctx->gexec, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return fail(ctx, TBMD_CUDA_ERROR, "graph instantiate: %s", cudaGetErrorString(e));
    ctx->graph_valid = true;
    ctx->graph_launches_per_step = nl;
    return TBMD_OK;
}

static tbmd_status check_device(tbmd_ctx *ctx)
{
    CK(cudaSetDevice(ctx->device));
    return TBMD_OK;
}

// Copies of particle columns k0..k1-1 (n doubles each) between caller host arrays and device
// columns.  Columns that lie back to back on both sides (the caller's arrays consecutive in memory,
// like the device state) go in one copy per run: one large copy is about 20 % faster than several
// 1 MB ones.  Null host entries and column `skip` are left out.
static cudaError_t copy_columns(double *const *host, double *const *dev, int k0, int k1, int64_t n,
                                cudaMemcpyKind kind, cudaStream_t st, int skip = -1)
{
    const size_t col = sizeof(double) * (size_t)n;
    for (int k = k0; k < k1;) {
        if (!host[k] || k == skip) {
            ++k;
            continue;
        }
        int e = k + 1;
        while (e < k1 && e != skip && host[e] == host[e - 1] + n && dev[e] == dev[e - 1] + n) ++e;
        const size_t bytes = col * (size_t)(e - k);
        const cudaError_t r = kind == cudaMemcpyHostToDevice
                                  ? cudaMemcpyAsync(dev[k], host[k], bytes, kind, st)
                                  : cudaMemcpyAsync(host[k], dev[k], bytes, kind, st);
        if (r != cudaSuccess) return r;
        k = e;
    }
    return cudaSuccess;
}

// ---------------------------------------------------------------------------------------------
// C ABI

extern "C" {

void tbmd_config_init(tbmd_config *cfg)
{
    if (!cfg) return;
    std::memset(cfg, 0, sizeof *cfg);
    cfg->algorithm = TBMD_AUTA;
    cfg->precision = TBMD_FP64;
    cfg->nu = 1.0;
    cfg->use_graph = 1;
}

int32_t tbmd_abi_version(void) { return TBMD_ABI_VERSION; }

const char *tbmd_status_string(tbmd_status s)
{
    switch (s) {
        case TBMD_OK: return "ok";
        case TBMD_INVALID_ARG: return "invalid argument";
        case TBMD_BAD_INPUT: return "bad input";
        case TBMD_NOT_READY: return "not ready";
        case TBMD_CAPACITY_RETRY: return "neighbour capacity exceeded";
        case TBMD_CUDA_ERROR: return "CUDA error";
        case TBMD_TIMEOUT: return "device wait timed out";
        case TBMD_NO_DEVICE: return "no sm_100 CUDA device";
        case TBMD_TOO_LARGE: return "n above the allocation-free limit";
        case TBMD_RANK_LAYOUT: return "the reference's run on that many ranks would stop";
    }
    return "unknown status";
}

const char *tbmd_last_error(const tbmd_ctx *ctx) { return ctx ? ctx->err.c_str() : "null context"; }

tbmd_status tbmd_create(const tbmd_config *cfg, tbmd_ctx **out)
{
    if (!cfg || !out) return TBMD_INVALID_ARG;
    *out = nullptr;
    if (cfg->algorithm < 0 || cfg->algorithm > 2 || cfg->precision < 0 || cfg->precision > 1)
        return TBMD_INVALID_ARG;
    if (!std::isfinite(cfg->dt) || !std::isfinite(cfg->nu) || !std::isfinite(cfg->cutoff) ||
        !std::isfinite(cfg->g[0]) || !std::isfinite(cfg->g[1]) || !std::isfinite(cfg->g[2]))
        return TBMD_INVALID_ARG;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0 || cfg->device < 0 || cfg->device >= ndev) {
        cudaGetLastError();
        return TBMD_NO_DEVICE;
    }
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, cfg->device) != cudaSuccess || prop.major != 10) return TBMD_NO_DEVICE;
    tbmd_ctx *ctx = new (std::nothrow) tbmd_ctx();
    if (!ctx) return TBMD_INVALID_ARG;
    ctx->cfg = *cfg;
    ctx->device = cfg->device;
    if (cudaSetDevice(ctx->device) != cudaSuccess) {
        delete ctx;
        return TBMD_NO_DEVICE;
    }
    if (cfg->stream) {
        ctx->stream = (cudaStream_t)cfg->stream;
    } else {
        if (cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess) {
            delete ctx;
            return TBMD_CUDA_ERROR;
        }
        ctx->own_stream = true;
    }
    if (ensure_scalars(ctx) != TBMD_OK) {
        tbmd_destroy(ctx);
        return TBMD_CUDA_ERROR;
    }
    ctx->tuning = "{}";
    *out = ctx;
    return TBMD_OK;
}

void tbmd_destroy(tbmd_ctx *ctx)
{
    if (!ctx) return;
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    invalidate_graph(ctx);
    for (auto &m : ctx->marks) cudaEventDestroy(m.second);
    for (cudaEvent_t e : ctx->event_pool) cudaEventDestroy(e);
    for (DevBuf *b : {&ctx->state, &ctx->snapshot, &ctx->scalars, &ctx->step_counts, &ctx->prefix, &ctx->partial,
                      &ctx->cell_n, &ctx->cell_c, &ctx->nbr_buf, &ctx->dirs, &ctx->hvp, &ctx->gset_single,
                      &ctx->sweep_sys, &ctx->bpos, &ctx->bout, &ctx->bsys, &ctx->bprefix, &ctx->ncell_tab,
                      &ctx->staging, &ctx->long_buf, &ctx->gen_buf, &ctx->bext})
        b->release();
    if (ctx->hpin) cudaFreeHost(ctx->hpin);
    if (ctx->copy_stream) {
        cudaStreamSynchronize(ctx->copy_stream);
        cudaStreamDestroy(ctx->copy_stream);
    }
    if (ctx->hstep) cudaFreeHost(ctx->hstep);
    if (ctx->pos_event) cudaEventDestroy(ctx->pos_event);
    if (ctx->own_stream && ctx->stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
}

int64_t tbmd_num_particles(const tbmd_ctx *ctx) { return ctx ? ctx->n : 0; }
uint64_t tbmd_kernel_launches(const tbmd_ctx *ctx) { return ctx ? ctx->launches : 0; }

// The incoming particle arrays are in ctx->staging (x y z vx vy vz ax ay az m, n each): check them on
// the device (non-finite values, masses <= 0, extremes of x, y, z for the domain) and make them the
// context's state.  The state is untouched when the check fails.  host_bad flags arrays that the
// caller checked on the host instead (bit k: array k holds a non-finite value).
static tbmd_status commit_staging(tbmd_ctx *ctx, int64_t n, const int32_t *id, unsigned int host_bad = 0)
{
    const size_t arr_bytes = sizeof(double) * 10 * (size_t)n;
    double *stg = ctx->staging.as<double>();
    ValidateResult *vr = (ValidateResult *)(ctx->staging.as<char>() + arr_bytes);
    int sms = 0;
    CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device));
    CK(launch_validate(n, stg, vr, sms * 4, ctx->stream));
    ctx->launches += 1;
    ValidateResult h{};
    CK(cudaMemcpyAsync(&h, vr, sizeof h, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));  // the caller's arrays are free again from here
    h.bad_arrays |= host_bad;
    if (h.bad_arrays) {
        int k = 0;
        while (!(h.bad_arrays & (1u << k))) ++k;
        return fail(ctx, TBMD_BAD_INPUT, "non-finite value in particle array %d", k);
    }
    if (h.bad_mass != ~0ull)
        return fail(ctx, TBMD_BAD_INPUT, "mass of particle %lld is not positive", (long long)h.bad_mass);
    if (ctx->n != n) invalidate_graph(ctx);
    CK(ctx->state.ensure(sizeof(double) * 13 * (size_t)n));
    for (int k = 0; k < 13; ++k) ctx->s[k] = ctx->state.as<double>() + (size_t)k * n;
    CK(cudaMemcpyAsync(ctx->s[0], stg, arr_bytes, cudaMemcpyDeviceToDevice, ctx->stream));
    CK(cudaMemsetAsync(ctx->s[10], 0, sizeof(double) * 3 * n, ctx->stream));
    ctx->id.resize(n);
    if (id) {
        std::memcpy(ctx->id.data(), id, sizeof(int32_t) * n);
    } else {
        for (int64_t i = 0; i < n; ++i) ctx->id[i] = (int32_t)i;
    }
    ctx->n = n;
    if (ctx->cfg.algorithm == TBMD_P3BCA) {
        // RegularGridDecomposition::getDomainMinMax + Init, from these (initial) positions
        for (int d = 0; d < 3; ++d) {
            const double a = key_to_double(h.min_key[d]) - 0.0001, b = key_to_double(h.max_key[d]) + 0.0001;
            ctx->lo[d] = a;
            ctx->L[d] = std::fabs(b - a);
        }
        ctx->domain_set = true;
        ctx->cap = 0;
    }
    return TBMD_OK;
}

static cudaError_t ensure_staging(tbmd_ctx *ctx, int64_t n)
{
    return ctx->staging.ensure(sizeof(double) * 10 * (size_t)n + sizeof(ValidateResult) + 256);
}

// tbmd_set_particles, and the input half of tbmd_step_host.  With `step_follows` the arrays ay and az
// are not copied: a step reads ax alone (the predictor applies ax on all three axes,
// structs.hpp:40-55) and the update overwrites all three, so their values cannot reach any result.
// They are still checked, on the host while the other arrays travel, so the call fails on the same
// inputs as tbmd_set_particles; the state holds zeros there until the first step.
static tbmd_status upload_particles(tbmd_ctx *ctx, int64_t n, const int32_t *id, const double *const src[10],
                                    bool step_follows)
{
    if (n < 1 || n > (int64_t)INT32_MAX / 2) return fail(ctx, TBMD_INVALID_ARG, "n = %lld out of range", (long long)n);
    for (int k = 0; k < 10; ++k)
        if (!src[k]) return fail(ctx, TBMD_INVALID_ARG, "null particle array %d", k);
    tbmd_status st = check_device(ctx);
    if (st != TBMD_OK) return st;
    CK(cudaStreamSynchronize(ctx->stream));
    CK(ensure_staging(ctx, n));
    double *stg = ctx->staging.as<double>();
    double *dcol[10], *hcol[10];
    for (int k = 0; k < 10; ++k) {
        dcol[k] = stg + (size_t)k * n;
        hcol[k] = const_cast<double *>(src[k]);
    }
    unsigned int host_bad = 0;
    if (step_follows) {
        hcol[7] = hcol[8] = nullptr;  // copy_columns leaves null host entries out
        CK(copy_columns(hcol, dcol, 0, 10, n, cudaMemcpyHostToDevice, ctx->stream));
        CK(cudaMemsetAsync(dcol[7], 0, sizeof(double) * 2 * (size_t)n, ctx->stream));  // ay, az adjacent
        for (int k = 7; k <= 8; ++k) {
            // branch-free, so the compiler vectorises it: |v| <= DBL_MAX is false for inf and NaN
            const double *a = src[k];
            int bad = 0;
            for (int64_t i = 0; i < n; ++i) bad |= !(std::fabs(a[i]) <= DBL_MAX);
            if (bad) host_bad |= 1u << k;
        }
    } else {
        CK(copy_columns(hcol, dcol, 0, 10, n, cudaMemcpyHostToDevice, ctx->stream));
    }
    return commit_staging(ctx, n, id, host_bad);
}

tbmd_status tbmd_set_particles(tbmd_ctx *ctx, int64_t n, const int32_t *id, const double *x, const double *y,
                               const double *z, const double *vx, const double *vy, const double *vz,
                               const double *ax, const double *ay, const double *az, const double *m)
{
    if (!ctx) return TBMD_INVALID_ARG;
    const double *src[10] = {x, y, z, vx, vy, vz, ax, ay, az, m};
    return upload_particles(ctx, n, id, src, false);
}

void tbmd_generator_init(tbmd_generator *g)
{
    if (!g) return;
    std::memset(g, 0, sizeof *g);
    g->kind = TBMD_GEN_UNIFORM;
    for (int d = 0; d < 3; ++d) g->box[d] = 10.0;
    g->mass = 1.0;
    g->seed0 = 926762934u;
    g->seed1 = 89347587u;
    g->n_clusters = 1;
    g->mean = 0.0;
    g->stddev = 1.0;
    g->csv_digits = 6;
}

// printf("%.6g") read back by strtod, on the host (the constant columns)
static double csv6(double v)
{
    char buf[64];
    std::snprintf(buf, sizeof buf, "%.6g", v);
    return std::strtod(buf, nullptr);
}

tbmd_status tbmd_generate_particles(tbmd_ctx *ctx, const tbmd_generator *g)
{
    if (!ctx) return TBMD_INVALID_ARG;
    if (!g) return fail(ctx, TBMD_INVALID_ARG, "null generator");
    if (g->kind != TBMD_GEN_UNIFORM && g->kind != TBMD_GEN_CLUSTERED_GAUSS)
        return fail(ctx, TBMD_INVALID_ARG, "unknown generator kind %d", g->kind);
    if (g->csv_digits != 0 && g->csv_digits != 6) return fail(ctx, TBMD_INVALID_ARG, "csv_digits must be 0 or 6");
    for (int d = 0; d < 3; ++d)
        if (!std::isfinite(g->box[d]) || !std::isfinite(g->corner[d]) || !std::isfinite(g->velocity[d]))
            return fail(ctx, TBMD_INVALID_ARG, "box, corner and velocity must be finite");
    if (!(g->mass > 0) || !std::isfinite(g->mass)) return fail(ctx, TBMD_INVALID_ARG, "mass must be positive");
    const bool clustered = g->kind == TBMD_GEN_CLUSTERED_GAUSS;
    if (clustered && (g->n_clusters < 1 || !std::isfinite(g->mean) || !std::isfinite(g->stddev)))
        return fail(ctx, TBMD_INVALID_ARG, "clustered generator needs n_clusters >= 1 and a finite mean/stddev");
    const int64_t per = clustered ? g->n / g->n_clusters : 1;
    const int64_t n = clustered ? per * g->n_clusters : g->n;  // ClusteredGaussGenerator.cpp:40
    if (n < 1 || n > (int64_t)INT32_MAX / 2)
        return fail(ctx, TBMD_INVALID_ARG, "n = %lld out of range", (long long)n);
    tbmd_status st = check_device(ctx);
    if (st != TBMD_OK) return st;
    CK(cudaStreamSynchronize(ctx->stream));
    CK(ensure_staging(ctx, n));
    double *stg = ctx->staging.as<double>();
    double *X = stg, *Y = stg + n, *Z = stg + 2 * n;
    cudaStream_t sm = ctx->stream;
    if (!clustered) {
        CK(ctx->gen_buf.ensure(sizeof(uint32_t) * 6 * (size_t)n));
        CK(launch_mt19937(g->seed0, 6 * n, ctx->gen_buf.as<uint32_t>(), sm));
        CK(launch_uniform_positions(n, ctx->gen_buf.as<uint32_t>(), g->corner, g->box, X, Y, Z, sm));
        ctx->launches += 2;
    } else {
        // cluster centres: uniform draws from mt19937(seed1); then the Gaussian offsets in passes
        const int64_t ncl = g->n_clusters;
        const int64_t attempts = polar_attempts_per_pass();
        const size_t cen_bytes = ((sizeof(double) * 3 * ncl + 255) / 256) * 256;
        const size_t word_bytes = ((sizeof(uint32_t) * 6 * ncl + 255) / 256) * 256;
        CK(ctx->gen_buf.ensure(cen_bytes + word_bytes + polar_scratch_bytes(attempts)));
        char *gb = ctx->gen_buf.as<char>();
        double *cen = (double *)gb;
        uint32_t *words = (uint32_t *)(gb + cen_bytes);
        void *scratch = gb + cen_bytes + word_bytes;
        CK(launch_mt19937(g->seed1, 6 * ncl, words, sm));
        CK(launch_uniform_positions(ncl, words, g->corner, g->box, cen, cen + ncl, cen + 2 * ncl, sm));
        ctx->launches += 2;
        const double *centres[3] = {cen, cen + ncl, cen + 2 * ncl};
        const uint64_t m31 = 2147483647ull, x0 = (uint64_t)g->seed0 % m31 == 0 ? 1 : (uint64_t)g->seed0 % m31;
        const unsigned long long G = 3ull * (unsigned long long)((n + 1) / 2);  // particle pairs x 3 axes
        unsigned long long done = 0, t0 = 0;
        int passes = 0;
        while (done < G) {
            if (++passes > 64) return fail(ctx, TBMD_CUDA_ERROR, "Gaussian generator did not converge");
            int64_t T = (int64_t)((double)(G - done) * 1.35) + 4096;
            if (T > attempts) T = attempts;
            unsigned long long end = 0;
            CK(launch_polar_pass(x0, t0, T, done, G, n, per, centres, g->mean, g->stddev, X, Y, Z, scratch, &end,
                                 sm));
            CK(cudaStreamSynchronize(sm));
            ctx->launches += 3;
            done = end;
            t0 += (unsigned long long)T;
        }
    }
    if (g->csv_digits == 6) {
        CK(launch_round_sig6(3 * n, stg, sm));
        ctx->launches += 1;
    }
    const double vel[3] = {g->csv_digits == 6 ? csv6(g->velocity[0]) : g->velocity[0],
                           g->csv_digits == 6 ? csv6(g->velocity[1]) : g->velocity[1],
                           g->csv_digits == 6 ? csv6(g->velocity[2]) : g->velocity[2]};
    const double mass = g->csv_digits == 6 ? csv6(g->mass) : g->mass;
    for (int d = 0; d < 3; ++d) CK(launch_fill(n, vel[d], stg + (3 + d) * n, sm));
    CK(cudaMemsetAsync(stg + 6 * n, 0, sizeof(double) * 3 * n, sm));
    CK(launch_fill(n, mass, stg + 9 * n, sm));
    ctx->launches += 4;
    return commit_staging(ctx, n, nullptr);
}

tbmd_status tbmd_set_domain(tbmd_ctx *ctx, const double *L, const double *lo)
{
    if (!ctx || !L || !lo) return TBMD_INVALID_ARG;
    for (int d = 0; d < 3; ++d)
        if (!(L[d] > 0) || !std::isfinite(L[d]) || !std::isfinite(lo[d]))
            return fail(ctx, TBMD_INVALID_ARG, "bad domain on axis %d", d);
    for (int d = 0; d < 3; ++d) {
        ctx->L[d] = L[d];
        ctx->lo[d] = lo[d];
    }
    ctx->domain_set = true;
    ctx->cap = 0;
    invalidate_graph(ctx);
    return TBMD_OK;
}

tbmd_status tbmd_get_particles(tbmd_ctx *ctx, int32_t *id, double *x, double *y, double *z, double *vx, double *vy,
                               double *vz, double *ax, double *ay, double *az, double *m, double *fx, double *fy,
                               double *fz)
{
    if (!ctx) return TBMD_INVALID_ARG;
    if (ctx->n == 0) return fail(ctx, TBMD_NOT_READY, "no particles set");
    tbmd_status st = check_device(ctx);
    if (st != TBMD_OK) return st;
    double *dst[13] = {x, y, z, vx, vy, vz, ax, ay, az, m, fx, fy, fz};
    CK(copy_columns(dst, ctx->s, 0, 13, ctx->n, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    if (id) std::memcpy(id, ctx->id.data(), sizeof(int32_t) * ctx->n);
    return TBMD_OK;
}

// Grow the neighbour capacity after an overflow; true if a retry is worthwhile.
// Overflow flags of the P3BCA lists: the longest list seen and the chunk-pair items requested.
struct CapSeen {
    int32_t max_count;
    uint32_t pad[3];
    uint32_t long_max;
};
static_assert(sizeof(CapSeen) == 20, "scalars 28..48");

static cudaError_t reset_cap_flags(tbmd_ctx *ctx, cudaStream_t st)
{
    cudaError_t e = cudaMemsetAsync(ctx->scalars.as<char>() + 28, 0, 4, st);
    if (e != cudaSuccess) return e;
    return cudaMemsetAsync(ctx->scalars.as<char>() + 44, 0, 4, st);
}

static cudaError_t read_cap_flags(tbmd_ctx *ctx, cudaStream_t st, CapSeen *seen)
{
    return cudaMemcpyAsync(seen, ctx->scalars.as<char>() + 28, sizeof(CapSeen), cudaMemcpyDeviceToHost, st);
}

// Grow the list capacity or the chunk-pair item capacity after an overflow; true if a retry is
// needed.
static bool grow_caps(tbmd_ctx *ctx, const CapSeen &seen)
{
    bool grew = false;
    if (seen.max_count > ctx->cap) {
        int want = (int)((double)seen.max_count * 1.25) + 32;
        ctx->cap = (want + 31) / 32 * 32;
        grew = true;
    }
    if ((int64_t)seen.long_max > (int64_t)ctx->long_cap) {
        ctx->long_cap = (int)((double)seen.long_max * 1.25) + 1024;
        grew = true;
    }
    if (grew) invalidate_graph(ctx);
    return grew;
}

// Host arrays that receive the state after the steps (tbmd_step_host); NULL entries are skipped.
struct HostOut {
    double *dst[13];  // x y z vx vy vz ax ay az m fx fy fz
};

// The steps of tbmd_step, with the capacity retry.  With `ho`, the state after the last step is
// also copied to the host: the positions (final once the last step's predictor has run) on the copy
// stream while the step's forces are computed, velocities, accelerations and forces after the step
// on the context stream, before the one synchronisation of the attempt.  A retried attempt issues
// its copies again, so the last (complete) attempt's values are the ones left in the host arrays.
static tbmd_status run_steps(tbmd_ctx *ctx, int32_t iterations, uint64_t *counts, const HostOut *ho,
                             const std::function<void()> &while_running = {})
{
    if (ctx->step_counts_cap < iterations) {
        CK(cudaStreamSynchronize(ctx->stream));
        CK(ctx->step_counts.ensure(sizeof(unsigned long long) * iterations));
        ctx->step_counts_cap = iterations;
        invalidate_graph(ctx);
    }
    const bool cut = is_p3bca_cut(ctx);
    const int64_t n = ctx->n;
    const size_t hbytes = sizeof(CapSeen) + 12 + sizeof(unsigned long long) * (size_t)iterations;
    if (ctx->hstep_bytes < hbytes) {
        CK(cudaStreamSynchronize(ctx->stream));
        if (ctx->hstep) CK(cudaFreeHost(ctx->hstep));
        ctx->hstep = nullptr;
        ctx->hstep_bytes = 0;
        CK(cudaHostAlloc(&ctx->hstep, hbytes, cudaHostAllocDefault));
        ctx->hstep_bytes = hbytes;
    }
    CapSeen *hseen = (CapSeen *)ctx->hstep;
    unsigned long long *hcounts = (unsigned long long *)((char *)ctx->hstep + 32);  // 8-byte aligned
    tbmd_status st = TBMD_OK;
    for (int attempt = 0; attempt < 4; ++attempt) {
        void *before[5] = {ctx->state.p, ctx->nbr_buf.p, ctx->cell_n.p, ctx->prefix.p, ctx->long_buf.p};
        st = prepare(ctx, n, false, false);
        if (st != TBMD_OK) return st;
        void *after[5] = {ctx->state.p, ctx->nbr_buf.p, ctx->cell_n.p, ctx->prefix.p, ctx->long_buf.p};
        if (std::memcmp(before, after, sizeof before)) invalidate_graph(ctx);
        CK(cudaMemsetAsync(ctx->scalars.as<char>() + 8, 0, 56, ctx->stream));
        if (cut) {
            CK(ctx->snapshot.ensure(sizeof(double) * 9 * (size_t)n));
            CK(cudaMemcpyAsync(ctx->snapshot.p, ctx->s[0], sizeof(double) * 9 * n, cudaMemcpyDeviceToDevice,
                               ctx->stream));
        }
        if (ctx->cfg.use_graph && !ctx->profiling) {
            if (!ctx->graph_valid) {
                st = build_graph(ctx);
                if (st != TBMD_OK) return st;
            }
            for (int it = 0; it < iterations; ++it) CK(cudaGraphLaunch(ctx->gexec, ctx->stream));
            ctx->launches += (uint64_t)ctx->graph_launches_per_step * iterations;
        } else {
            for (int it = 0; it < iterations; ++it) {
                int nl = 0;
                st = enqueue_step(ctx, ctx->stream, &nl);
                if (st != TBMD_OK) return st;
                ctx->launches += nl;
            }
        }
        if (ho) {
            // the last recorded position event belongs to the last step just enqueued
            CK(cudaStreamWaitEvent(ctx->copy_stream, ctx->pos_event, 0));
            CK(copy_columns(ho->dst, ctx->s, 0, 3, n, cudaMemcpyDeviceToHost, ctx->copy_stream));
            CK(copy_columns(ho->dst, ctx->s, 3, 13, n, cudaMemcpyDeviceToHost, ctx->stream, 9));
        }
        CK(cudaMemcpyAsync(hcounts, ctx->step_counts.p, sizeof(unsigned long long) * iterations,
                           cudaMemcpyDeviceToHost, ctx->stream));
        CK(read_cap_flags(ctx, ctx->stream, hseen));
        if (attempt == 0 && while_running) while_running();  // host work that overlaps the device
        CK(cudaStreamSynchronize(ctx->stream));
        if (ho) CK(cudaStreamSynchronize(ctx->copy_stream));
        const CapSeen seen = *hseen;
        phase_resolve(ctx);
        if (cut && grow_caps(ctx, seen)) {
            CK(cudaMemcpyAsync(ctx->s[0], ctx->snapshot.p, sizeof(double) * 9 * n, cudaMemcpyDeviceToDevice,
                               ctx->stream));
            continue;
        }
        if (cut) {
            ctx->cap_used = ctx->cap;
            ctx->cap_used_n = n;
        }
        if (counts)
            for (int it = 0; it < iterations; ++it) counts[it] = hcounts[it];
        return TBMD_OK;
    }
    return fail(ctx, TBMD_CAPACITY_RETRY, "neighbour capacity still exceeded after retries (cap %d)", ctx->cap);
}

tbmd_status tbmd_step(tbmd_ctx *ctx, int32_t iterations, uint64_t *counts)
{
    if (!ctx) return TBMD_INVALID_ARG;
    if (iterations < 0) return fail(ctx, TBMD_INVALID_ARG, "iterations < 0");
    if (ctx->n == 0) return fail(ctx, TBMD_NOT_READY, "no particles set");
    if (iterations == 0) return TBMD_OK;
    tbmd_status st = check_device(ctx);
    if (st != TBMD_OK) return st;
    return run_steps(ctx, iterations, counts, nullptr);
}

tbmd_status tbmd_step_host(tbmd_ctx *ctx, int64_t n, const int32_t *id, const double *x, const double *y,
                           const double *z, const double *vx, const double *vy, const double *vz, const double *ax,
                           const double *ay, const double *az, const double *m, int32_t iterations,
                           uint64_t *triplets_per_step, int32_t *id_out, double *x_out, double *y_out, double *z_out,
                           double *vx_out, double *vy_out, double *vz_out, double *ax_out, double *ay_out,
                           double *az_out, double *m_out, double *fx_out, double *fy_out, double *fz_out)
{
    if (!ctx) return TBMD_INVALID_ARG;
    if (iterations < 0) return fail(ctx, TBMD_INVALID_ARG, "iterations < 0");
    tbmd_status st = check_device(ctx);
    if (st != TBMD_OK) return st;
    if (!ctx->copy_stream) {
        CK(cudaStreamCreateWithFlags(&ctx->copy_stream, cudaStreamNonBlocking));
        CK(cudaEventCreateWithFlags(&ctx->pos_event, cudaEventDisableTiming));
        invalidate_graph(ctx);  // the step graph gains the position event
    }
    const double *src[10] = {x, y, z, vx, vy, vz, ax, ay, az, m};
    st = upload_particles(ctx, n, id, src, iterations > 0);
    if (st != TBMD_OK) return st;
    HostOut ho{{x_out, y_out, z_out, vx_out, vy_out, vz_out, ax_out, ay_out, az_out, m_out, fx_out, fy_out, fz_out}};
    // masses (no step changes them) and IDs come from the inputs, on the host, while the GPU works
    auto host_columns = [&]() {
        if (m_out && m_out != m) std::memmove(m_out, m, sizeof(double) * (size_t)n);
        if (id_out && id_out != ctx->id.data()) std::memcpy(id_out, ctx->id.data(), sizeof(int32_t) * (size_t)n);
    };
    if (iterations == 0) {
        CK(copy_columns(ho.dst, ctx->s, 0, 13, n, cudaMemcpyDeviceToHost, ctx->stream, 9));
        host_columns();
        CK(cudaStreamSynchronize(ctx->stream));
        return TBMD_OK;
    }
    // the host copies run while the first attempt's device work is in flight
    return run_steps(ctx, iterations, triplets_per_step, &ho, host_columns);
}

// Forward (dual = false) or adjoint (dual = true) evaluation with capacity retry, on ctx's state
// or on caller device pointers.
static tbmd_status evaluate(tbmd_ctx *ctx, int64_t n, Pos pos, Out out, bool dual, double *energy,
                            unsigned long long *count, cudaStream_t st)
{
    for (int attempt = 0; attempt < 4; ++attempt) {
        tbmd_status s = prepare(ctx, n, dual, energy != nullptr);
        if (s != TBMD_OK) return s;
        CK(reset_cap_flags(ctx, st));
        if (energy) CK(cudaMemsetAsync(energy, 0, sizeof(double), st));
        if (count) CK(cudaMemsetAsync(count, 0, sizeof(unsigned long long), st));
        int nl = 0;
        s = enqueue_forces(ctx, n, pos, out, dual, energy, count, st, &nl);
        if (s != TBMD_OK) return s;
        phase_mark(ctx, st, PH_END, nl);
        ctx->launches += nl;
        if (ctx->profiling) {
            CK(cudaStreamSynchronize(st));
            phase_resolve(ctx);
        }
        if (!is_p3bca_cut(ctx)) return TBMD_OK;
        CapSeen seen{};
        CK(read_cap_flags(ctx, st, &seen));
        CK(cudaStreamSynchronize(st));
        if (!grow_caps(ctx, seen)) {
            ctx->cap_used = ctx->cap;
            ctx->cap_used_n = n;
            return TBMD_OK;
        }
    }
    return fail(ctx, TBMD_CAPACITY_RETRY, "neighbour capacity still exceeded after retries (cap %d)", ctx->cap);
}

tbmd_status tbmd_forces(tbmd_ctx *ctx, double *fx, double *fy, double *fz, double *energy, uint64_t *triplets)
{
    if (!ctx) return TBMD_INVALID_ARG;
    if (ctx->n == 0) return fail(ctx, TBMD_NOT_READY, "no particles set");
    tbmd_status st = check_device(ctx);
    if (st != TBMD_OK) return st;
    st = ensure_scalars(ctx);
    if (st != TBMD_OK) return st;
    st = evaluate(ctx, ctx->n, state_pos(ctx), state_out(ctx), false, energy_ptr(ctx), count_ptr(ctx), ctx->stream);
    if (st != TBMD_OK) return st;
    double e = 0;
    unsigned long long c = 0;
    const int64_t n = ctx->n;
    if (fx) CK(cudaMemcpyAsync(fx, ctx->s[10], sizeof(double) * n, cudaMemcpyDeviceToHost, ctx->stream));
    if (fy) CK(cudaMemcpyAsync(fy, ctx->s[11], sizeof(double) * n, cudaMemcpyDeviceToHost, ctx->stream));
    if (fz) CK(cudaMemcpyAsync(fz, ctx->s[12], sizeof(double) * n, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaMemcpyAsync(&e, energy_ptr(ctx), sizeof e, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaMemcpyAsync(&c, count_ptr(ctx), sizeof c, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    if (energy) *energy = e;
    if (triplets) *triplets = c;
    return TBMD_OK;
}

tbmd_status tbmd_forces_device(tbmd_ctx *ctx, int64_t n, const double *x, const double *y, const double *z,
                               double *fx, double *fy, double *fz, double *energy, uint64_t *triplets, void *stream)
{
    if (!ctx || !x || !y || !z || !fx || !fy || !fz) return TBMD_INVALID_ARG;
    if (n < 1) return fail(ctx, TBMD_INVALID_ARG, "n < 1");
    tbmd_status st = check_device(ctx);
    if (st != TBMD_OK) return st;
    cudaStream_t s = stream ? (cudaStream_t)stream : ctx->stream;
    return evaluate(ctx, n, Pos{x, y, z, nullptr, nullptr, nullptr}, Out{fx, fy, fz, nullptr, nullptr, nullptr}, false,
                    energy, (unsigned long long *)triplets, s);
}

tbmd_status tbmd_adjoint_device(tbmd_ctx *ctx, int64_t n, const double *x, const double *y, const double *z,
                                const double *gfx, const double *gfy, const double *gfz, const double *g_energy,
                                double *fx, double *fy, double *fz, double *energy, double *gx, double *gy, double *gz,
                                void *stream)
{
    (void)g_energy;
    if (!ctx || !x || !y || !z || !gfx || !gfy || !gfz || !fx || !fy || !fz || !gx || !gy || !gz)
        return TBMD_INVALID_ARG;
    if (n < 1) return fail(ctx, TBMD_INVALID_ARG, "n < 1");
    tbmd_status st = check_device(ctx);
    if (st != TBMD_OK) return st;
    cudaStream_t s = stream ? (cudaStream_t)stream : ctx->stream;
    // gx receives H * gf; the caller adds g_energy * f (a device-side axpy it already owns).
    return evaluate(ctx, n, Pos{x, y, z, gfx, gfy, gfz}, Out{fx, fy, fz, gx, gy, gz}, true, energy, nullptr, s);
}

tbmd_status tbmd_adjoint(tbmd_ctx *ctx, const double *gfx, const double *gfy, const double *gfz, double g_energy,
                         double *gx, double *gy, double *gz, double *g_nu)
{
    if (!ctx || !gfx || !gfy || !gfz) return TBMD_INVALID_ARG;
    if (ctx->n == 0) return fail(ctx, TBMD_NOT_READY, "no particles set");
    if (!std::isfinite(g_energy)) return fail(ctx, TBMD_INVALID_ARG, "g_energy not finite");
    tbmd_status st = check_device(ctx);
    if (st != TBMD_OK) return st;
    st = ensure_scalars(ctx);
    if (st != TBMD_OK) return st;
    const int64_t n = ctx->n;
    CK(ctx->dirs.ensure(sizeof(double) * 3 * (size_t)n));
    CK(ctx->hvp.ensure(sizeof(double) * 3 * (size_t)n));
    double *d = ctx->dirs.as<double>(), *h = ctx->hvp.as<double>();
    CK(cudaMemcpyAsync(d, gfx, sizeof(double) * n, cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(d + n, gfy, sizeof(double) * n, cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(d + 2 * n, gfz, sizeof(double) * n, cudaMemcpyHostToDevice, ctx->stream));
    const double nu = ctx->cfg.nu;
    if (nu == 0.0) ctx->cfg.nu = 1.0;  // f and E are linear in nu: evaluate the nu = 1 parts
    st = evaluate(ctx, n, Pos{ctx->s[0], ctx->s[1], ctx->s[2], d, d + n, d + 2 * n},
                  Out{ctx->s[10], ctx->s[11], ctx->s[12], h, h + n, h + 2 * n}, true, energy_ptr(ctx), nullptr,
                  ctx->stream);
    ctx->cfg.nu = nu;
    if (st != TBMD_OK) return st;
    std::vector<double> f(3 * n), hv(3 * n);
    double e = 0;
    for (int k = 0; k < 3; ++k)
        CK(cudaMemcpyAsync(f.data() + k * n, ctx->s[10 + k], sizeof(double) * n, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaMemcpyAsync(hv.data(), h, sizeof(double) * 3 * n, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaMemcpyAsync(&e, energy_ptr(ctx), sizeof e, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    const double scale = nu == 0.0 ? 0.0 : 1.0;  // with nu = 0 the true f, E and H are zero
    const double *g3[3] = {gfx, gfy, gfz};
    double *o3[3] = {gx, gy, gz};
    double dot = 0.0;
    for (int k = 0; k < 3; ++k)
        for (int64_t i = 0; i < n; ++i) dot += g3[k][i] * f[k * n + i];
    for (int k = 0; k < 3; ++k)
        if (o3[k])
            for (int64_t i = 0; i < n; ++i) o3[k][i] = scale * (hv[k * n + i] + g_energy * f[k * n + i]);
    if (g_nu) *g_nu = nu == 0.0 ? dot + g_energy * e : (dot + g_energy * e) / nu;
    if (nu == 0.0)  // leave the stored forces equal to the nu = 0 forces
        for (int k = 0; k < 3; ++k) CK(cudaMemsetAsync(ctx->s[10 + k], 0, sizeof(double) * n, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return TBMD_OK;
}

tbmd_status tbmd_cells(tbmd_ctx *ctx, int32_t *cell_of_particle, int32_t *dims, double *L, double *lo)
{
    if (!ctx) return TBMD_INVALID_ARG;
    if (!ctx->domain_set) return fail(ctx, TBMD_NOT_READY, "no P3BCA domain");
    if (!(ctx->cfg.cutoff > 0)) return fail(ctx, TBMD_INVALID_ARG, "no cutoff, no cell grid");
    tbmd_status st = check_device(ctx);
    if (st != TBMD_OK) return st;
    make_grid(ctx);
    if (dims)
        for (int d = 0; d < 3; ++d) dims[d] = ctx->grid.dims[d];
    if (L)
        for (int d = 0; d < 3; ++d) L[d] = ctx->L[d];
    if (lo)
        for (int d = 0; d < 3; ++d) lo[d] = ctx->lo[d];
    if (cell_of_particle) {
        if (ctx->n == 0) return fail(ctx, TBMD_NOT_READY, "no particles set");
        st = ensure_scalars(ctx);
        if (st != TBMD_OK) return st;
        st = ensure_cells(ctx, ctx->n, false, false);
        if (st != TBMD_OK) return st;
        int nl = 0;
        CK(launch_cell_build(ctx->n, state_pos(ctx), ctx->grid, ctx->gset, ctx->cb, false, ctx->stream, &nl));
        ctx->launches += nl;
        CK(cudaMemcpyAsync(cell_of_particle, ctx->cb.cell_of, sizeof(int32_t) * ctx->n, cudaMemcpyDeviceToHost,
                           ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
    }
    return TBMD_OK;
}

tbmd_status tbmd_sync(tbmd_ctx *ctx)
{
    if (!ctx) return TBMD_INVALID_ARG;
    CK(cudaStreamSynchronize(ctx->stream));
    return TBMD_OK;
}

const char *tbmd_tuning(const tbmd_ctx *ctx) { return ctx ? ctx->tuning.c_str() : "{}"; }

int32_t tbmd_bounds_report(int64_t *violations, int32_t *site, int64_t *index, int64_t *size)
{
    BoundsRecord k{}, gen{};
    const bool ok = cudaDeviceSynchronize() == cudaSuccess && bounds_read_kernels(&k) == cudaSuccess &&
                    bounds_read_gen(&gen) == cudaSuccess;
    const BoundsRecord &first = k.count ? k : gen;
    if (violations) *violations = ok ? (int64_t)k.count + (int64_t)gen.count : -1;
    if (site) *site = first.site;
    if (index) *index = first.index;
    if (size) *size = first.size;
#ifdef TBMD_BOUNDS_CHECK
    return 1;
#else
    return 0;
#endif
}

tbmd_status tbmd_set_profiling(tbmd_ctx *ctx, int32_t on)
{
    if (!ctx) return TBMD_INVALID_ARG;
    CK(cudaStreamSynchronize(ctx->stream));
    phase_resolve(ctx);
    ctx->profiling = on != 0;
    for (int k = 0; k < 5; ++k) {
        ctx->phase_ms[k] = 0;
        ctx->phase_calls[k] = 0;
        ctx->phase_launches[k] = 0;
    }
    return TBMD_OK;
}

int32_t tbmd_phase_times(const tbmd_ctx *ctx, double *ms, uint64_t *calls, uint64_t *launches, int32_t max)
{
    if (!ctx) return 0;
    int32_t k = max < 5 ? max : 5;
    for (int32_t i = 0; i < k; ++i) {
        if (ms) ms[i] = ctx->phase_ms[i];
        if (calls) calls[i] = ctx->phase_calls[i];
        if (launches) launches[i] = ctx->phase_launches[i];
    }
    return 5;
}

}  // extern "C"

// ---------------------------------------------------------------------------------------------
// Autotuner: time each launch variant of the context's algorithm/precision at its current n on the
// particle state (forces only), keep the fastest.  Cache: JSON Lines, one object per key
// {"key": "<gpu>|<alg>|<prec>|n2^<bucket>", "R": r, "warps": w, "ms": t}.

static std::string tune_key(tbmd_ctx *ctx)
{
    cudaDeviceProp prop;
    cudaGetDeviceProperties(&prop, ctx->device);
    int bucket = 0;
    while ((int64_t(1) << (bucket + 1)) <= ctx->n) ++bucket;
    char buf[400];
    snprintf(buf, sizeof buf, "%s|%d|%d|cut%d|n2^%d", prop.name, ctx->cfg.algorithm, ctx->cfg.precision,
             is_p3bca_cut(ctx) ? 1 : 0, bucket);
    return buf;
}

static bool cache_lookup(const char *path, const std::string &key, int *R, int *warps)
{
    if (!path) return false;
    FILE *f = fopen(path, "r");
    if (!f) return false;
    char line[1024];
    bool found = false;
    std::string needle = "\"key\": \"" + key + "\"";
    while (fgets(line, sizeof line, f)) {
        if (!strstr(line, needle.c_str())) continue;
        const char *r = strstr(line, "\"R\": ");
        const char *w = strstr(line, "\"warps\": ");
        if (r && w) {
            *R = atoi(r + 5);
            *warps = atoi(w + 9);
            found = true;
        }
    }
    fclose(f);
    return found;
}

static void cache_store(const char *path, const std::string &key, int R, int warps, float ms)
{
    if (!path) return;
    FILE *f = fopen(path, "a");
    if (!f) return;
    fprintf(f, "{\"key\": \"%s\", \"R\": %d, \"warps\": %d, \"ms\": %.6f}\n", key.c_str(), R, warps, ms);
    fclose(f);
}

static void apply_tuning(tbmd_ctx *ctx, int R, int warps)
{
    if (!mixed(ctx))
        ctx->R_fp64 = R;
    else if (ctx->cfg.algorithm == TBMD_NATA)
        ctx->R_nata = R;
    else
        ctx->R_auta = R;
    ctx->p3_warps = warps;
    invalidate_graph(ctx);
    char buf[160];
    snprintf(buf, sizeof buf, "{\"R\": %d, \"warps\": %d}", sweep_R(ctx), ctx->p3_warps);
    ctx->tuning = buf;
}

extern "C" tbmd_status tbmd_autotune(tbmd_ctx *ctx, const char *cache_path)
{
    if (!ctx) return TBMD_INVALID_ARG;
    if (ctx->n == 0) return fail(ctx, TBMD_NOT_READY, "autotune needs particles");
    tbmd_status st = check_device(ctx);
    if (st != TBMD_OK) return st;
    st = ensure_scalars(ctx);
    if (st != TBMD_OK) return st;
    const std::string key = tune_key(ctx);
    int R = sweep_R(ctx), warps = ctx->p3_warps;
    if (cache_lookup(cache_path, key, &R, &warps)) {
        apply_tuning(ctx, R, warps);
        return TBMD_OK;
    }
    std::vector<std::pair<int, int>> cand;
    if (is_p3bca_cut(ctx)) {
        for (int w : {2, 4, 8}) cand.push_back({R, w});
    } else {
        for (int r : {1, 2, 4}) cand.push_back({r, warps});
    }
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    float best = 1e30f;
    std::pair<int, int> arg = cand[0];
    for (auto &c : cand) {
        apply_tuning(ctx, c.first, c.second);
        st = evaluate(ctx, ctx->n, state_pos(ctx), state_out(ctx), false, nullptr, nullptr, ctx->stream);  // warm-up
        if (st != TBMD_OK) break;
        CK(cudaEventRecord(e0, ctx->stream));
        for (int rep = 0; rep < 3 && st == TBMD_OK; ++rep)
            st = evaluate(ctx, ctx->n, state_pos(ctx), state_out(ctx), false, nullptr, nullptr, ctx->stream);
        CK(cudaEventRecord(e1, ctx->stream));
        CK(cudaEventSynchronize(e1));
        float ms = 0;
        CK(cudaEventElapsedTime(&ms, e0, e1));
        if (ms < best) {
            best = ms;
            arg = c;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (st != TBMD_OK) return st;
    apply_tuning(ctx, arg.first, arg.second);
    cache_store(cache_path, key, arg.first, arg.second, best / 3);
    return TBMD_OK;
}

// ---------------------------------------------------------------------------------------------
// Batched evaluation: nsys independent systems packed back to back, each with its own P3BCA
// domain, evaluated together: one sweep launch over all systems (no cutoff), or one cell build,
// one neighbour pass and one triplet launch over all systems (P3BCA).

// Results of a batched evaluation, in the context's pinned host buffer (valid until the next
// batched call on the context).
struct BatchResult {
    double *f = nullptr, *h = nullptr;  // 3 * N each (h only for the adjoint)
    double *energy = nullptr;           // nsys
    std::vector<uint64_t> counts;       // nsys
};

// Pinned host memory of the context for batched results (device-to-host copies as direct DMA).
static cudaError_t ensure_host_pinned(tbmd_ctx *ctx, size_t bytes)
{
    if (bytes <= ctx->hpin_bytes && ctx->hpin) return cudaSuccess;
    if (ctx->hpin) cudaFreeHost(ctx->hpin);
    ctx->hpin = nullptr;
    ctx->hpin_bytes = 0;
    cudaError_t e = cudaMallocHost(&ctx->hpin, bytes);
    if (e == cudaSuccess) ctx->hpin_bytes = bytes;
    return e;
}

static tbmd_status batch_eval(tbmd_ctx *ctx, int32_t nsys, const int64_t *offsets, const double *box,
                              const double *lo, const double *x, const double *y, const double *z, const double *gfx,
                              const double *gfy, const double *gfz, BatchResult &res)
{
    if (!ctx || !offsets || !x || !y || !z) return TBMD_INVALID_ARG;
    if (nsys < 1) return fail(ctx, TBMD_INVALID_ARG, "nsys < 1");
    if (offsets[0] != 0) return fail(ctx, TBMD_INVALID_ARG, "offsets[0] must be 0");
    for (int s = 0; s < nsys; ++s)
        if (offsets[s + 1] < offsets[s]) return fail(ctx, TBMD_INVALID_ARG, "offsets must not decrease");
    const int64_t N = offsets[nsys];
    if (N < 1 || N > (int64_t)INT32_MAX / 2) return fail(ctx, TBMD_INVALID_ARG, "total n out of range");
    const bool dual = gfx != nullptr;
    tbmd_status st = check_device(ctx);
    if (st != TBMD_OK) return st;
    st = ensure_scalars(ctx);
    if (st != TBMD_OK) return st;
    CK(cudaStreamSynchronize(ctx->stream));
    invalidate_graph(ctx);
    const bool mx = mixed(ctx);
    const double nu = ctx->cfg.nu == 0.0 ? 1.0 : ctx->cfg.nu;  // nu = 0: evaluate the nu = 1 parts
    cudaStream_t sm = ctx->stream;

    // positions (+ direction) and outputs (f, h, energy[nsys], counts[nsys])
    CK(ctx->bpos.ensure(sizeof(double) * 6 * (size_t)N));
    double *P = ctx->bpos.as<double>();
    CK(cudaMemcpyAsync(P, x, sizeof(double) * N, cudaMemcpyHostToDevice, sm));
    CK(cudaMemcpyAsync(P + N, y, sizeof(double) * N, cudaMemcpyHostToDevice, sm));
    CK(cudaMemcpyAsync(P + 2 * N, z, sizeof(double) * N, cudaMemcpyHostToDevice, sm));
    if (dual) {
        CK(cudaMemcpyAsync(P + 3 * N, gfx, sizeof(double) * N, cudaMemcpyHostToDevice, sm));
        CK(cudaMemcpyAsync(P + 4 * N, gfy, sizeof(double) * N, cudaMemcpyHostToDevice, sm));
        CK(cudaMemcpyAsync(P + 5 * N, gfz, sizeof(double) * N, cudaMemcpyHostToDevice, sm));
    }
    // positions checked and each system's extremes found on the device
    const size_t ob = sizeof(int64_t) * (nsys + 1);
    CK(ctx->bext.ensure(ob + 16 + sizeof(unsigned long long) * 6 * (size_t)nsys));
    int64_t *d_off = ctx->bext.as<int64_t>();
    unsigned int *d_bad = (unsigned int *)(ctx->bext.as<char>() + ob);
    unsigned long long *d_keys = (unsigned long long *)(ctx->bext.as<char>() + ob + 16);
    CK(cudaMemcpyAsync(d_off, offsets, ob, cudaMemcpyHostToDevice, sm));
    {
        int sms = 0;
        CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device));
        CK(launch_batch_extents(N, P, P + N, P + 2 * N, d_off, nsys, d_bad, d_keys, sms * 4, sm));
    }
    std::vector<unsigned long long> keys(6 * (size_t)nsys);
    unsigned int bad = 0;
    CK(cudaMemcpyAsync(&bad, d_bad, sizeof bad, cudaMemcpyDeviceToHost, sm));
    CK(cudaMemcpyAsync(keys.data(), d_keys, sizeof(unsigned long long) * keys.size(), cudaMemcpyDeviceToHost, sm));
    CK(cudaStreamSynchronize(sm));
    if (bad) return fail(ctx, TBMD_BAD_INPUT, "non-finite position");
    CK(ctx->bout.ensure(sizeof(double) * (6 * (size_t)N + 2 * (size_t)nsys)));
    double *O = ctx->bout.as<double>();
    double *E = O + 6 * N;
    unsigned long long *CNT = (unsigned long long *)(E + nsys);
    CK(cudaMemsetAsync(E, 0, sizeof(double) * 2 * nsys, sm));
    const Pos pos{P, P + N, P + 2 * N, dual ? P + 3 * N : nullptr, dual ? P + 4 * N : nullptr,
                  dual ? P + 5 * N : nullptr};
    const Out out{O, O + N, O + 2 * N, O + 3 * N, O + 4 * N, O + 5 * N};
    res.counts.assign(nsys, 0);
    int nl = 0;

    if (is_p3bca_cut(ctx)) {
        // per-system grids: the given box, or the reference's domain rule on that system's positions
        std::vector<Grid> grids(nsys);
        std::vector<int64_t> cell_off(nsys + 1, 0);
        int cap = 32, stage = 256;
        for (int s = 0; s < nsys; ++s) {
            double Ls[3], los[3];
            const int64_t b = offsets[s], e = offsets[s + 1];
            for (int d = 0; d < 3; ++d) {
                if (box) {
                    Ls[d] = box[3 * s + d];
                    los[d] = lo ? lo[3 * s + d] : 0.0;
                } else {
                    // the reference's domain rule on this system's extremes (0 for an empty system)
                    const double mn = e > b ? key_to_double(keys[6 * s + d]) : 0.0;
                    const double mxv = e > b ? key_to_double(keys[6 * s + 3 + d]) : 0.0;
                    los[d] = mn - 0.0001;
                    Ls[d] = std::fabs((mxv + 0.0001) - los[d]);
                }
                if (!(Ls[d] > 0) || !std::isfinite(Ls[d]) || !std::isfinite(los[d]))
                    return fail(ctx, TBMD_INVALID_ARG, "bad box of system %d", s);
            }
            grids[s] = system_grid(ctx, Ls, los);
            cell_off[s + 1] = cell_off[s] + grids[s].ncells;
            const double vol = Ls[0] * Ls[1] * Ls[2], c = ctx->cfg.cutoff;
            const double half = 4.18879020478639 * c * c * c * ((double)(e - b) / vol) * 0.5;
            int want = ((int)(2.0 * half + 48.0) + 31) / 32 * 32;
            cap = want > cap ? want : cap;
            const int sc = neighbor_stage_cap(grids[s], e - b);
            stage = sc > stage ? sc : stage;
        }
        // the neighbour-cell table depends only on each system's cell counts per axis: rebuilt when
        // they change (or after a single-system evaluation replaced it)
        std::vector<int32_t> tkey(3 * (size_t)nsys);
        for (int s = 0; s < nsys; ++s)
            for (int d = 0; d < 3; ++d) tkey[3 * s + d] = grids[s].dims[d];
        if (ctx->ncell_single || tkey != ctx->ncell_batch_key) {
            std::vector<int32_t> tab27((size_t)cell_off[nsys] * 27);
            for (int s = 0; s < nsys; ++s) neighbor_cell_table(grids[s], cell_off[s], tab27.data());
            CK(ctx->ncell_tab.ensure(sizeof(int32_t) * tab27.size()));
            CK(cudaMemcpyAsync(ctx->ncell_tab.p, tab27.data(), sizeof(int32_t) * tab27.size(), cudaMemcpyHostToDevice,
                               sm));
            CK(cudaStreamSynchronize(sm));  // tab27 lives on this stack frame
            ctx->ncell_batch_key = tkey;
        }
        ctx->ncell_single = false;  // the single-system table is rebuilt on the next single evaluation
        const size_t gbytes = sizeof(Grid) * nsys, obytes = sizeof(int64_t) * (nsys + 1);
        CK(ctx->bsys.ensure(gbytes + 2 * obytes + 64));
        char *tb = ctx->bsys.as<char>();
        CK(cudaMemcpyAsync(tb, grids.data(), gbytes, cudaMemcpyHostToDevice, sm));
        CK(cudaMemcpyAsync(tb + gbytes, cell_off.data(), obytes, cudaMemcpyHostToDevice, sm));
        CK(cudaMemcpyAsync(tb + gbytes + obytes, offsets, obytes, cudaMemcpyHostToDevice, sm));
        const int saved_cap = ctx->cap;
        Grid all = grids[0];
        all.ncells = cell_off[nsys];
        ctx->cap = cap;
        tbmd_status r = TBMD_CAPACITY_RETRY;
        for (int attempt = 0; attempt < 4; ++attempt) {
            ctx->grid = all;
            ctx->gset = GridSet{(const Grid *)tb, (const int64_t *)(tb + gbytes), (const int64_t *)(tb + gbytes + obytes),
                                nsys};
            ctx->max_stage = stage;
            r = ensure_cell_bufs(ctx, N, all.ncells, dual, true);
            if (r != TBMD_OK) break;
            CK(reset_cap_flags(ctx, sm));
            CK(cudaMemsetAsync(E, 0, sizeof(double) * 2 * nsys, sm));
            CellBufs &cb = ctx->cb;
            CK(launch_cell_build(N, pos, ctx->grid, ctx->gset, cb, dual, sm, &nl));
            CK(launch_neighbors(N, ctx->grid, ctx->gset, ctx->ncell_tab.as<int32_t>(), ctx->max_stage, cb, sm));
            CK(cudaMemsetAsync(cb.fs[0], 0, sizeof(double) * 3 * N, sm));  // fs[0..2] are adjacent
            if (dual) CK(cudaMemsetAsync(cb.hs[0], 0, sizeof(double) * 3 * N, sm));
            CK(launch_p3bca(mx, dual, true, N, ctx->grid, ctx->gset, cb, nu, E, CNT, ctx->plan, sm));
            CK(launch_unsort(N, cb, out, dual, sm));
            nl += 3 + (dual ? 1 : 0);
            CapSeen seen{};
            CK(read_cap_flags(ctx, sm, &seen));
            CK(cudaStreamSynchronize(sm));
            r = TBMD_OK;
            if (!grow_caps(ctx, seen)) break;
            r = TBMD_CAPACITY_RETRY;
        }
        ctx->cap = saved_cap > ctx->cap ? saved_cap : ctx->cap;  // the next ensure_cells rebuilds the single grid
        if (r != TBMD_OK) return r == TBMD_CAPACITY_RETRY ? fail(ctx, r, "neighbour capacity exceeded") : r;
        std::vector<unsigned long long> c(nsys);
        CK(cudaMemcpyAsync(c.data(), CNT, sizeof(unsigned long long) * nsys, cudaMemcpyDeviceToHost, sm));
        CK(cudaStreamSynchronize(sm));
        for (int s = 0; s < nsys; ++s) res.counts[s] = c[s];
    } else {
        // one sweep over all systems (AUTA work items; NATA gives the same forces)
        const int R = dual ? (mx ? 2 : 1) : (mx ? ctx->R_auta : ctx->R_fp64);
        const int JB = 32 * R;
        std::vector<int64_t> prefix, sys_items(nsys + 1, 0), sys_prefix(nsys, 0);
        std::vector<int32_t> sys_nb(nsys, 0);
        for (int s = 0; s < nsys; ++s) {
            const int64_t ns = offsets[s + 1] - offsets[s];
            const int64_t nb = ns >= 3 ? (ns - 2 + JB) / JB : 0;
            std::vector<int64_t> pre((size_t)nb + 1, 0);
            const int64_t items = sweep_items(TBMD_AUTA, ns, JB, pre.data());
            sys_prefix[s] = (int64_t)prefix.size();
            sys_nb[s] = (int32_t)nb;
            prefix.insert(prefix.end(), pre.begin(), pre.end());
            sys_items[s + 1] = sys_items[s] + items;
            res.counts[s] = choose3(ns);
        }
        if (sys_items[nsys] >= (int64_t)UINT32_MAX - 65536) return fail(ctx, TBMD_INVALID_ARG, "too many work items");
        const size_t pb = sizeof(int64_t) * prefix.size();
        CK(ctx->bprefix.ensure(pb + 64));
        CK(cudaMemcpyAsync(ctx->bprefix.p, prefix.data(), pb, cudaMemcpyHostToDevice, sm));
        const size_t ib = sizeof(int64_t) * (nsys + 1), nbb = sizeof(int32_t) * nsys;
        CK(ctx->bsys.ensure(3 * ib + nbb + 64));
        char *tb = ctx->bsys.as<char>();
        CK(cudaMemcpyAsync(tb, sys_items.data(), ib, cudaMemcpyHostToDevice, sm));
        CK(cudaMemcpyAsync(tb + ib, offsets, ib, cudaMemcpyHostToDevice, sm));
        CK(cudaMemcpyAsync(tb + 2 * ib, sys_prefix.data(), sizeof(int64_t) * nsys, cudaMemcpyHostToDevice, sm));
        CK(cudaMemcpyAsync(tb + 3 * ib, sys_nb.data(), nbb, cudaMemcpyHostToDevice, sm));
        SweepWork w{ctx->bprefix.as<int64_t>(), 0, sys_items[nsys], sweep_counter(ctx), nsys, (const int64_t *)tb,
                    (const int64_t *)(tb + ib), (const int64_t *)(tb + 2 * ib), (const int32_t *)(tb + 3 * ib)};
        CK(cudaMemsetAsync(O, 0, sizeof(double) * (dual ? 6 : 3) * N, sm));
        CK(cudaMemsetAsync(w.counter, 0, sizeof(unsigned int), sm));
        int sms = 0;
        CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device));
        CK(launch_auta(mx, dual, R, true, N, pos, out, E, nu, w, sms * 8, sm));
        nl += 1;
    }
    ctx->launches += nl;
    CK(ensure_host_pinned(ctx, sizeof(double) * (6 * (size_t)N + nsys)));
    res.f = (double *)ctx->hpin;
    res.h = res.f + 3 * N;
    res.energy = res.h + 3 * N;
    CK(cudaMemcpyAsync(res.f, O, sizeof(double) * 3 * N, cudaMemcpyDeviceToHost, sm));
    if (dual) CK(cudaMemcpyAsync(res.h, O + 3 * N, sizeof(double) * 3 * N, cudaMemcpyDeviceToHost, sm));
    CK(cudaMemcpyAsync(res.energy, E, sizeof(double) * nsys, cudaMemcpyDeviceToHost, sm));
    CK(cudaStreamSynchronize(sm));
    if (ctx->cfg.nu == 0.0) {  // the nu = 1 parts were evaluated; the true f, E and H vanish
        std::fill(res.f, res.f + 3 * N, 0.0);
        if (dual) std::fill(res.h, res.h + 3 * N, 0.0);
        std::fill(res.energy, res.energy + nsys, 0.0);
    }
    return TBMD_OK;
}

extern "C" tbmd_status tbmd_batch_forces(tbmd_ctx *ctx, int32_t nsys, const int64_t *offsets, const double *box,
                                         const double *lo, const double *x, const double *y, const double *z,
                                         double *fx, double *fy, double *fz, double *energy, uint64_t *triplets)
{
    BatchResult r;
    tbmd_status st = batch_eval(ctx, nsys, offsets, box, lo, x, y, z, nullptr, nullptr, nullptr, r);
    if (st != TBMD_OK) return st;
    const int64_t N = offsets[nsys];
    double *o3[3] = {fx, fy, fz};
    for (int k = 0; k < 3; ++k)
        if (o3[k]) std::memcpy(o3[k], r.f + k * N, sizeof(double) * N);
    for (int s = 0; s < nsys; ++s) {
        if (energy) energy[s] = r.energy[s];
        if (triplets) triplets[s] = r.counts[s];
    }
    return TBMD_OK;
}

extern "C" tbmd_status tbmd_batch_adjoint(tbmd_ctx *ctx, int32_t nsys, const int64_t *offsets, const double *box,
                                          const double *lo, const double *x, const double *y, const double *z,
                                          const double *gfx, const double *gfy, const double *gfz,
                                          const double *g_energy, double *gx, double *gy, double *gz, double *g_nu)
{
    if (!gfx || !gfy || !gfz || !g_energy) return ctx ? fail(ctx, TBMD_INVALID_ARG, "null cotangent") : TBMD_INVALID_ARG;
    BatchResult r;
    tbmd_status st = batch_eval(ctx, nsys, offsets, box, lo, x, y, z, gfx, gfy, gfz, r);
    if (st != TBMD_OK) return st;
    const int64_t N = offsets[nsys];
    const double *g3[3] = {gfx, gfy, gfz};
    double *o3[3] = {gx, gy, gz};
    const double nu = ctx->cfg.nu;
    // with nu = 0 batch_eval zeroed f, E and H (so gx = 0); g_nu needs the nu = 1 parts, recomputed
    // here (into the same pinned buffer: f and E are replaced, h is no longer needed)
    if (nu == 0.0) {
        BatchResult r1;
        ctx->cfg.nu = 1.0;
        st = batch_eval(ctx, nsys, offsets, box, lo, x, y, z, nullptr, nullptr, nullptr, r1);
        ctx->cfg.nu = 0.0;
        if (st != TBMD_OK) return st;
        r.f = r1.f;
        r.energy = r1.energy;
    }
    for (int s = 0; s < nsys; ++s) {
        const double ge = g_energy[s];
        if (!std::isfinite(ge)) return fail(ctx, TBMD_INVALID_ARG, "g_energy of system %d not finite", s);
        double dot = 0.0;
        for (int k = 0; k < 3; ++k)
            for (int64_t i = offsets[s]; i < offsets[s + 1]; ++i) {
                dot += g3[k][i] * r.f[k * N + i];
                if (o3[k]) o3[k][i] = nu == 0.0 ? 0.0 : r.h[k * N + i] + ge * r.f[k * N + i];
            }
        if (g_nu) g_nu[s] = nu == 0.0 ? dot + ge * r.energy[s] : (dot + ge * r.energy[s]) / nu;
    }
    return TBMD_OK;
}
