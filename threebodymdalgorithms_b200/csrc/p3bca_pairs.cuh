// P3BCA triplets, pair-compacted form: k_p3pair (forces and energy; FP32 geometry for the mixed
// form, FP64 for the FP64 drop-in).  Included by tbmd_kernels.cu after k_p3bca, whose work items,
// slot types and helpers it shares; the adjoint (dual types) keeps k_p3bca.
//
// Work items are those of k_p3bca: a particle s whose half list holds at most P3_CHUNK (64) entries
// (one "triangle" item: every pair of its entries), or a chunk pair (I < J) of a longer list (one
// "cross" item: every pair of an entry of chunk I with an entry of chunk J), both taken from dynamic
// counters.  The entries are staged as slots in the warp's shared memory: the edge e = x_t - x_s
// (hi part, and b = e.e; the lo part for the mixed form), a gradient accumulator and the neighbour
// index.  Every triplet (s, j, k) with j, k two slots is then a pair of slots; it is inside the
// cutoff when the third edge x_k - x_j is (both edges from s are, by the half list).
//
// An item runs in three phases:
//   1. Adjacency.  Every candidate slot pair is tested once, in FP32 on the hi parts of the edges:
//      the raw squared distance for an item none of whose entries wraps around the box (the box at
//      least 4 cutoffs wide), else the reference's periodic formula (structs.hpp:106-115).  Outside a
//      guard band around cutoff^2 the FP32 value decides; inside it the reference's own FP64 test on
//      the two neighbours' positions, so the pair set is exactly the reference's (Algorithm.cpp:94-100,
//      d == cutoff inside).  Row slot a gets a 64-bit mask of the partner slots after it (or of chunk
//      J's slots), column slot b the mask of the rows that pair with it.  The item's triplet count is
//      the total population count.  Pairs are visited in circular diagonals inside a 32-slot block
//      (lane x against slot (x + d) mod m, the partner's bit arriving by a shuffle) and by broadcast
//      across blocks (all lanes against one slot, its column mask being the ballot).
//   2. Compute.  The passing pairs, in row-major order, are cut into batches of whole rows holding at
//      most PB pairs, and a batch's pairs into 32 equal contiguous ranges, one per lane: the triplet
//      math runs only on pairs inside the cutoff, and the lanes stay busy whatever the list looks
//      like.  A lane keeps its current row slot's edge in registers and sums the row side of its
//      pairs there (one record per row segment); the column side of each pair is written to a
//      staging record at the pair's column-major place in the batch, found from the column mask by a
//      population count, so no two pairs share a record and nothing needs an atomic.
//   3. Gather.  Each lane adds, for the slots it owns, their row segments and their column records
//      into the slot accumulators (plain shared-memory adds: a slot has one owner lane).  At the end
//      of the item every slot is flushed into the FP64 forces with one atomic per component, and s
//      gets minus their sum (translation invariance holds per triplet).
// Accumulation is factored as in k_p3bca: a slot's gradient is (scalar) * (its own edge) + (vector),
// the row side of a pair adding (alpha, gamma w) and the column side (beta, -gamma w).

// Shared memory of one warp in k_p3pair (byte offsets; arrays of Slot4 start on their alignment).
template <class S>
struct PairLayout {
    static constexpr int SL = 2 * P3_CHUNK;                  // staged slots: one chunk or two
    static constexpr int RM = P3_CHUNK;                      // rows / columns of an item
    static constexpr int PB = sizeof(S) == 4 ? 192 : 96;     // staged pairs of one batch
    static constexpr bool lo = HasLo<S>::value;              // mixed: lo parts of the edges
    static constexpr bool f32 = !lo;                         // FP64: an FP32 copy of the edges for phase 1
    static constexpr size_t eh = 0;                                        // Slot4<S>[SL] edge, w = e.e
    static constexpr size_t el = eh + SL * sizeof(Slot4<S>);               // Slot4<S>[SL] lo part (mixed)
    static constexpr size_t ef = el + (lo ? SL * sizeof(Slot4<S>) : 0);    // float4[SL] FP32 edge (FP64)
    static constexpr size_t acc = ef + (f32 ? SL * sizeof(float4) : 0);    // Slot4<S>[SL] accumulators
    static constexpr size_t part = acc + SL * sizeof(Slot4<S>);            // Slot4<S>[PB] column-side records
    static constexpr size_t segr = part + PB * sizeof(Slot4<S>);           // Slot4<S>[RM] row-start segments
    static constexpr size_t segl = segr + RM * sizeof(Slot4<S>);           // Slot4<S>[32] lane-start segments
    static constexpr size_t rmask = segl + 32 * sizeof(Slot4<S>);          // uint64[RM] row masks
    static constexpr size_t col = rmask + RM * sizeof(uint64_t);           // ColMeta[RM] column masks, places
    static constexpr size_t rstart = col + RM * 16;                        // int[RM + 8] row starts
    static constexpr size_t gidx = rstart + (RM + 8) * sizeof(int);        // int[SL] neighbour index
    static constexpr size_t bytes = (gidx + SL * sizeof(int) + 127) / 128 * 128;
};

// Column j of an item: its mask of rows, and the place of its first record in the batch's staging
// (start) and that place less the column's pairs with rows before the batch (base).
struct alignas(16) ColMeta {
    unsigned int lo, hi;
    int base, start;
};

__device__ __forceinline__ uint64_t bits_below(int x) { return x >= 64 ? ~0ull : ((1ull << x) - 1ull); }
__device__ __forceinline__ uint64_t bits_above(int x) { return x >= 63 ? 0ull : (~0ull << (x + 1)); }

__device__ __forceinline__ int warp_inclusive_scan(int v, int lane)
{
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int t = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += t;
    }
    return v;
}

template <class S>
__device__ __forceinline__ Slot4<S> slot4_zero()
{
    return Slot4<S>{szero<S>(), szero<S>(), szero<S>(), szero<S>()};
}
template <class S>
__device__ __forceinline__ Slot4<S> slot4_add(Slot4<S> a, const Slot4<S> &b)
{
    a.x = a.x + b.x;
    a.y = a.y + b.y;
    a.z = a.z + b.z;
    a.w = a.w + b.w;
    return a;
}

template <class S>
struct P3PairMinBlocks {  // resident CTAs of 256 threads the register budget is planned for
    static constexpr int value = sizeof(S) == 4 ? 2 : 1;
};

template <class S, bool ENERGY>
__global__ void __launch_bounds__(256, P3PairMinBlocks<S>::value)
    k_p3pair(int64_t n, const __grid_constant__ Grid g, GridSet set, CellBufs cb, double nu_d, double *energy_out,
             unsigned long long *count_out)
{
    using L = PairLayout<S>;
    extern __shared__ __align__(128) unsigned char smem[];
    const int lane = threadIdx.x & 31;
    unsigned char *base = smem + (size_t)(threadIdx.x >> 5) * L::bytes;
    Slot4<S> *const EH = (Slot4<S> *)(base + L::eh);
    Slot4<S> *const EL = (Slot4<S> *)(base + L::el);
    // FP32 edges of phase 1: for the mixed form the hi edges themselves
    const float4 *const EF = (const float4 *)(base + (L::f32 ? L::ef : L::eh));
    float4 *const EFw = (float4 *)(base + L::ef);
    Slot4<S> *const AC = (Slot4<S> *)(base + L::acc);
    Slot4<S> *const PART = (Slot4<S> *)(base + L::part);
    Slot4<S> *const SEGR = (Slot4<S> *)(base + L::segr);
    Slot4<S> *const SEGL = (Slot4<S> *)(base + L::segl);
    uint64_t *const RMASK = (uint64_t *)(base + L::rmask);
    ColMeta *const COL = (ColMeta *)(base + L::col);
    int *const RSTART = (int *)(base + L::rstart);
    int *const GIDX = (int *)(base + L::gidx);
    constexpr unsigned FULL = 0xffffffffu;

    const S nu = constant<S>(nu_d), nu3 = constant<S>(-3.0 * nu_d), nu15 = constant<S>(15.0 * nu_d);
    const Out outs = {cb.fs[0], cb.fs[1], cb.fs[2], nullptr, nullptr, nullptr};
    const int cap = cb.cap;
    const double cwrap = sqrt(g.sqcut) * 1.0000001;
    unsigned long long cnt = 0;  // warp-uniform
    double en_acc = 0.0;
    S en = szero<S>();
    int cur_sys = 0;
    auto flush = [&](int sys) {
        if (lane == 0 && count_out && cnt) atomicAdd(count_out + sys, cnt);
        cnt = 0;
        if (ENERGY) {
            const double e = warp_sum(en_acc + to_acc(en));
            if (lane == 0) atomicAdd(energy_out + sys, e);
            en_acc = 0.0;
            en = szero<S>();
        }
    };

    auto item = [&](int s, int offI, int mI, int offJ, int mJ) {
        const int sys = system_of(set.sys_off, set.nsys, s);
        if (sys != cur_sys) {
            flush(cur_sys);
            cur_sys = sys;
        }
        const Grid &G = set.nsys > 1 ? set.grids[sys] : g;
        const bool cross = mJ > 0;
        const int Ms = mI + mJ;
        const int R = mI;              // rows
        const int C = cross ? mJ : mI;  // columns
        const int c0 = cross ? mI : 0;  // slot of column 0

        // stage the slots
        const double xi = cb.xs[s], yi = cb.ys[s], zi = cb.zs[s];
        bool nowrap = true;
        for (int e = lane; e < Ms; e += 32) {
            const int pos_in_list = e < mI ? offI + e : offJ + (e - mI);
            const int32_t t = (int32_t)TBMD_IX(cb.nbr[(int64_t)s * cap + pos_in_list], n, BS_LIST);
            GIDX[e] = t;
            const double ddx = cb.xs[t] - xi, ddy = cb.ys[t] - yi, ddz = cb.zs[t] - zi;
            nowrap = nowrap && fabs(ddx) <= cwrap && fabs(ddy) <= cwrap && fabs(ddz) <= cwrap;
            V3<S> v, l;
            split<S>(ddx, 0.0, v.x, l.x);
            split<S>(ddy, 0.0, v.y, l.y);
            split<S>(ddz, 0.0, v.z, l.z);
            EH[e] = Slot4<S>{v.x, v.y, v.z, dot3(v, v)};
            if (L::lo) EL[e] = Slot4<S>{l.x, l.y, l.z, szero<S>()};
            if (L::f32) EFw[e] = make_float4((float)ddx, (float)ddy, (float)ddz, 0.f);
            AC[e] = slot4_zero<S>();
        }
        const bool rawok = G.raw_ok && __all_sync(FULL, nowrap);
        const float t_lo = rawok ? G.hi_lo : (float)G.sqcut - G.band;
        const float t_hi = rawok ? G.hi_hi : (float)G.sqcut + G.band;
        const float Lx = (float)G.L[0], Ly = (float)G.L[1], Lz = (float)G.L[2];
        __syncwarp();

        // ---- phase 1: adjacency.  test(): slots p (FP32 edge ep, held by the caller) and q; false
        // for lanes with act false.  All lanes call it together.
        auto test = [&](bool act, float4 ep, int p, int q) -> bool {
            const float4 eq = EF[q];
            const float dx = eq.x - ep.x, dy = eq.y - ep.y, dz = eq.z - ep.z;
            float d2;
            if (rawok) {
                d2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
            } else {
                const float ax = fabsf(dx), ay = fabsf(dy), az = fabsf(dz);
                const float mx = fminf(ax, Lx - ax), my = fminf(ay, Ly - ay), mz = fminf(az, Lz - az);
                d2 = fmaf(mx, mx, fmaf(my, my, mz * mz));
            }
            bool in = act && d2 <= t_lo;
            const bool amb = act && !in && d2 <= t_hi;
            if (__any_sync(FULL, amb)) {
                if (amb) {
                    const int32_t tp = GIDX[p], tq = GIDX[q];
                    in = sqdist_periodic(cb.xs[tp], cb.ys[tp], cb.zs[tp], cb.xs[tq], cb.ys[tq], cb.zs[tq], G) <= G.sqcut;
                }
            }
            return in;
        };

        uint64_t rm0 = 0, rm1 = 0, cm0 = 0, cm1 = 0;  // rows / columns lane and lane + 32
        if (!cross) {
            uint64_t A0 = 0, A1 = 0;  // all partners of slots lane and 32 + lane
            const int mA = min(R, 32);
            {
                const bool own = lane < mA;
                const int x = own ? lane : 0;
                const float4 ep = EF[x];
                int y = x;
                for (int d = 1; 2 * d <= mA; ++d) {
                    y = (y + 1 == mA) ? 0 : y + 1;  // (x + d) mod mA
                    const bool act = own && (2 * d < mA || lane < d);
                    const bool in = test(act, ep, x, own ? y : 0);
                    if (in) A0 |= 1ull << y;
                    int src = lane - d;  // the lane whose partner this step is `lane`
                    if (src < 0) src += mA;
                    const bool in_src = __shfl_sync(FULL, in, src & 31);
                    if (own && in_src && (2 * d < mA || src < d)) A0 |= 1ull << src;
                }
            }
            if (R > 32) {
                const int mB = R - 32;
                {
                    const bool own = lane < mB;
                    const int x = own ? lane : 0;
                    const float4 ep = EF[32 + x];
                    int y = x;
                    for (int d = 1; 2 * d <= mB; ++d) {
                        y = (y + 1 == mB) ? 0 : y + 1;
                        const bool act = own && (2 * d < mB || lane < d);
                        const bool in = test(act, ep, 32 + x, 32 + (own ? y : 0));
                        if (in) A1 |= 1ull << (32 + y);
                        int src = lane - d;
                        if (src < 0) src += mB;
                        const bool in_src = __shfl_sync(FULL, in, src & 31);
                        if (own && in_src && (2 * d < mB || src < d)) A1 |= 1ull << (32 + src);
                    }
                }
                // block A (32 slots, one per lane) against each slot b of block B
                const float4 ea = EF[lane];
                for (int b = 32; b < R; ++b) {
                    const bool in = test(true, ea, lane, b);
                    if (in) A0 |= 1ull << b;
                    const unsigned ball = __ballot_sync(FULL, in);
                    if (lane == b - 32) A1 |= (uint64_t)ball;
                }
            }
            rm0 = A0 & bits_above(lane);
            cm0 = A0 & bits_below(lane);
            rm1 = A1 & bits_above(32 + lane);
            cm1 = A1 & bits_below(32 + lane);
        } else {
            const bool own0 = lane < R, own1 = lane + 32 < R;
            const float4 e0 = EF[own0 ? lane : 0], e1 = EF[own1 ? lane + 32 : 0];
            const bool two = R > 32;
            for (int j = 0; j < C; ++j) {
                const int q = c0 + j;
                const bool in0 = test(own0, e0, own0 ? lane : 0, q);
                const bool in1 = two ? test(own1, e1, own1 ? lane + 32 : 0, q) : false;
                if (in0) rm0 |= 1ull << j;
                if (in1) rm1 |= 1ull << j;
                const unsigned b0 = __ballot_sync(FULL, in0), b1 = __ballot_sync(FULL, in1);
                if (lane == (j & 31)) {
                    const uint64_t colm = (uint64_t)b0 | ((uint64_t)b1 << 32);
                    if (j < 32)
                        cm0 = colm;
                    else
                        cm1 = colm;
                }
            }
        }
        RMASK[lane] = rm0;
        RMASK[lane + 32] = rm1;
        COL[lane].lo = (unsigned)cm0;
        COL[lane].hi = (unsigned)(cm0 >> 32);
        COL[lane + 32].lo = (unsigned)cm1;
        COL[lane + 32].hi = (unsigned)(cm1 >> 32);
        int T;
        {
            const int r0 = __popcll(rm0), r1 = __popcll(rm1);
            const int i0 = warp_inclusive_scan(r0, lane), i1 = warp_inclusive_scan(r1, lane);
            const int t0 = __shfl_sync(FULL, i0, 31);
            T = t0 + __shfl_sync(FULL, i1, 31);
            RSTART[lane] = i0 - r0;
            RSTART[lane + 32] = t0 + i1 - r1;
            if (lane == 0) RSTART[64] = T;
        }
        cnt += (unsigned long long)T;
        __syncwarp();

        // ---- phases 2 and 3, batch by batch
        int a0 = 0;
        while (a0 < R && RSTART[a0] < T) {
            const int p0 = RSTART[a0];
            // batch rows [a0, a1): the longest run of whole rows with at most PB pairs (one row holds
            // at most 64, so a1 > a0)
            const int ca = a0 + 1 + lane, cb2 = a0 + 33 + lane;
            const bool ok0 = ca <= R && RSTART[ca] - p0 <= L::PB;
            const bool ok1 = cb2 <= R && RSTART[cb2] - p0 <= L::PB;
            const int a1 = a0 + __popc(__ballot_sync(FULL, ok0)) + __popc(__ballot_sync(FULL, ok1));
            const int P = RSTART[a1] - p0;
            const uint64_t rows_in = bits_below(a1) & ~bits_below(a0), rows_before = bits_below(a0);
            {
                // column places: exclusive scan of the columns' pair counts in this batch
                const ColMeta k0 = COL[lane], k1 = COL[lane + 32];
                const uint64_t m0 = (uint64_t)k0.lo | ((uint64_t)k0.hi << 32);
                const uint64_t m1 = (uint64_t)k1.lo | ((uint64_t)k1.hi << 32);
                const int n0 = __popcll(m0 & rows_in), n1 = __popcll(m1 & rows_in);
                const int i0 = warp_inclusive_scan(n0, lane), i1 = warp_inclusive_scan(n1, lane);
                const int t0 = __shfl_sync(FULL, i0, 31);
                const int s0 = i0 - n0, s1 = t0 + i1 - n1;
                COL[lane].start = s0;
                COL[lane].base = s0 - __popcll(m0 & rows_before);
                COL[lane + 32].start = s1;
                COL[lane + 32].base = s1 - __popcll(m1 & rows_before);
            }
            __syncwarp();
            const int Q = (P + 31) >> 5;
            int q = lane * Q;
            const int qe = min(q + Q, P);
            if (q < qe) {
                // the row of pair p0 + q: the last row a in [a0, a1) with RSTART[a] <= p0 + q
                const int p = p0 + q;
                int lo_ = a0, hi_ = a1;
                while (hi_ - lo_ > 1) {
                    const int mid = (lo_ + hi_) >> 1;
                    if (RSTART[mid] <= p)
                        lo_ = mid;
                    else
                        hi_ = mid;
                }
                int a = lo_;
                uint64_t mask = RMASK[a];
                for (int r = p - RSTART[a]; r > 0; --r) mask &= mask - 1ull;
                // where the current row segment's record goes: the row's own record when the
                // segment starts the row, else this lane's
                int seg = p == RSTART[a] ? a : -1 - lane;
                Slot4<S> od = EH[a];
                V3<S> u = {od.x, od.y, od.z};
                S aa = od.w;
                V3<S> ul = vzero<S>();
                if (L::lo) {
                    const Slot4<S> ol = EL[a];
                    ul = {ol.x, ol.y, ol.z};
                }
                uint64_t below_a = bits_below(a);
                Slot4<S> racc = slot4_zero<S>();
                for (; q < qe; ++q) {
                    if (mask == 0ull) {
                        // the row ends inside this lane's range: close its segment, go to the next
                        // row with pairs
                        if (seg >= 0)
                            SEGR[TBMD_IX(seg, a1, BS_PAIR_SEG)] = racc;
                        else
                            SEGL[TBMD_IX(-1 - seg, 32, BS_PAIR_SEG)] = racc;
                        racc = slot4_zero<S>();
                        do {
                            ++a;
                            mask = RMASK[TBMD_IX(a, a1, BS_PAIR_ROW)];
                        } while (mask == 0ull && a + 1 < a1);
                        seg = a;
                        od = EH[a];
                        u = {od.x, od.y, od.z};
                        aa = od.w;
                        if (L::lo) {
                            const Slot4<S> ol = EL[a];
                            ul = {ol.x, ol.y, ol.z};
                        }
                        below_a = bits_below(a);
                    }
                    const int j = __ffsll((long long)mask) - 1;
                    mask &= mask - 1ull;
                    const Slot4<S> pd = EH[TBMD_IX(c0 + j, Ms, BS_SLOT)];
                    const V3<S> v = {pd.x, pd.y, pd.z};
                    V3<S> vl = vzero<S>();
                    if (L::lo) {
                        const Slot4<S> pl = EL[c0 + j];
                        vl = {pl.x, pl.y, pl.z};
                    }
                    const ColMeta cm = COL[TBMD_IX(j, C, BS_PAIR_COL)];
                    const V3<S> w = third_edge(u, ul, v, vl);
                    const ATCoef<S> cf = at_coef<ENERGY>(aa, pd.w, dot3(w, w), dot3(u, v), dot3(u, w), dot3(v, w),
                                                         nu, nu3, nu15, true, en);
                    const V3<S> gw = w * cf.gamma;
                    racc.x = racc.x + gw.x;
                    racc.y = racc.y + gw.y;
                    racc.z = racc.z + gw.z;
                    racc.w = racc.w + cf.alpha;
                    const int place = cm.base + __popc(cm.lo & (unsigned)below_a) +
                                      __popc(cm.hi & (unsigned)(below_a >> 32));
                    PART[TBMD_IX(place, P, BS_PAIR_PLACE)] = Slot4<S>{gw.x, gw.y, gw.z, cf.beta};
                }
                if (seg >= 0)
                    SEGR[seg] = racc;
                else
                    SEGL[-1 - seg] = racc;
            }
            __syncwarp();
            // gather: rows of this batch owned by the lane, then its columns
            for (int h = 0; h < 2; ++h) {
                const int a = lane + 32 * h;
                if (a >= a0 && a < a1) {
                    const int rs = RSTART[a] - p0, re = RSTART[a + 1] - p0;
                    if (rs < re) {
                        Slot4<S> sum = SEGR[a];
                        for (int l = rs / Q + 1; l * Q < re; ++l) sum = slot4_add(sum, SEGL[l]);
                        AC[a] = slot4_add(AC[a], sum);
                    }
                }
            }
            for (int h = 0; h < 2; ++h) {
                const int j = lane + 32 * h;
                if (j < C) {
                    const int cs = COL[j].start, ce = j + 1 < C ? COL[j + 1].start : P;
                    Slot4<S> sum = slot4_zero<S>();
                    for (int k = cs; k < ce; ++k) sum = slot4_add(sum, PART[k]);
                    Slot4<S> a = AC[c0 + j];
                    a.x = a.x - sum.x;
                    a.y = a.y - sum.y;
                    a.z = a.z - sum.z;
                    a.w = a.w + sum.w;
                    AC[c0 + j] = a;
                }
            }
            __syncwarp();
            a0 = a1;
        }

        // flush the slots: gradient = scalar * edge + vector, in FP64; s gets minus the sum
        V3<double> gia = {0.0, 0.0, 0.0};
        for (int e = lane; e < Ms; e += 32) {
            const Slot4<S> a = AC[e], ed = EH[e];
            const double sc = to_double(a.w);
            const V3<double> ge = {fma(sc, to_double(ed.x), to_double(a.x)), fma(sc, to_double(ed.y), to_double(a.y)),
                                   fma(sc, to_double(ed.z), to_double(a.z))};
            atomic_out(outs, GIDX[e], ge);
            gia = gia + ge;
        }
        gia = warp_sum3(gia);
        if (lane == 0) atomic_out(outs, s, V3<double>{-gia.x, -gia.y, -gia.z});
        if (ENERGY) {
            en_acc += to_acc(en);
            en = szero<S>();
        }
        __syncwarp();
    };

    // lists of at most one chunk: one item per particle
    unsigned int wk = 0;
    if (lane == 0) wk = atomicAdd(cb.work_counter, 1u);
    wk = __shfl_sync(FULL, wk, 0);
    while ((int64_t)wk < n) {
        unsigned int wn = 0;
        if (lane == 0) wn = atomicAdd(cb.work_counter, 1u);
        const int s = (int)wk;
        const int M = min(cb.nbr_count[s], cap);
        if (M <= P3_CHUNK && M > 1) item(s, 0, M, 0, 0);
        wk = __shfl_sync(FULL, wn, 0);
    }
    // longer lists: the chunk-pair items the neighbour kernel queued
    const unsigned int nlong = min(*cb.long_count, (unsigned int)cb.long_cap);
    if (lane == 0) wk = atomicAdd(cb.work_counter + 1, 1u);
    wk = __shfl_sync(FULL, wk, 0);
    while (wk < nlong) {
        unsigned int wn = 0;
        if (lane == 0) wn = atomicAdd(cb.work_counter + 1, 1u);
        const unsigned long long it = cb.long_items[wk];
        const int s = (int)TBMD_IX((int64_t)(it >> 32), n, BS_LONG_ITEM), I = (int)((it >> 16) & 0xffffu),
                  J = (int)(it & 0xffffu);
        const int M = min(cb.nbr_count[s], cap);
        const int mI = min(P3_CHUNK, M - I * P3_CHUNK);
        const int mJ = J != I ? min(P3_CHUNK, M - J * P3_CHUNK) : 0;
        item(s, I * P3_CHUNK, mI, J * P3_CHUNK, mJ);
        wk = __shfl_sync(FULL, wn, 0);
    }
    flush(cur_sys);
}
