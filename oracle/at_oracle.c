/*
 * CPU oracle for the Axilrod-Teller three-body hot path of dmartin13/ThreeBodyMDAlgorithms.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the oracle the CUDA path is compared against; it is
 * never linked into the product library, and nothing in the product calls it.  Only tests/, the
 * smoke check and bench.py's CPU-baseline leg load it (through oracle/oracle.py).
 *
 * It is a plain-C restatement of the reference's algorithm at one rank:
 *   - per-triplet gradient          src/potential/AxilrodTeller.cpp:23-129
 *   - i<j<k triple loop + cutoff    src/algorithm/Algorithm.cpp:72-141 (cutoff test 94-100)
 *   - three buffer copies summed    src/algorithm/Algorithm.cpp:237-271 (SumUpParticles)
 *   - periodic squared distance     src/utility/structs.hpp:106-115 (GetSqrDistPeriodic)
 *   - domain size L (fixed at init) src/decomposition/RegularGridDecomposition.cpp:24-28, 135-166
 *   - predictor / update            src/utility/structs.hpp:40-55, 57-99
 *   - step loop                     src/simulation/Simulation.cpp:28-81
 * Single-threaded, it evaluates the triplets in the reference's order with the reference's
 * arithmetic, so it reproduces the reference built with -ffp-contract=off bit for bit (checked by
 * tests/test_oracle.py against oracle/_ref and the committed golden fixtures).  With more threads
 * the i-loop is split across threads and the per-thread buffers are summed in thread order.
 *
 * The cell-list variant enumerates exactly the same triplet set in the same order (it only skips
 * pairs that the exact test would reject anyway), so it serves as the oracle at sizes where the
 * reference's O(N^3) loop cannot run.
 *
 * Energy has no counterpart in the reference (it computes none); tbo_energy evaluates
 * E = nu * (1 + 3 cos g1 cos g2 cos g3) / (r1 r2 r3)^3 over the same triplet set, from dot
 * products, independently of the CUDA kernels' formulation.
 *
 * Build: gcc -O2 -fopenmp -ffp-contract=off -shared -fPIC at_oracle.c -o liboracle.so -lm
 */
#include <math.h>
#include <omp.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define TBO_CELL_MARGIN 1.000001 /* cell width >= cutoff * margin, so cutoff pairs are in adjacent cells */

/* RegularGridDecomposition::getDomainMinMax + Init (RegularGridDecomposition.cpp:135-166, 24-28):
 * lo = min - 1e-4, hi = max + 1e-4, L = |hi - lo| per axis, from the positions given. */
void tbo_domain(int64_t n, const double *x, const double *y, const double *z, double *L, double *lo)
{
    const double *p[3] = {x, y, z};
    for (int d = 0; d < 3; ++d) {
        double mn = 1.79769313486231570815e+308, mx = -1.79769313486231570815e+308;
        for (int64_t i = 0; i < n; ++i) {
            if (p[d][i] < mn) mn = p[d][i];
            if (p[d][i] > mx) mx = p[d][i];
        }
        double a = mn - 0.0001, b = mx + 0.0001;
        lo[d] = a;
        L[d] = fabs(b - a);
    }
}

/* Particle::GetSqrDistPeriodic (structs.hpp:106-115): per axis min(|d|, L - |d|), squared, summed. */
static inline double sqdist_periodic(double xa, double ya, double za, double xb, double yb, double zb,
                                     const double *L)
{
    double ax = fabs(xb - xa), ay = fabs(yb - ya), az = fabs(zb - za);
    double mx = fmin(ax, L[0] - ax), my = fmin(ay, L[1] - ay), mz = fmin(az, L[2] - az);
    return mx * mx + my * my + mz * mz;
}

/* One of the three radial derivatives of AxilrodTeller.cpp:68-81, (1/r) dV/dr for side r with the
 * other two sides s and t (the expression is symmetric in s and t).  Arguments are the powers
 * r^1..r^6, s^1..s^5, t^1..t^5; terms are summed in the reference's order. */
static inline double at_radial(double nu, const double *r, const double *s, const double *t)
{
    /* r[k] = r^k etc., index 0 unused */
    double sum = -8. / (r[4] * s[3] * t[3]) - 1. / (s[5] * t[5]) + 5. * s[1] / (r[6] * t[5]) +
                 5. * t[1] / (r[6] * s[5]) - 1. / (r[2] * s[3] * t[5]) - 1. / (r[2] * s[5] * t[3]) -
                 3. / (r[4] * s[1] * t[5]) - 3. / (r[4] * s[5] * t[1]) - 5. / (r[6] * s[1] * t[3]) -
                 5. / (r[6] * s[3] * t[1]) + 6. / (r[4] * s[3] * t[3]);
    return (3. * nu / (8. * r[1])) * sum;
}

static inline void powers(double d, double *pw)
{
    pw[1] = d;
    pw[2] = pw[1] * d;
    pw[3] = pw[2] * d;
    pw[4] = pw[3] * d;
    pw[5] = pw[4] * d;
    pw[6] = pw[5] * d;
}

/* AxilrodTeller::CalculateForces (AxilrodTeller.cpp:23-129): the amounts the reference subtracts
 * from f of i, j and k.  The stored force is therefore +grad E (checked by finite differences). */
static inline void at_triplet(double nu, double xi, double yi, double zi, double xj, double yj, double zj, double xk,
                              double yk, double zk, double *ci, double *cj, double *ck)
{
    /* sides a = j - i, b = i - k, c = j - k and their lengths (Eigen norm: sqrt((x^2 + y^2) + z^2)) */
    double ax = xj - xi, ay = yj - yi, az = zj - zi;
    double bx = xi - xk, by = yi - yk, bz = zi - zk;
    double cx = xj - xk, cy = yj - yk, cz = zj - zk;
    double pa[7], pb[7], pc[7];
    powers(sqrt((ax * ax + ay * ay) + az * az), pa);
    powers(sqrt((bx * bx + by * by) + bz * bz), pb);
    powers(sqrt((cx * cx + cy * cy) + cz * cz), pc);

    /* component differences dXa = j - i, dXb = k - i, dXc = k - j */
    double dxa = xj - xi, dya = yj - yi, dza = zj - zi;
    double dxb = xk - xi, dyb = yk - yi, dzb = zk - zi;
    double dxc = xk - xj, dyc = yk - yj, dzc = zk - zj;

    double ra = at_radial(nu, pa, pb, pc);
    double rb = at_radial(nu, pb, pa, pc);
    double rc = at_radial(nu, pc, pb, pa);

    ci[0] = dxa * ra + dxb * rb;
    ci[1] = dya * ra + dyb * rb;
    ci[2] = dza * ra + dzb * rb;
    cj[0] = dxa * (-ra) + dxc * rc;
    cj[1] = dya * (-ra) + dyc * rc;
    cj[2] = dza * (-ra) + dzc * rc;
    ck[0] = dxb * (-rb) + dxc * (-rc);
    ck[1] = dyb * (-rb) + dyc * (-rc);
    ck[2] = dzb * (-rb) + dzc * (-rc);
}

/* Accumulation buffers: the reference subtracts into three copies b0, b1, b2 of the particle
 * vector and adds them as f = f0 + (f1 + f2) afterwards (Algorithm.cpp:245-248). */
typedef struct {
    double *f0, *f1, *f2; /* each 3*n, interleaved xyz */
} tbo_bufs;

static int bufs_alloc(tbo_bufs *b, int64_t n)
{
    b->f0 = (double *)calloc((size_t)(9 * n), sizeof(double));
    if (!b->f0) return -1;
    b->f1 = b->f0 + 3 * n;
    b->f2 = b->f1 + 3 * n;
    return 0;
}

static inline void apply_triplet(double nu, const double *x, const double *y, const double *z, int64_t i, int64_t j,
                                 int64_t k, tbo_bufs *b)
{
    double ci[3], cj[3], ck[3];
    at_triplet(nu, x[i], y[i], z[i], x[j], y[j], z[j], x[k], y[k], z[k], ci, cj, ck);
    for (int d = 0; d < 3; ++d) {
        b->f0[3 * i + d] -= ci[d];
        b->f1[3 * j + d] -= cj[d];
        b->f2[3 * k + d] -= ck[d];
    }
}

/* Sum per-thread buffers in thread order, then f = f0 + (f1 + f2) per particle. */
static void reduce_bufs(tbo_bufs *tb, int nt, int64_t n, double *fx, double *fy, double *fz)
{
    for (int t = 1; t < nt; ++t)
        for (int64_t q = 0; q < 9 * n; ++q) tb[0].f0[q] += tb[t].f0[q];
    for (int64_t i = 0; i < n; ++i) {
        fx[i] = tb[0].f0[3 * i + 0] + (tb[0].f1[3 * i + 0] + tb[0].f2[3 * i + 0]);
        fy[i] = tb[0].f0[3 * i + 1] + (tb[0].f1[3 * i + 1] + tb[0].f2[3 * i + 1]);
        fz[i] = tb[0].f0[3 * i + 2] + (tb[0].f1[3 * i + 2] + tb[0].f2[3 * i + 2]);
    }
}

static int clamp_threads(int nthreads)
{
    if (nthreads <= 0) nthreads = omp_get_max_threads();
    if (nthreads < 1) nthreads = 1;
    return nthreads;
}

/* Algorithm::calculateInteractions with b0 = b1 = b2 and one owner (Algorithm.cpp:72-141):
 * i < j < k, cutoff test only when cutoff > 0, a triplet is skipped iff some pair has
 * periodic d^2 > cutoff^2 (so d == cutoff is inside).  Returns the triplet count; forces are
 * overwritten.  Returns UINT64_MAX on allocation failure. */
uint64_t tbo_forces_bruteforce(int64_t n, const double *x, const double *y, const double *z, double nu, double cutoff,
                               const double *L, double *fx, double *fy, double *fz, int nthreads)
{
    nthreads = clamp_threads(nthreads);
    tbo_bufs *tb = (tbo_bufs *)calloc((size_t)nthreads, sizeof(tbo_bufs));
    if (!tb) return UINT64_MAX;
    int fail = 0;
    for (int t = 0; t < nthreads; ++t) fail |= bufs_alloc(&tb[t], n);
    if (fail) return UINT64_MAX;
    double sq = cutoff * cutoff;
    uint64_t total = 0;
#pragma omp parallel num_threads(nthreads) reduction(+ : total)
    {
        tbo_bufs *b = &tb[omp_get_thread_num()];
#pragma omp for schedule(dynamic, 1)
        for (int64_t i = 0; i < n; ++i) {
            for (int64_t j = i + 1; j < n; ++j) {
                for (int64_t k = j + 1; k < n; ++k) {
                    if (cutoff > 0) {
                        if (sqdist_periodic(x[i], y[i], z[i], x[j], y[j], z[j], L) > sq ||
                            sqdist_periodic(x[i], y[i], z[i], x[k], y[k], z[k], L) > sq ||
                            sqdist_periodic(x[j], y[j], z[j], x[k], y[k], z[k], L) > sq)
                            continue;
                    }
                    apply_triplet(nu, x, y, z, i, j, k, b);
                    total++;
                }
            }
        }
    }
    reduce_bufs(tb, nthreads, n, fx, fy, fz);
    for (int t = 0; t < nthreads; ++t) free(tb[t].f0);
    free(tb);
    return total;
}

/* Cell grid used to enumerate cutoff pairs.  Per axis n_d = floor(L_d / (cutoff * margin)); if
 * that is below 3 the axis gets a single cell (all its particles are candidates).  A particle's
 * cell coordinate is floor((x - lo) / (L / n)) wrapped into [0, n), so particles that drifted out of
 * the initial box are wrapped periodically.  The CUDA cell build uses the same arithmetic (no FMA
 * contraction), so cell assignments match bit for bit. */
void tbo_cell_dims(const double *L, double cutoff, int *dims, double *width)
{
    for (int d = 0; d < 3; ++d) {
        double m = floor(L[d] / (cutoff * TBO_CELL_MARGIN));
        int nd = (m >= 3.0) ? (m > 1024.0 ? 1024 : (int)m) : 1;
        dims[d] = nd;
        width[d] = L[d] / (double)nd;
    }
}

/* A non-finite coordinate lands in cell 0 (same rule as the CUDA cell build). */
static inline int cell_coord(double x, double lo, double w, int nd)
{
    double t = floor((x - lo) / w);
    double m = fmod(t, (double)nd);
    if (m < 0) m += (double)nd;
    if (!(m >= 0.0 && m < (double)nd)) return 0;
    return (int)m;
}

void tbo_cell_assign(int64_t n, const double *x, const double *y, const double *z, double cutoff, const double *L,
                     const double *lo, int *dims, int32_t *cell)
{
    double w[3];
    tbo_cell_dims(L, cutoff, dims, w);
    for (int64_t i = 0; i < n; ++i) {
        int cx = cell_coord(x[i], lo[0], w[0], dims[0]);
        int cy = cell_coord(y[i], lo[1], w[1], dims[1]);
        int cz = cell_coord(z[i], lo[2], w[2], dims[2]);
        cell[i] = (int32_t)((cz * dims[1] + cy) * dims[0] + cx);
    }
}

/* Half neighbour lists in original index order: for each i, the ascending list of j > i with
 * periodic d^2 <= cutoff^2.  CSR layout (start[n+1], nbr[]).  Returns 0 on success. */
static int build_half_lists(int64_t n, const double *x, const double *y, const double *z, double cutoff,
                            const double *L, const double *lo, int64_t **start_out, int64_t **nbr_out, int nthreads)
{
    int dims[3];
    double w[3];
    tbo_cell_dims(L, cutoff, dims, w);
    int64_t ncell = (int64_t)dims[0] * dims[1] * dims[2];
    int32_t *cell = (int32_t *)malloc((size_t)n * sizeof(int32_t));
    int64_t *cstart = (int64_t *)calloc((size_t)(ncell + 1), sizeof(int64_t));
    int64_t *members = (int64_t *)malloc((size_t)n * sizeof(int64_t));
    int64_t *cnt = (int64_t *)calloc((size_t)(n + 1), sizeof(int64_t));
    if (!cell || !cstart || !members || !cnt) return -1;
    tbo_cell_assign(n, x, y, z, cutoff, L, lo, dims, cell);
    for (int64_t i = 0; i < n; ++i) cstart[cell[i] + 1]++;
    for (int64_t c = 0; c < ncell; ++c) cstart[c + 1] += cstart[c];
    {
        int64_t *fill = (int64_t *)malloc((size_t)ncell * sizeof(int64_t));
        if (!fill) return -1;
        memcpy(fill, cstart, (size_t)ncell * sizeof(int64_t));
        for (int64_t i = 0; i < n; ++i) members[fill[cell[i]]++] = i; /* ascending i within a cell */
        free(fill);
    }
    double sq = cutoff * cutoff;
    int ox[3] = {-1, 0, 1};
    /* two passes: count, then fill; neighbour cells are de-duplicated for axes with one cell */
    int64_t *start = NULL, *nbr = NULL;
    for (int pass = 0; pass < 2; ++pass) {
#pragma omp parallel for schedule(dynamic, 64) num_threads(clamp_threads(nthreads))
        for (int64_t i = 0; i < n; ++i) {
            int c = cell[i];
            int cxi = c % dims[0], cyi = (c / dims[0]) % dims[1], czi = c / (dims[0] * dims[1]);
            int64_t m = 0;
            int64_t *dst = pass ? nbr + start[i] : NULL;
            for (int a = 0; a < 3; ++a) {
                if (dims[2] == 1 && a != 1) continue;
                for (int b = 0; b < 3; ++b) {
                    if (dims[1] == 1 && b != 1) continue;
                    for (int e = 0; e < 3; ++e) {
                        if (dims[0] == 1 && e != 1) continue;
                        int nx = (cxi + ox[e] + dims[0]) % dims[0];
                        int ny = (cyi + ox[b] + dims[1]) % dims[1];
                        int nz = (czi + ox[a] + dims[2]) % dims[2];
                        int64_t nc = ((int64_t)nz * dims[1] + ny) * dims[0] + nx;
                        for (int64_t q = cstart[nc]; q < cstart[nc + 1]; ++q) {
                            int64_t j = members[q];
                            if (j <= i) continue;
                            if (sqdist_periodic(x[i], y[i], z[i], x[j], y[j], z[j], L) > sq) continue;
                            if (pass) dst[m] = j;
                            m++;
                        }
                    }
                }
            }
            if (!pass) cnt[i + 1] = m;
        }
        if (!pass) {
            for (int64_t i = 0; i < n; ++i) cnt[i + 1] += cnt[i];
            start = cnt;
            nbr = (int64_t *)malloc((size_t)(start[n] > 0 ? start[n] : 1) * sizeof(int64_t));
            if (!nbr) return -1;
        }
    }
    /* sort each list ascending so the triplet order equals the reference's i<j<k order */
#pragma omp parallel for schedule(dynamic, 256) num_threads(clamp_threads(nthreads))
    for (int64_t i = 0; i < n; ++i) {
        int64_t *l = nbr + start[i];
        int64_t len = start[i + 1] - start[i];
        for (int64_t p = 1; p < len; ++p) {
            int64_t v = l[p], q = p - 1;
            while (q >= 0 && l[q] > v) {
                l[q + 1] = l[q];
                q--;
            }
            l[q + 1] = v;
        }
    }
    free(cell);
    free(cstart);
    free(members);
    *start_out = start;
    *nbr_out = nbr;
    return 0;
}

/* Same triplet set and order as tbo_forces_bruteforce with cutoff > 0, via half neighbour lists. */
uint64_t tbo_forces_cells(int64_t n, const double *x, const double *y, const double *z, double nu, double cutoff,
                          const double *L, const double *lo, double *fx, double *fy, double *fz, int nthreads)
{
    if (!(cutoff > 0)) return tbo_forces_bruteforce(n, x, y, z, nu, cutoff, L, fx, fy, fz, nthreads);
    nthreads = clamp_threads(nthreads);
    int64_t *start, *nbr;
    if (build_half_lists(n, x, y, z, cutoff, L, lo, &start, &nbr, nthreads)) return UINT64_MAX;
    tbo_bufs *tb = (tbo_bufs *)calloc((size_t)nthreads, sizeof(tbo_bufs));
    if (!tb) return UINT64_MAX;
    int fail = 0;
    for (int t = 0; t < nthreads; ++t) fail |= bufs_alloc(&tb[t], n);
    if (fail) return UINT64_MAX;
    double sq = cutoff * cutoff;
    uint64_t total = 0;
#pragma omp parallel num_threads(nthreads) reduction(+ : total)
    {
        tbo_bufs *b = &tb[omp_get_thread_num()];
#pragma omp for schedule(dynamic, 16)
        for (int64_t i = 0; i < n; ++i) {
            const int64_t *l = nbr + start[i];
            int64_t len = start[i + 1] - start[i];
            for (int64_t p = 0; p < len; ++p) {
                int64_t j = l[p];
                for (int64_t q = p + 1; q < len; ++q) {
                    int64_t k = l[q];
                    if (sqdist_periodic(x[j], y[j], z[j], x[k], y[k], z[k], L) > sq) continue;
                    apply_triplet(nu, x, y, z, i, j, k, b);
                    total++;
                }
            }
        }
    }
    reduce_bufs(tb, nthreads, n, fx, fy, fz);
    for (int t = 0; t < nthreads; ++t) free(tb[t].f0);
    free(tb);
    free(start);
    free(nbr);
    return total;
}

/* Neumaier's compensated addition: *sum + *err carries the exact running total to working precision. */
static inline void neumaier_add(double *sum, double *err, double v)
{
    const double t = *sum + v;
    if (fabs(*sum) >= fabs(v))
        *err += (*sum - t) + v;
    else
        *err += (v - t) + *sum;
    *sum = t;
}

/* Stored force (+grad E) on each of the nsel particles sel[] from every triplet that contains it,
 * with no cutoff: NATA's view of one particle (NATA.cpp:27-55 sums, for particle i, the triplets
 * it takes part in).  Each triplet {p, j, k} is evaluated with the reference's arithmetic in its
 * sorted order a < b < c (at_triplet, AxilrodTeller.cpp:23-129), and p's share is the amount the
 * reference subtracts for p's role; the three roles are summed like SumUpParticles
 * (Algorithm.cpp:245-248): f = f0 + (f1 + f2).  O(n^2) per particle, so the C(n,3) force of a few
 * particles of a large system can be pinned without the whole O(n^3) loop.  The sums are compensated
 * (Neumaier: a running sum and a running rounding error per role and component; threads split the
 * j loop and their compensated partial sums are merged the same way), so the result does not depend
 * on the summation order to working precision.  Plain FP64 sums of the 3.4e7 terms of one particle
 * at n = 8192 cancel heavily and move by about 1e-11 relative between summation orders. */
void tbo_forces_selected(int64_t n, const double *x, const double *y, const double *z, double nu,
                         const int64_t *sel, int64_t nsel, double *fx, double *fy, double *fz, int nthreads)
{
    nthreads = clamp_threads(nthreads);
    double *part = (double *)calloc((size_t)(18 * nthreads), sizeof(double));
    if (!part) return;
    for (int64_t s = 0; s < nsel; ++s) {
        const int64_t p = sel[s];
        memset(part, 0, sizeof(double) * 18 * (size_t)nthreads);
#pragma omp parallel num_threads(nthreads)
        {
            double *acc = part + 18 * omp_get_thread_num(); /* sums [role][xyz], then their errors */
#pragma omp for schedule(dynamic, 8)
            for (int64_t j = 0; j < n; ++j) {
                if (j == p) continue;
                for (int64_t k = j + 1; k < n; ++k) {
                    if (k == p) continue;
                    int64_t a = p, b = j, c = k; /* sort into a < b < c, remembering p's role */
                    int role;
                    if (p < j) {
                        role = 0;
                    } else if (p < k) {
                        a = j;
                        b = p;
                        role = 1;
                    } else {
                        a = j;
                        b = k;
                        c = p;
                        role = 2;
                    }
                    double ci[3], cj[3], ck[3];
                    at_triplet(nu, x[a], y[a], z[a], x[b], y[b], z[b], x[c], y[c], z[c], ci, cj, ck);
                    const double *cp = role == 0 ? ci : (role == 1 ? cj : ck);
                    for (int d = 0; d < 3; ++d) neumaier_add(&acc[3 * role + d], &acc[9 + 3 * role + d], -cp[d]);
                }
            }
        }
        for (int t = 1; t < nthreads; ++t)
            for (int q = 0; q < 9; ++q) {
                neumaier_add(&part[q], &part[9 + q], part[18 * t + q]);
                neumaier_add(&part[q], &part[9 + q], part[18 * t + 9 + q]);
            }
        double r[9];
        for (int q = 0; q < 9; ++q) r[q] = part[q] + part[9 + q];
        fx[s] = r[0] + (r[3] + r[6]);
        fy[s] = r[1] + (r[4] + r[7]);
        fz[s] = r[2] + (r[5] + r[8]);
    }
    free(part);
}

/* Triplet energy from dot products: u = xj - xi, v = xk - xi, w = xk - xj,
 * cos_i cos_j cos_k = -(u.v)(u.w)(v.w) / (|u|^2 |v|^2 |w|^2). */
/* scale = 0: the triplet energy nu (1 + 3 cos cos cos) / (r1 r2 r3)^3.
 * scale = 1: its magnitude scale |nu| (1 + 3 |cos cos cos|) / (r1 r2 r3)^3, the size of both parts of
 * the term, against which a rounding error in the geometry is measured. */
static inline double at_energy_s(double nu, const double *x, const double *y, const double *z, int64_t i,
                                 int64_t j, int64_t k, int scale)
{
    double ux = x[j] - x[i], uy = y[j] - y[i], uz = z[j] - z[i];
    double vx = x[k] - x[i], vy = y[k] - y[i], vz = z[k] - z[i];
    double wx = x[k] - x[j], wy = y[k] - y[j], wz = z[k] - z[j];
    double uu = ux * ux + uy * uy + uz * uz, vv = vx * vx + vy * vy + vz * vz, ww = wx * wx + wy * wy + wz * wz;
    double uv = ux * vx + uy * vy + uz * vz, uw = ux * wx + uy * wy + uz * wz, vw = vx * wx + vy * wy + vz * wz;
    double cosprod = -(uv * uw * vw) / (uu * vv * ww);
    double r3 = sqrt(uu * vv * ww);
    if (scale) return fabs(nu) * (1.0 + 3.0 * fabs(cosprod)) / (r3 * r3 * r3);
    return nu * (1.0 + 3.0 * cosprod) / (r3 * r3 * r3);
}
static inline double at_energy(double nu, const double *x, const double *y, const double *z, int64_t i, int64_t j,
                               int64_t k)
{
    return at_energy_s(nu, x, y, z, i, j, k, 0);
}

/* Total AT energy over the triplet set of tbo_forces_* (cells used when cutoff > 0). */
/* Sum over the triplet set of E_t (absval = 0) or of the magnitude scales of at_energy_s (absval =
 * 1).  The second is the scale of the energy's rounding error: the terms have both signs
 * (1 + 3 cos cos cos < 0 for nearly collinear triplets), so |sum E_t| can be much smaller. */
static double energy_sum(int64_t n, const double *x, const double *y, const double *z, double nu, double cutoff,
                         const double *L, const double *lo, int nthreads, int absval)
{
    nthreads = clamp_threads(nthreads);
    double e = 0.0;
    if (cutoff > 0) {
        int64_t *start, *nbr;
        if (build_half_lists(n, x, y, z, cutoff, L, lo, &start, &nbr, nthreads)) return NAN;
        double sq = cutoff * cutoff;
#pragma omp parallel for schedule(dynamic, 16) num_threads(nthreads) reduction(+ : e)
        for (int64_t i = 0; i < n; ++i) {
            const int64_t *l = nbr + start[i];
            int64_t len = start[i + 1] - start[i];
            for (int64_t p = 0; p < len; ++p)
                for (int64_t q = p + 1; q < len; ++q) {
                    int64_t j = l[p], k = l[q];
                    if (sqdist_periodic(x[j], y[j], z[j], x[k], y[k], z[k], L) > sq) continue;
                    e += at_energy_s(nu, x, y, z, i, j, k, absval);
                }
        }
        free(start);
        free(nbr);
    } else {
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads) reduction(+ : e)
        for (int64_t i = 0; i < n; ++i)
            for (int64_t j = i + 1; j < n; ++j)
                for (int64_t k = j + 1; k < n; ++k) {
                    e += at_energy_s(nu, x, y, z, i, j, k, absval);
                }
    }
    return e;
}

double tbo_energy(int64_t n, const double *x, const double *y, const double *z, double nu, double cutoff,
                  const double *L, const double *lo, int nthreads)
{
    return energy_sum(n, x, y, z, nu, cutoff, L, lo, nthreads, 0);
}

double tbo_energy_abs(int64_t n, const double *x, const double *y, const double *z, double nu, double cutoff,
                      const double *L, const double *lo, int nthreads)
{
    return energy_sum(n, x, y, z, nu, cutoff, L, lo, nthreads, 1);
}

/* Particle::UpdatePredictorStage (structs.hpp:40-55): x += v*dt + (aX, aX, aX) * (dt*dt*0.5).
 * The acceleration vector is built from aX three times, as in the reference. */
void tbo_predictor(int64_t n, double *x, double *y, double *z, const double *vx, const double *vy, const double *vz,
                   const double *ax, double dt)
{
    double h = dt * dt * 0.5;
    for (int64_t i = 0; i < n; ++i) {
        double a = ax[i];
        x[i] = (x[i] + vx[i] * dt) + a * h;
        y[i] = (y[i] + vy[i] * dt) + a * h;
        z[i] = (z[i] + vz[i] * dt) + a * h;
    }
}

/* Particle::Update (structs.hpp:57-99): a = g - f/m; v += a * (dt*0.5); positions unchanged. */
void tbo_update(int64_t n, double *vx, double *vy, double *vz, double *ax, double *ay, double *az, const double *fx,
                const double *fy, const double *fz, const double *m, double dt, const double *g)
{
    double h = dt * 0.5;
    for (int64_t i = 0; i < n; ++i) {
        double nx = g[0] - fx[i] / m[i], ny = g[1] - fy[i] / m[i], nz = g[2] - fz[i] / m[i];
        vx[i] = vx[i] + nx * h;
        vy[i] = vy[i] + ny * h;
        vz[i] = vz[i] + nz * h;
        ax[i] = nx;
        ay[i] = ny;
        az[i] = nz;
    }
}

/* Simulation::Start at one rank (Simulation.cpp:28-81): per step predictor, force reset + triplet
 * forces, update.  algorithm: 0 = NATA, 1 = P3BCA, 2 = AUTA (enums.hpp numbering).  NATA and AUTA
 * use no cutoff (Algorithm.cpp:26-32); P3BCA uses the cutoff with L from the INITIAL positions
 * (RegularGridDecomposition::Init), fixed for the run.  counts[step] receives the triplet count.
 * All arrays are updated in place.  Returns 0, or -1 on allocation failure. */
int tbo_simulate(int algorithm, int iterations, int64_t n, double *x, double *y, double *z, double *vx, double *vy,
                 double *vz, double *ax, double *ay, double *az, double *fx, double *fy, double *fz, const double *m,
                 double dt, const double *g, double cutoff, double nu, uint64_t *counts, int nthreads)
{
    double L[3] = {-1, -1, -1}, lo[3] = {0, 0, 0};
    int use_cut = (algorithm == 1) && cutoff > 0;
    if (algorithm == 1) tbo_domain(n, x, y, z, L, lo);
    for (int it = 0; it < iterations; ++it) {
        tbo_predictor(n, x, y, z, vx, vy, vz, ax, dt);
        uint64_t c = use_cut ? tbo_forces_cells(n, x, y, z, nu, cutoff, L, lo, fx, fy, fz, nthreads)
                             : tbo_forces_bruteforce(n, x, y, z, nu, -1.0, L, fx, fy, fz, nthreads);
        if (c == UINT64_MAX) return -1;
        counts[it] = c;
        tbo_update(n, vx, vy, vz, ax, ay, az, fx, fy, fz, m, dt, g);
    }
    return 0;
}
