// Layout of the reference's P-rank run (host only).  The GPU evaluates every triplet of the system
// in one process, so results do not depend on P; what P decides in the reference is which process
// grid is built and whether the run starts at all.  This file restates those decisions so that the
// drop-in executable (option -np P) and library callers stop, with the same message, where an
// `mpiexec -n P` run of the reference would.
//
//   process grid (P3BCA)    main.cpp:546-551, utility.cpp:96-107, CartTopology.cpp:6-57
//                           (above 1024 ranks the tables have no entry and the reference's run
//                           fails in CartTopology::Init; here that is TBMD_RANK_LAYOUT with a message)
//   local cell width        RegularGridDecomposition.cpp:24-32
//   cutoff boxes, check     P3BCA.cpp:29-70
//   shift steps             P3BCA.cpp:79-92
//   dummy padding (NATA, AUTA)  AtomDecomposition.cpp:15-41
#include <cmath>
#include <cstdio>
#include <cstring>
#include <sstream>
#include <string>

#include "tbmd.h"

namespace {

// The reference ships its process grids as a table for P = 1..1024 (utility/decompositions.hpp).
// Naive: {P}.  Optimal: every entry is the factorisation of P into one to three non-decreasing
// factors, each at least 3 unless the single factor is P itself, with the smallest sum of factors;
// among equal sums the first in increasing lexicographic order, except P = 360, listed as
// 6 x 6 x 10 (its other minimal-sum grid is 5 x 8 x 9).
constexpr int kMaxTableP = 1024;

int optimal_grid(int P, int d[3])
{
    if (P == 360) {
        d[0] = 6;
        d[1] = 6;
        d[2] = 10;
        return 3;
    }
    int best = 1, bsum = P;
    d[0] = P;
    d[1] = d[2] = 1;
    // two factors a <= b
    for (int a = 3; a * a <= P; ++a) {
        if (P % a) continue;
        const int b = P / a;
        if (a + b < bsum) {
            bsum = a + b;
            best = 2;
            d[0] = a;
            d[1] = b;
            d[2] = 1;
        }
    }
    // three factors a <= b <= c, visited after all two-factor grids and in increasing (a, b): a
    // strictly smaller sum replaces, an equal one does not
    for (int a = 3; a * a * a <= P; ++a) {
        if (P % a) continue;
        const int r = P / a;
        for (int b = a; b * b <= r; ++b) {
            if (r % b) continue;
            const int c = r / b;
            if (a + b + c < bsum) {
                bsum = a + b + c;
                best = 3;
                d[0] = a;
                d[1] = b;
                d[2] = c;
            }
        }
    }
    return best;
}

// std::ostream's default formatting of a double (6 significant digits, %g style), as the
// reference's std::cerr prints it
std::string g6(double v)
{
    std::ostringstream o;
    o << v;
    return o.str();
}

void put_msg(char *msg, int32_t len, const std::string &s)
{
    if (!msg || len <= 0) return;
    const size_t k = s.size() < (size_t)(len - 1) ? s.size() : (size_t)(len - 1);
    std::memcpy(msg, s.data(), k);
    msg[k] = 0;
}

}  // namespace

extern "C" tbmd_status tbmd_rank_layout_of(int32_t algorithm, int32_t world_size, int32_t optimal_decomposition,
                                           double cutoff, const double *L, int64_t n, tbmd_rank_layout *out,
                                           char *msg, int32_t msg_len)
{
    put_msg(msg, msg_len, "");
    if (!out || world_size < 1 || n < 0 || !std::isfinite(cutoff)) return TBMD_INVALID_ARG;
    if (algorithm != TBMD_NATA && algorithm != TBMD_AUTA && algorithm != TBMD_P3BCA) return TBMD_INVALID_ARG;
    std::memset(out, 0, sizeof(*out));
    out->world_size = world_size;
    out->dims[0] = world_size;
    out->dims[1] = out->dims[2] = 1;
    out->num_dims = 1;

    if (algorithm != TBMD_P3BCA) {
        // ring topology over all ranks; AtomDecomposition gives the first P - n mod P ranks
        // n / P particles plus one dummy when n mod P != 0, the others n / P + 1
        const int64_t P = world_size;
        out->particles_per_rank = n / P + (n % P != 0 ? 1 : 0);
        out->dummies = (n % P != 0) ? P - n % P : 0;
        return TBMD_OK;
    }

    if (!L || !(L[0] > 0.0) || !(L[1] > 0.0) || !(L[2] > 0.0)) return TBMD_INVALID_ARG;
    if (world_size > kMaxTableP) {
        // no table entry: Utility::getDecomposition returns an empty grid, whose first element
        // CartTopology::Init reads (CartTopology.cpp:10-12), so that run fails without a message
        out->num_dims = 0;
        put_msg(msg, msg_len, "no process grid for " + std::to_string(world_size) +
                                  " ranks: the reference's decomposition tables end at 1024");
        return TBMD_RANK_LAYOUT;
    }
    int d[3] = {world_size, 1, 1};
    out->num_dims = optimal_decomposition ? optimal_grid(world_size, d) : 1;
    for (int k = 0; k < 3; ++k) {
        out->dims[k] = d[k];
        out->cell_size[k] = L[k] / (double)d[k];
    }
    const int nd = out->num_dims;
    int *nCb = out->cutoff_boxes;
    nCb[0] = world_size == 1 ? 0 : (world_size == 2 ? 1 : (int)std::ceil(cutoff / out->cell_size[0]));
    nCb[1] = nd > 1 ? (int)std::ceil(cutoff / out->cell_size[1]) : 0;
    nCb[2] = nd > 2 ? (int)std::ceil(cutoff / out->cell_size[2]) : 0;
    switch (nd) {
        case 1: out->shift_steps = nCb[0] + 1; break;
        case 2: out->shift_steps = 2 * nCb[0] * nCb[1] + nCb[0] + nCb[1] + 1; break;
        default:
            out->shift_steps = 1 + nCb[2] + nCb[1] * (nCb[2] * 2 + 1) + nCb[0] * ((nCb[1] * 2 + 1) * (nCb[2] * 2 + 1));
    }
    // cutoff window: at least one cell and under half the grid per axis; the x axis is checked only
    // for more than two ranks
    static const char *axis[3] = {"dimX", "dimY", "dimZ"};
    for (int k = 0; k < nd; ++k) {
        if (k == 0 && world_size <= 2) continue;
        if (nCb[k] < 1 || (double)nCb[k] >= (double)d[k] / 2.0) {
            put_msg(msg, msg_len,
                    "invalid cutoff: " + g6(cutoff) + ", with " + std::to_string(nCb[k]) + " cutoff boxes, " +
                        axis[k] + ": " + std::to_string(d[k]) + ", and a cell size of " + g6(out->cell_size[k]));
            return TBMD_RANK_LAYOUT;
        }
    }
    return TBMD_OK;
}
