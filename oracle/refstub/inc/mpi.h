/*
 * Single-rank stand-in for the MPI C API, written for this repository.
 *
 * Test infrastructure only: it exists so that the reference's own hot-path
 * sources (src/simulation, src/algorithm, src/potential, src/decomposition,
 * src/topology, src/utility of dmartin13/ThreeBodyMDAlgorithms) compile and run
 * as ONE rank without an MPI installation.  With one rank every collective is a
 * local copy, every barrier is a no-op, a Cartesian or ring shift targets the
 * caller itself (MPI_Sendrecv_replace to self leaves the buffer unchanged), and
 * point-to-point messages to another rank cannot occur.  The reference only
 * reaches MPI_Send/Recv/Isend/Irecv/Probe when its buffer owner differs from the
 * rank (P3BCA.cpp:415-504, AUTA.cpp:144-234, RegularGridDecomposition.cpp:50-123),
 * which never happens at one rank; those entry points abort loudly if reached.
 *
 * Datatypes are small integers into a registry that records the extent, so that
 * MPI_Gather/Gatherv of the reference's Particle struct (structs.hpp:124-155)
 * copy the right number of bytes.
 *
 * Layout mode (the ref_layout driver): with TBMD_STUB_WORLD_SIZE=P and TBMD_STUB_RANK=r in the
 * environment the world has P ranks and this process is rank r, so that the reference's set-up
 * code (topologies, decompositions, Algorithm::Init) lays out a P-rank run for rank r.  Cartesian
 * coordinates are row-major, as MPI defines them.  Set-up exchanges no message; every call that
 * would move data between ranks aborts in this mode.  Without the variables the world is one rank.
 */
#ifndef TBMD_REFSTUB_MPI_H
#define TBMD_REFSTUB_MPI_H

#include <stddef.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Request;
typedef int MPI_Info;
typedef int MPI_Op;
typedef ptrdiff_t MPI_Aint;
typedef struct {
    int MPI_SOURCE;
    int MPI_TAG;
    int MPI_ERROR;
    int count_bytes;
} MPI_Status;

#define MPI_SUCCESS 0
#define MPI_COMM_WORLD 1
#define MPI_COMM_NULL 0
#define MPI_INFO_NULL 0
#define MPI_ANY_SOURCE (-1)
#define MPI_ANY_TAG (-1)
#define MPI_ROOT (-3)
#define MPI_STATUS_IGNORE ((MPI_Status *)0)
#define MPI_STATUSES_IGNORE ((MPI_Status *)0)
#define MPI_ERRCODES_IGNORE ((int *)0)
#define MPI_SUM 1
#define MPI_MAX 2

/* builtin datatypes: index into the extent registry */
#define MPI_CHAR 1
#define MPI_INT 2
#define MPI_DOUBLE 3
#define MPI_C_BOOL 4
#define MPI_UNSIGNED_LONG 5
#define MPI_INT64_T 6
#define MPI_UINT64_T 7
#define MPI_UINT 8
#define MPI_UNSIGNED 8
#define TBMD_STUB_FIRST_DERIVED 16
#define TBMD_STUB_MAX_TYPES 64

/* One registry for the whole program: C++ inline functions share their static locals across
 * translation units (the reference registers its Particle type in main.cpp and uses it in
 * Simulation.cpp). */
inline MPI_Aint *tbmd_stub_extents(void)
{
    static MPI_Aint ext[TBMD_STUB_MAX_TYPES] = {0, 1, 4, 8, 1, 8, 8, 8, 4};
    return ext;
}
inline int *tbmd_stub_next_type(void)
{
    static int next = TBMD_STUB_FIRST_DERIVED;
    return &next;
}
static inline MPI_Aint tbmd_stub_extent(MPI_Datatype t)
{
    if (t <= 0 || t >= TBMD_STUB_MAX_TYPES || tbmd_stub_extents()[t] == 0) {
        fprintf(stderr, "mpi stub: unknown datatype %d\n", t);
        abort();
    }
    return tbmd_stub_extents()[t];
}
static inline int tbmd_stub_unreachable(const char *what)
{
    fprintf(stderr, "mpi stub: %s needs a second rank, which a single-rank run never has\n", what);
    abort();
    return 1;
}

/* world size and own rank: {1, 0}, or the layout-mode environment */
inline const int *tbmd_stub_world(void)
{
    static int w[2] = {-1, -1};
    if (w[0] < 0) {
        const char *ps = getenv("TBMD_STUB_WORLD_SIZE"), *rs = getenv("TBMD_STUB_RANK");
        const int P = ps ? atoi(ps) : 1, r = rs ? atoi(rs) : 0;
        if (P < 1 || r < 0 || r >= P) {
            fprintf(stderr, "mpi stub: bad TBMD_STUB_WORLD_SIZE / TBMD_STUB_RANK\n");
            abort();
        }
        w[0] = P;
        w[1] = r;
    }
    return w;
}
/* the Cartesian grid of the last MPI_Cart_create: {ndims, d0, d1, d2} */
inline int *tbmd_stub_cart(void)
{
    static int d[4] = {1, 1, 1, 1};
    return d;
}
static inline void tbmd_stub_one_rank(const char *what)
{
    if (tbmd_stub_world()[0] > 1) {
        fprintf(stderr, "mpi stub: %s moves data between ranks; layout mode runs set-up only\n", what);
        abort();
    }
}

static inline int MPI_Init(int *argc, char ***argv) { (void)argc; (void)argv; return MPI_SUCCESS; }
static inline int MPI_Finalize(void) { return MPI_SUCCESS; }
static inline int MPI_Initialized(int *flag) { *flag = 1; return MPI_SUCCESS; }
static inline int MPI_Finalized(int *flag) { *flag = 0; return MPI_SUCCESS; }
static inline int MPI_Comm_size(MPI_Comm c, int *size) { (void)c; *size = tbmd_stub_world()[0]; return MPI_SUCCESS; }
static inline int MPI_Comm_rank(MPI_Comm c, int *rank) { (void)c; *rank = tbmd_stub_world()[1]; return MPI_SUCCESS; }
static inline int MPI_Comm_dup(MPI_Comm c, MPI_Comm *out) { *out = c; return MPI_SUCCESS; }
static inline int MPI_Comm_free(MPI_Comm *c) { *c = MPI_COMM_NULL; return MPI_SUCCESS; }
static inline int MPI_Comm_get_parent(MPI_Comm *parent) { *parent = MPI_COMM_NULL; return MPI_SUCCESS; }
static inline int MPI_Barrier(MPI_Comm c) { (void)c; return MPI_SUCCESS; }

/* Struct extent = end of the last member rounded up to the largest member alignment (at most 8 here). */
static inline int MPI_Type_create_struct(int count, const int *blocklengths, const MPI_Aint *offsets,
                                         const MPI_Datatype *types, MPI_Datatype *newtype)
{
    MPI_Aint end = 0, align = 1;
    for (int i = 0; i < count; ++i) {
        MPI_Aint e = tbmd_stub_extent(types[i]);
        MPI_Aint stop = offsets[i] + e * blocklengths[i];
        if (stop > end) end = stop;
        if (e > align) align = e;
    }
    end = (end + align - 1) / align * align;
    int id = (*tbmd_stub_next_type())++;
    if (id >= TBMD_STUB_MAX_TYPES) return tbmd_stub_unreachable("too many derived datatypes");
    tbmd_stub_extents()[id] = end;
    *newtype = id;
    return MPI_SUCCESS;
}
static inline int MPI_Type_commit(MPI_Datatype *t) { (void)t; return MPI_SUCCESS; }
static inline int MPI_Type_free(MPI_Datatype *t) { (void)t; return MPI_SUCCESS; }

static inline int MPI_Gather(const void *sb, int sc, MPI_Datatype st, void *rb, int rc, MPI_Datatype rt, int root,
                             MPI_Comm c)
{
    (void)rc; (void)rt; (void)root; (void)c;
    tbmd_stub_one_rank("MPI_Gather");
    if (rb && sb && sc > 0) memcpy(rb, sb, (size_t)(sc * tbmd_stub_extent(st)));
    return MPI_SUCCESS;
}
static inline int MPI_Gatherv(const void *sb, int sc, MPI_Datatype st, void *rb, const int *rcs, const int *displs,
                              MPI_Datatype rt, int root, MPI_Comm c)
{
    (void)rcs; (void)root; (void)c;
    tbmd_stub_one_rank("MPI_Gatherv");
    if (rb && sb && sc > 0)
        memcpy((char *)rb + displs[0] * tbmd_stub_extent(rt), sb, (size_t)(sc * tbmd_stub_extent(st)));
    return MPI_SUCCESS;
}
static inline int MPI_Allreduce(const void *sb, void *rb, int count, MPI_Datatype t, MPI_Op op, MPI_Comm c)
{
    (void)op; (void)c;
    tbmd_stub_one_rank("MPI_Allreduce");
    if (sb != rb) memcpy(rb, sb, (size_t)(count * tbmd_stub_extent(t)));
    return MPI_SUCCESS;
}
static inline int MPI_Bcast(void *b, int count, MPI_Datatype t, int root, MPI_Comm c)
{
    (void)b; (void)count; (void)t; (void)root; (void)c;
    tbmd_stub_one_rank("MPI_Bcast");
    return MPI_SUCCESS;
}

/* Cartesian topology: periodic, row-major (the last coordinate varies fastest).  With one rank
 * every coordinate is 0 and every shift returns the caller. */
static inline int MPI_Cart_create(MPI_Comm old, int nd, const int *dims, const int *periods, int reorder,
                                  MPI_Comm *cart)
{
    (void)periods; (void)reorder;
    int *g = tbmd_stub_cart();
    int prod = 1;
    g[0] = nd;
    for (int i = 0; i < 3; ++i) g[1 + i] = i < nd ? dims[i] : 1;
    for (int i = 0; i < nd; ++i) prod *= dims[i];
    if (nd < 1 || nd > 3 || prod != tbmd_stub_world()[0]) {
        fprintf(stderr, "mpi stub: Cartesian grid does not match the world size\n");
        abort();
    }
    *cart = old;
    return MPI_SUCCESS;
}
static inline int MPI_Cart_coords(MPI_Comm c, int rank, int nd, int *coords)
{
    (void)c;
    const int *g = tbmd_stub_cart();
    for (int i = nd - 1; i >= 0; --i) {
        coords[i] = rank % g[1 + i];
        rank /= g[1 + i];
    }
    return MPI_SUCCESS;
}
static inline int MPI_Cart_rank(MPI_Comm c, const int *coords, int *rank)
{
    (void)c;
    const int *g = tbmd_stub_cart();
    int r = 0;
    for (int i = 0; i < g[0]; ++i) r = r * g[1 + i] + ((coords[i] % g[1 + i]) + g[1 + i]) % g[1 + i];
    *rank = r;
    return MPI_SUCCESS;
}
static inline int MPI_Cart_shift(MPI_Comm c, int dir, int disp, int *src, int *dst)
{
    const int *g = tbmd_stub_cart();
    int co[3] = {0, 0, 0};
    MPI_Cart_coords(c, tbmd_stub_world()[1], g[0], co);
    const int k = co[dir];
    co[dir] = k + disp;
    MPI_Cart_rank(c, co, dst);
    co[dir] = k - disp;
    MPI_Cart_rank(c, co, src);
    return MPI_SUCCESS;
}
/* A ring shift to oneself: the buffer is sent and received unchanged. */
static inline int MPI_Sendrecv_replace(void *b, int count, MPI_Datatype t, int dst, int stag, int src, int rtag,
                                       MPI_Comm c, MPI_Status *st)
{
    (void)b; (void)count; (void)t; (void)dst; (void)stag; (void)src; (void)rtag; (void)c; (void)st;
    tbmd_stub_one_rank("MPI_Sendrecv_replace");
    return MPI_SUCCESS;
}

static inline int MPI_Send(const void *b, int n, MPI_Datatype t, int d, int tag, MPI_Comm c)
{
    (void)b; (void)n; (void)t; (void)d; (void)tag; (void)c;
    return tbmd_stub_unreachable("MPI_Send");
}
static inline int MPI_Recv(void *b, int n, MPI_Datatype t, int s, int tag, MPI_Comm c, MPI_Status *st)
{
    (void)b; (void)n; (void)t; (void)s; (void)tag; (void)c; (void)st;
    return tbmd_stub_unreachable("MPI_Recv");
}
static inline int MPI_Isend(const void *b, int n, MPI_Datatype t, int d, int tag, MPI_Comm c, MPI_Request *r)
{
    (void)b; (void)n; (void)t; (void)d; (void)tag; (void)c; (void)r;
    return tbmd_stub_unreachable("MPI_Isend");
}
static inline int MPI_Irecv(void *b, int n, MPI_Datatype t, int s, int tag, MPI_Comm c, MPI_Request *r)
{
    (void)b; (void)n; (void)t; (void)s; (void)tag; (void)c; (void)r;
    return tbmd_stub_unreachable("MPI_Irecv");
}
static inline int MPI_Probe(int s, int tag, MPI_Comm c, MPI_Status *st)
{
    (void)s; (void)tag; (void)c; (void)st;
    return tbmd_stub_unreachable("MPI_Probe");
}
static inline int MPI_Get_count(const MPI_Status *st, MPI_Datatype t, int *n)
{
    (void)st; (void)t; (void)n;
    return tbmd_stub_unreachable("MPI_Get_count");
}
static inline int MPI_Wait(MPI_Request *r, MPI_Status *st)
{
    (void)r; (void)st;
    return tbmd_stub_unreachable("MPI_Wait");
}
static inline int MPI_Waitall(int n, MPI_Request *r, MPI_Status *st)
{
    (void)n; (void)r; (void)st;
    return tbmd_stub_unreachable("MPI_Waitall");
}

#endif
