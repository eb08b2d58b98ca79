/*
 * tbmd.h - C ABI of the B200 implementation of the Axilrod-Teller three-body hot path
 * (NATA / AUTA / P3BCA force evaluation and the Simulation step that integrates it).
 *
 * Plain C: pointers and sizes only, no exceptions, no C++ or torch types.  All host arrays are
 * owned by the caller and copied in or out during the call; the context owns all device memory
 * (particle state, cell grid, neighbour lists, CUDA graph).  One context per host thread; every
 * device operation of a context runs on that context's CUDA stream.
 *
 * Reference seams replaced (paths inside dmartin13/ThreeBodyMDAlgorithms):
 *   Simulation ctor / Init / Start     src/simulation/Simulation.cpp:3-19, 28-81
 *   Algorithm::SimulationStep          src/algorithm/Algorithm.hpp:60 (NATA.cpp:82-200,
 *                                      AUTA.cpp:236-384, P3BCA.cpp:516-805)
 *   Potential::CalculateForces         src/potential/Potential.hpp:25, AxilrodTeller.cpp:7-149
 *   DomainDecomposition::Get/SetMyParticles, Update, UpdatePredictorStage, ResetForces
 *                                      src/decomposition/DomainDecomposition.hpp:23-30
 *   Simulation::GetNumParticleInteractions / GetNumBufferInteractions   Simulation.cpp:89-96
 */
#ifndef TBMD_H
#define TBMD_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define TBMD_ABI_VERSION 1

typedef struct tbmd_ctx tbmd_ctx;

/* Status codes.  The reference prints a message and calls exit(1) on bad input
 * (cli.hpp:57-59, P3BCA.cpp:54-69, AUTA.cpp:129); here every entry point returns a status and
 * tbmd_last_error() holds the message. */
typedef enum {
    TBMD_OK = 0,
    TBMD_INVALID_ARG = 1,     /* null pointer, bad enum, n out of range, dt/nu not finite */
    TBMD_BAD_INPUT = 2,       /* NaN/inf coordinates or mass <= 0 */
    TBMD_NOT_READY = 3,       /* no particles set */
    TBMD_CAPACITY_RETRY = 4,  /* neighbour capacity still too small after the automatic retries */
    TBMD_CUDA_ERROR = 5,      /* a CUDA runtime call failed; see tbmd_last_error */
    TBMD_TIMEOUT = 6,         /* reserved; never returned (no kernel of this path waits on another) */
    TBMD_NO_DEVICE = 7,       /* no CUDA device, or not an sm_100 device */
    TBMD_TOO_LARGE = 8,       /* n above the limit of an allocation-free entry point */
    TBMD_RANK_LAYOUT = 9      /* the reference's run on that many MPI ranks would stop (tbmd_rank_layout_of) */
} tbmd_status;

/* Same numbering as the reference's AlgorithmType (src/utility/enums.hpp). */
typedef enum { TBMD_NATA = 0, TBMD_P3BCA = 1, TBMD_AUTA = 2 } tbmd_algorithm;

typedef enum {
    TBMD_FP64 = 0,  /* drop-in: all arithmetic in FP64 */
    TBMD_MIXED = 1  /* FP32 triplet geometry, FP64 displacements/accumulation/integration */
} tbmd_precision;

/* Simulation parameters: the reference's CLI values (cli.hpp:12-25) plus the GPU options. */
typedef struct {
    int32_t algorithm;  /* tbmd_algorithm */
    int32_t precision;  /* tbmd_precision */
    double cutoff;      /* P3BCA only; <= 0 means no cutoff, like the reference (Algorithm.cpp:94) */
    double dt;          /* -d */
    double g[3];        /* -gx -gy -gz */
    double nu;          /* AT strength; the reference uses AxilrodTeller(1.0) (main.cpp:41,66,91) */
    int32_t device;     /* CUDA device ordinal */
    int32_t use_graph;  /* 1: capture multi-step runs in a CUDA graph */
    void *stream;       /* cudaStream_t to run on, or NULL for a non-blocking stream owned by the
                           context (multi-step graphs need a stream that is not the legacy default) */
    int32_t reserved[8];
} tbmd_config;

/* Fill *cfg with the reference's defaults: AUTA, FP64, cutoff 0, dt 0, g 0, nu 1, device 0,
 * graphs on, own stream. */
void tbmd_config_init(tbmd_config *cfg);

/* Simulation constructor + Init (Simulation.cpp:3-19). */
tbmd_status tbmd_create(const tbmd_config *cfg, tbmd_ctx **out);
void tbmd_destroy(tbmd_ctx *ctx);
const char *tbmd_last_error(const tbmd_ctx *ctx);
const char *tbmd_status_string(tbmd_status s);
int32_t tbmd_abi_version(void);

/* Load the particle set (the reference's CSV input, utility.cpp:14-24, as SoA host arrays).
 * id may be NULL (0..n-1).  For P3BCA this also fixes the periodic domain from these positions:
 * L = |(max + 1e-4) - (min - 1e-4)| per axis (RegularGridDecomposition.cpp:24-28, 135-166).
 * Forces are reset to zero.  n must be >= 1. */
tbmd_status tbmd_set_particles(tbmd_ctx *ctx, int64_t n, const int32_t *id, const double *x, const double *y,
                               const double *z, const double *vx, const double *vy, const double *vz,
                               const double *ax, const double *ay, const double *az, const double *m);

/* Copy the current state out (DomainDecomposition::GetMyParticles, in input order).  Any pointer
 * may be NULL to skip that field.  fx/fy/fz are the stored forces (+grad E, like the reference). */
tbmd_status tbmd_get_particles(tbmd_ctx *ctx, int32_t *id, double *x, double *y, double *z, double *vx,
                               double *vy, double *vz, double *ax, double *ay, double *az, double *m,
                               double *fx, double *fy, double *fz);

int64_t tbmd_num_particles(const tbmd_ctx *ctx);

/* Particle generation on the device (the reference's particlegenerator, src/tools/particleToCSV.cpp,
 * UniformGenerator.cpp:12-28, ClusteredGaussGenerator.cpp:15-47), loaded as the context's particles
 * like tbmd_set_particles: ids 0..n-1, the given velocity, zero acceleration, the given mass.
 * Positions are the generator's exact sequence (std::mt19937 / std::minstd_rand0 with libstdc++'s
 * distributions); with csv_digits = 6 every value is rounded to 6 significant digits, which is what
 * the reference's main reads back from the generator's CSV. */
typedef enum { TBMD_GEN_UNIFORM = 0, TBMD_GEN_CLUSTERED_GAUSS = 1 } tbmd_generator_kind;
typedef struct {
    int32_t kind;        /* tbmd_generator_kind (--generator uniform | clusteredgauss) */
    int64_t n;           /* --numparticles; clustered: n / n_clusters particles per cluster */
    double box[3];       /* --blx --bly --blz */
    double corner[3];    /* bottomLeftCorner (not a generator flag; the tool's is 0, 0, 0) */
    double velocity[3];  /* --vx --vy --vz */
    double mass;         /* --mass */
    uint32_t seed0;      /* --seed0 */
    uint32_t seed1;      /* --seed1 (cluster centres) */
    int32_t n_clusters;  /* --numclusters */
    double mean;         /* --distmean */
    double stddev;       /* --diststddev */
    int32_t csv_digits;  /* 6: the CSV round trip; 0: exact doubles */
    int32_t reserved[7];
} tbmd_generator;
/* Defaults: uniform, n 0, box 10^3, corner 0, velocity 0, mass 1, seeds 926762934 / 89347587 (the
 * reference's documented seeds), 1 cluster, mean 0, stddev 1, csv_digits 6. */
void tbmd_generator_init(tbmd_generator *gen);
tbmd_status tbmd_generate_particles(tbmd_ctx *ctx, const tbmd_generator *gen);

/* Simulation::Start for `iterations` steps (Simulation.cpp:28-81): per step predictor
 * (structs.hpp:40-55), force reset + triplet forces (Algorithm::SimulationStep), update
 * (structs.hpp:57-99).  triplets_per_step (may be NULL) receives, per step, the value the
 * reference returns from GetNumParticleInteractions(step). */
tbmd_status tbmd_step(tbmd_ctx *ctx, int32_t iterations, uint64_t *triplets_per_step);

/* tbmd_set_particles, tbmd_step and tbmd_get_particles in one call, for callers whose particles live
 * in host arrays between steps, as the reference's Simulation keeps them in host vectors
 * (Simulation.cpp:28-81; its Start loop with a CSV written after every step, Simulation.cpp:74-79).
 * Inputs as tbmd_set_particles (checked; for P3BCA the domain is taken from them), `iterations`
 * steps with their triplet counts as tbmd_step, then the state as tbmd_get_particles: any output
 * may be NULL, and an output may be the very input array of the same field, but outputs must not
 * overlap one another.  The results are those of the three calls.  What differs is the overlap:
 * the last step's positions are final once its predictor has run and are copied back while its
 * forces are computed, masses (which no step changes) and IDs are copied on the host meanwhile,
 * and the whole call waits on the device once per attempt instead of once per call.  With
 * iterations > 0, ay and az are checked on the host but not copied to the device: a step reads ax
 * alone (the predictor applies it on all three axes) and the update overwrites all three. */
tbmd_status tbmd_step_host(tbmd_ctx *ctx, int64_t n, const int32_t *id, const double *x, const double *y,
                           const double *z, const double *vx, const double *vy, const double *vz, const double *ax,
                           const double *ay, const double *az, const double *m, int32_t iterations,
                           uint64_t *triplets_per_step, int32_t *id_out, double *x_out, double *y_out, double *z_out,
                           double *vx_out, double *vy_out, double *vz_out, double *ax_out, double *ay_out,
                           double *az_out, double *m_out, double *fx_out, double *fy_out, double *fz_out);

/* Algorithm::SimulationStep alone at the current positions, without integration (how the
 * reference's tests call it, tests.cpp:539).  Writes the stored forces into the context and,
 * if non-NULL, to fx/fy/fz, the total AT energy to *energy, the triplet count to *triplets. */
tbmd_status tbmd_forces(tbmd_ctx *ctx, double *fx, double *fy, double *fz, double *energy, uint64_t *triplets);

/* Adjoint of tbmd_forces (no reference counterpart).  Given cotangents gf on the stored forces and
 * g_energy on the energy, returns gx = H gf + g_energy * f (H = Hessian of the AT energy; the
 * triplet set is held fixed) and g_nu = (gf . f + g_energy * E) / nu.  Geometry is recomputed,
 * nothing per triplet is stored.  Any output may be NULL. */
tbmd_status tbmd_adjoint(tbmd_ctx *ctx, const double *gfx, const double *gfy, const double *gfz, double g_energy,
                         double *gx, double *gy, double *gz, double *g_nu);

/* Device-pointer variants for callers that already hold device memory (torch tensors).  They run
 * asynchronously on `stream` (cudaStream_t; NULL = the context stream, which is a non-blocking
 * stream: pass cudaStreamLegacy, i.e. (void *)1, to order with the legacy default stream, which
 * torch reports as handle 0) with positions of length n
 * given by the caller; the context's P3BCA domain is used (set it first with tbmd_set_domain or
 * tbmd_set_particles).  energy and triplets are device scalars (may be NULL). */
tbmd_status tbmd_forces_device(tbmd_ctx *ctx, int64_t n, const double *x, const double *y, const double *z,
                               double *fx, double *fy, double *fz, double *energy, uint64_t *triplets, void *stream);
tbmd_status tbmd_adjoint_device(tbmd_ctx *ctx, int64_t n, const double *x, const double *y, const double *z,
                                const double *gfx, const double *gfy, const double *gfz, const double *g_energy,
                                double *fx, double *fy, double *fz, double *energy, double *gx, double *gy,
                                double *gz, void *stream);

/* Fix the P3BCA periodic domain explicitly (L = box lengths, lo = lower corner). */
tbmd_status tbmd_set_domain(tbmd_ctx *ctx, const double *L, const double *lo);
/* Read the domain and the cell grid: dims = cells per axis (an axis shorter than 3 cutoffs is one
 * cell), cell_of_particle[n] (may be NULL) = linear cell index (cz*dy + cy)*dx + cx of each
 * particle at the current positions, in input order. */
tbmd_status tbmd_cells(tbmd_ctx *ctx, int32_t *cell_of_particle, int32_t *dims, double *L, double *lo);

/* Batched forces/energy (no reference counterpart): nsys independent systems packed back to back
 * (system s owns particles offsets[s] .. offsets[s+1]-1), each with its own P3BCA domain
 * (box[3*s .. 3*s+2] lengths, lo[3*s ..] lower corners; ignored without a cutoff), evaluated in
 * one persistent launch.  Host arrays.  energy and triplets are per system (may be NULL). */
tbmd_status tbmd_batch_forces(tbmd_ctx *ctx, int32_t nsys, const int64_t *offsets, const double *box,
                              const double *lo, const double *x, const double *y, const double *z, double *fx,
                              double *fy, double *fz, double *energy, uint64_t *triplets);
/* Batched adjoint: per-system g_energy[s]; returns gx (H gf + g_energy f) and g_nu per system. */
tbmd_status tbmd_batch_adjoint(tbmd_ctx *ctx, int32_t nsys, const int64_t *offsets, const double *box,
                               const double *lo, const double *x, const double *y, const double *z,
                               const double *gfx, const double *gfy, const double *gfz, const double *g_energy,
                               double *gx, double *gy, double *gz, double *g_nu);

/* Autotuner: times the kernel variants of this context's algorithm/precision at its current n and
 * keeps the fastest.  Results are cached as JSON in cache_path (NULL: no file) keyed by GPU name,
 * algorithm, precision and n bucket; a cached entry is reused without timing. */
tbmd_status tbmd_autotune(tbmd_ctx *ctx, const char *cache_path);
/* The variant in use, as a short JSON object (valid until the next call on ctx). */
const char *tbmd_tuning(const tbmd_ctx *ctx);

/* Per-phase device timing, the counterpart of the reference's PROFILE_3BMDA phase timers
 * (Algorithm.hpp:33-38, main.cpp:127-451).  While on, steps run eagerly (no CUDA graph) with CUDA
 * events between phases on the context stream; times accumulate until tbmd_set_profiling is
 * called again.  Phases, in this order: 0 predictor, 1 cell build (counting sort), 2 neighbour
 * lists, 3 triplet forces (the P3BCA kernel or the NATA/AUTA sweep), 4 update (incl. unsort and
 * count bookkeeping).  In a P3BCA step the predictor is fused into the cell build and reported
 * there (phase 0 stays empty).  tbmd_phase_times fills up to max entries of ms (milliseconds), calls (phase
 * executions) and launches (kernels launched in the phase) and returns the number of phases. */
tbmd_status tbmd_set_profiling(tbmd_ctx *ctx, int32_t on);
int32_t tbmd_phase_times(const tbmd_ctx *ctx, double *ms, uint64_t *calls, uint64_t *launches, int32_t max);

/* Allocation-free NATA forces.  No counterpart in the reference: this entry point exists for
 * callers that cannot allocate device memory when they need forces (a fixed pre-reserved memory
 * budget, a callback inside another library that owns the allocator, a latency-critical loop that
 * must not synchronise in cudaMalloc).  It needs no context: positions x, y, z and forces fx, fy, fz
 * are caller device buffers of n doubles, and the only scratch is a fixed static device array of
 * about 3 MiB inside the library (held on every GPU that loads it until exit).  It computes the
 * stored forces (+grad E, no cutoff, strength nu) of all C(n,3) triplets with the NATA kernel in
 * FP64 or mixed precision on `stream` (cudaStream_t, NULL = legacy default stream), asynchronously.
 * 1 <= n <= TBMD_NOALLOC_MAX_N; larger n returns TBMD_TOO_LARGE without launching anything; a
 * non-finite nu returns TBMD_INVALID_ARG.  The first call on a device looks up the scratch address
 * in the context current at that time and caches it with that context's unique id; a call made
 * while another context is current (after cudaDeviceReset, or a context the caller created) looks
 * it up again.  Make the first call, and the first one after such a change, before any stream
 * capture.  All calls share the scratch, so calls that overlap on the GPU race and must be
 * serialised. */
#define TBMD_NOALLOC_MAX_N 4096
tbmd_status tbmd_nata_forces_noalloc(int64_t n, const double *x, const double *y, const double *z, double nu,
                                     int32_t precision, double *fx, double *fy, double *fz, void *stream);

/* Debug-build index checks.  No counterpart in the reference (its debug aid would be a
 * compute-sanitizer run).  A library built with -DTBMD_BOUNDS_CHECK (python -m
 * threebodymdalgorithms_b200.build --bounds-check, libtbmd_checked.so) checks the computed indices of
 * its kernels (cells, sorted slots, neighbour lists, staged slots, pair places, sweep items): an
 * index outside its array is recorded on the device and replaced by 0, so the kernel neither faults
 * nor traps.  This call waits for the device, writes the number of violations since the last call
 * (-1 if the device could not be read) and the site, index and array size of the first one, clears
 * the record and returns 1 for a checked build; a normal build records nothing and returns 0. */
int32_t tbmd_bounds_report(int64_t *violations, int32_t *site, int64_t *index, int64_t *size);

/* Layout of the reference's run on P MPI ranks (host only, no device work).  Results do not depend
 * on P: every rank layout evaluates each triplet once, and the GPU evaluates them all in one
 * process.  What P decides in the reference is the process grid and whether the run starts, and
 * this entry point restates that so that a caller (and tbmd_main -np P) stops where an
 * `mpiexec -n P` run would, with the same message.
 *
 *   P3BCA: the process grid of main.cpp:546-551 (utility.cpp:96-107 over the tables of
 *     utility/decompositions.hpp): naive = {P}; optimal = the factorisation of P into one to three
 *     non-decreasing factors, each at least 3 unless it is P itself, with the smallest sum, the
 *     lexicographically first among equal sums except P = 360 (6 x 6 x 10).  Tables end at
 *     P = 1024; above it the grid is empty and the reference's CartTopology::Init reads past it
 *     (CartTopology.cpp:10-12): TBMD_RANK_LAYOUT, with a message saying so.
 *     Local cell width L / dims (RegularGridDecomposition.cpp:24-32), cutoff boxes per axis and
 *     the cutoff-window check (P3BCA.cpp:29-70), shift steps per Simulation step (P3BCA.cpp:79-92).
 *   NATA / AUTA: ring of P ranks; AtomDecomposition (AtomDecomposition.cpp:15-41) pads the first
 *     P - n mod P ranks with one dummy particle each when n mod P != 0.
 *
 * L is the physical domain size (tbmd_cells returns it; P3BCA only, may be NULL otherwise).
 * Returns TBMD_OK; TBMD_INVALID_ARG (bad algorithm, world_size < 1, n < 0, cutoff not finite,
 * L not positive); TBMD_RANK_LAYOUT where the reference's run stops, with its stderr line in msg.
 * msg may be NULL; otherwise up to msg_len bytes including the terminating 0 are written. */
typedef struct tbmd_rank_layout {
    int32_t world_size;
    int32_t num_dims;            /* process-grid dimensions (1 for the NATA / AUTA ring) */
    int32_t dims[3];             /* ranks per axis, 1 for unused axes */
    int32_t cutoff_boxes[3];     /* P3BCA nCbX, nCbY, nCbZ */
    int32_t shift_steps;         /* P3BCA CalculateInteractions rounds per Simulation step */
    int32_t reserved;
    double cell_size[3];         /* P3BCA local cell width per axis */
    int64_t particles_per_rank;  /* NATA / AUTA particles per rank, dummies included */
    int64_t dummies;             /* NATA / AUTA dummy particles over all ranks */
} tbmd_rank_layout;
tbmd_status tbmd_rank_layout_of(int32_t algorithm, int32_t world_size, int32_t optimal_decomposition, double cutoff,
                                const double *L, int64_t n, tbmd_rank_layout *out, char *msg, int32_t msg_len);

/* Wait for all work of the context's stream. */
tbmd_status tbmd_sync(tbmd_ctx *ctx);

/* Number of kernels this context has launched since creation (all of them are this library's). */
uint64_t tbmd_kernel_launches(const tbmd_ctx *ctx);

#ifdef __cplusplus
}
#endif

#endif /* TBMD_H */
