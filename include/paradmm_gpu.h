/*
 * paradmm_gpu.h -- C-ABI of the B200 parADMM engine (libparadmm_b200.so).
 *
 * Replaces the reference GPU back-end (core/paradmm-gpu.h:16-29 and the
 * user-launched kernel loop of packing/gpu.cu:257-291): instead of deep
 * copying the graph with one cudaMalloc per factor and launching five kernels
 * per sweep, a caller creates an engine handle from a host `graph`
 * (paradmm.h), iterates or solves on the device, and downloads the state back
 * into the graph in the reference's FP64 [edge][dim] layout.
 *
 * Every function returns PARADMM_OK (0) or a negative PARADMM_E* code and
 * never exits the process; paradmm_last_error_string() describes the last
 * failure of the calling thread.  A handle owns its device memory and its
 * CUDA stream; calls on one handle are synchronous and must not overlap.
 *
 * Engines.  A graph whose factors are the three circle-packing operators
 * (pair non-overlap, half-plane wall, radius reward) over consistent
 * (centre, radius) variable couples, with every pair of circles present once
 * and per-position uniform pair penalties, runs on the fused packing engine:
 * FP32 edge state in a tiled structure-of-arrays layout, FP64 consensus and
 * residuals, one persistent grid-synchronised kernel for many sweeps.  Any
 * other graph of those operators runs on the generic engine (CSR incidence,
 * FP64 or FP32 state, reference summation order).  Graphs with operators the
 * engine does not know are rejected with PARADMM_EUNSUPPORTED_OP.
 */
#ifndef PARADMM_B200_PARADMM_GPU_H
#define PARADMM_B200_PARADMM_GPU_H

#include <stdint.h>
#include "paradmm.h"

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---- */
enum {
    PARADMM_OK = 0,
    PARADMM_EINVAL = -1,             /* bad argument or inconsistent graph        */
    PARADMM_ENOMEM = -2,             /* host or device allocation failed          */
    PARADMM_ECUDA = -3,              /* CUDA runtime error                        */
    PARADMM_EUNSUPPORTED_OP = -4,    /* a factor's operator is not known          */
    PARADMM_EUNSUPPORTED_GRAPH = -5, /* the requested engine cannot run this graph */
    PARADMM_ENONFINITE = -6,         /* NaN/Inf appeared in the residuals         */
    PARADMM_ETIMEOUT = -7,           /* a device-side wait ran out (grid barrier) */
    PARADMM_ENODEVICE = -8           /* no usable CUDA device                     */
};

/* ---- operator kinds (the three packing operators, packing/host.c:31-132) ---- */
enum {
    PARADMM_OP_UNKNOWN = 0,
    PARADMM_OP_PAIR = 1,   /* disk_collision_variable_radius, 4 edges          */
    PARADMM_OP_WALL = 2,   /* disk_plane_collision_variable_radius, 2 edges,
                              params = [v (numdims), p (numdims)] doubles     */
    PARADMM_OP_RADIUS = 3, /* maximize_sum_of_squared_disk_radii_alpha, any
                              number of edges, params[0] = exponent           */
    PARADMM_OP_USER = 4    /* a caller's operator with a device twin given as
                              source (paradmm_gpu_register_op_source)         */
};

/* ---- engine selection ---- */
enum {
    PARADMM_ENGINE_AUTO = 0,        /* packing engine when eligible, else generic FP64 */
    PARADMM_ENGINE_PACKING = 1,     /* fused packing engine (FP32 state, FP64 consensus) */
    PARADMM_ENGINE_GENERIC_F64 = 2, /* CSR engine, FP64, reference summation order       */
    PARADMM_ENGINE_GENERIC_F32 = 3  /* CSR engine, FP32 state, FP64 consensus            */
};

typedef struct paradmm_gpu paradmm_gpu; /* opaque engine handle */

typedef struct paradmm_gpu_opts {
    int device;       /* CUDA device ordinal                                   */
    int engine;       /* PARADMM_ENGINE_*                                      */
    int block_width;  /* packing engine: circles per tile side (32, 64, 128); 0 = tuned */
    int ctas_per_sm;  /* packing engine: resident CTAs per SM; 0 = tuned       */
    int check_every;  /* sweeps between residual-based stopping checks; 0 = 1  */
    int schedule;     /* packing engine: PARADMM_SCHEDULE_*                      */
    int cluster_size; /* per-instance schedule: CTAs per large instance (1, 2, 4, 8); 0 = default (2) */
    int reserved[6];  /* reserved[0]: per-instance schedule, smallest N solved by a whole cluster (0 = 200);
                         reserved[1]: 1 = launch per-instance solves directly, not as a replayed CUDA graph;
                         reserved[2]: tail hand-off of the per-instance schedule (paradmm_gpu_set_tail_handoff) */
} paradmm_gpu_opts;

/* How the packing engine spreads a handle's instances over the GPU. */
enum {
    PARADMM_SCHEDULE_AUTO = 0,     /* per-instance CTAs for batches of small instances, else grid-wide */
    PARADMM_SCHEDULE_GRID = 1,     /* every CTA works on every instance; grid barrier per sweep        */
    PARADMM_SCHEDULE_INSTANCE = 2, /* one CTA per instance at a time, no grid barrier (N <= 1024)      */
    PARADMM_SCHEDULE_ONCHIP = 3    /* per instance, its whole state held in the shared memory of a
                                      group of 1-16 CTAs of a thread-block cluster for the solve
                                      (instances up to ~450 circles, <= 4 walls per circle)          */
};

typedef struct paradmm_stats {
    int64_t iterations;   /* sweeps performed by the call                       */
    int converged;        /* 1 when primal + dual <= tol was met                */
    int status;           /* PARADMM_OK or the error that stopped the call      */
    double primal;        /* RMS over all (edge, dim) of X - Z_v(e)             */
    double dual;          /* RMS over all (edge, dim) of Z_v(e) - Zprev_v(e)    */
    double max_violation; /* packing: max pair overlap / wall penetration / -r  */
    double total_radius;  /* packing: sum of consensus radii                    */
    double device_ms;     /* device time of the call                            */
} paradmm_stats;

/* Default options (device 0, AUTO engine, tuned shapes). */
void paradmm_gpu_default_opts(paradmm_gpu_opts *opts);

/* Declares that host function `op` is one of the packing operators, so that
 * graphs built with the caller's own copy of that operator are accepted.
 * The library's exported operators (paradmm.h) are known without this. */
int paradmm_gpu_register_op(paradmm_op_fn op, int kind);

/* Any other operator: the caller gives the device twin of host operator
 * `op` as CUDA C++ source defining
 *     __device__ void <function_name>(double *x, double *n, double *rhos,
 *                                     int numvars, int numdims, void *params)
 * with the reference operator contract (core/paradmm.h:41: read n and rhos,
 * write x; it may write rhos).  This replaces the reference GPU back-end's
 * user-supplied __device__ operators called through device function pointers
 * (core/paradmm-gpu.cu:23-47, packing/gpu.cu:177-184).  The source is
 * compiled at run time (NVRTC, for this device, FP64 without FMA
 * contraction, as the generic engine itself is built) the first time a
 * graph uses it; graphs with such factors run on the generic FP64 engine,
 * every phase on the GPU.  A factor's params are copied to the device by the
 * byte size given to addNodeWithParamSize (a factor with params but no size
 * is rejected with PARADMM_EINVAL), each copy 16-byte aligned.  Errors: the
 * compiler's log is in paradmm_last_error_string() (PARADMM_EINVAL);
 * PARADMM_EUNSUPPORTED_OP when the run-time compiler cannot be loaded.
 * Registering the same `op` again replaces its source. */
int paradmm_gpu_register_op_source(paradmm_op_fn op, const char *device_source, const char *function_name);

/* Builds a handle for graph G: classifies its factors, lays out the state on
 * the device and uploads the state arrays (X, N, U, Z, RHOS, ALPHAS) that G
 * holds.  G is only read; the handle does not keep pointers into it. */
int paradmm_gpu_create(const graph *G, const paradmm_gpu_opts *opts, paradmm_gpu **out);

/* Re-uploads the state arrays of G (same topology as at create). */
int paradmm_gpu_upload(paradmm_gpu *h, const graph *G);

/* Runs n full sweeps (updateG semantics). */
int paradmm_gpu_iterate(paradmm_gpu *h, int n);

/* Runs up to maxiter sweeps, stopping once primal + dual <= tol (tol < 0:
 * never).  Packing engine: the residuals of iterate k are reduced on the
 * device while sweeps k+1 and k+2 run, so the state returned is two sweeps
 * past the first iterate whose residuals met the tolerance (the stats give
 * that iterate's residuals); the generic engine stops at that iterate.
 * stats may be NULL. */
int paradmm_gpu_solve(paradmm_gpu *h, int maxiter, double tol, paradmm_stats *stats);

/* Writes X, M, N, U and Z of the current iterate into G (reference layout,
 * FP64).  G must have the create-time topology and allocated state arrays. */
int paradmm_gpu_download(paradmm_gpu *h, graph *G);

/* Residuals and packing metrics of the current iterate. */
int paradmm_gpu_stats(paradmm_gpu *h, paradmm_stats *out);

/* Which engine the handle runs (PARADMM_ENGINE_*). */
int paradmm_gpu_engine(const paradmm_gpu *h);

void paradmm_gpu_destroy(paradmm_gpu *h);

/* ---- structured packing problems (no host graph needed) ----
 *
 * Describes the graph the reference demo builds (packing/host.c:283-343):
 * n_circles circles, one radius factor per circle, each listed half-plane
 * applied to every circle, and every pair of circles, with penalties rho
 * (rho_radius on the radius factors' edges) and step alpha.  Initial state:
 * Z from `init` ([cx, cy, r] per circle), X_e = Z_v(e), U = 0.  Its edge
 * numbering is that of the graph built in packing/host.c's order: radius
 * factors, then walls (wall-major), then pairs (row-major i < j). */
typedef struct paradmm_packing_desc {
    int n_circles;
    int n_walls;          /* <= 8 */
    const double *walls;  /* n_walls x [v_x, v_y, p_x, p_y]: v.(c - p) + r <= 0 */
    double exponent;      /* radius reward exponent (params[0] of the radius op) */
    double rho;           /* penalty of pair and wall edges                     */
    double rho_radius;    /* penalty of radius-factor edges                     */
    double alpha;         /* dual step on every edge                            */
    const double *init;   /* n_circles x [cx, cy, r]                            */
} paradmm_packing_desc;

/* One handle holding `count` independent packing instances (count = 1 for a
 * single problem).  Instances may differ in every field.  They share one
 * persistent launch; each stops on its own residual in solve. */
int paradmm_gpu_create_packing(const paradmm_packing_desc *descs, int count,
                               const paradmm_gpu_opts *opts, paradmm_gpu **out);

/* Number of instances of a handle (1 for graph handles). */
int paradmm_gpu_instances(const paradmm_gpu *h);

/* Per-instance statistics of the last solve / current state
 * (stats must hold paradmm_gpu_instances(h) entries). */
int paradmm_gpu_instance_stats(paradmm_gpu *h, paradmm_stats *stats);

/* Consensus circles [cx, cy, r] of one instance (n_circles x 3 doubles). */
int paradmm_gpu_get_circles(paradmm_gpu *h, int instance, double *out);

/* Replaces an instance's state by a warm start: consensus Z from `circles`
 * ([cx, cy, r] per circle), X_e = Z_v(e), and the duals U of the pair edges
 * from `pair_duals` (may be NULL for U = 0).  pair_duals holds, for every
 * pair i < j in row-major order, the six pair-edge duals
 * [u_cx_i, u_cy_i, u_r_i, u_cx_j, u_cy_j, u_r_j]. */
int paradmm_gpu_warm_start(paradmm_gpu *h, int instance, const double *circles, const float *pair_duals);

/* The reference's warm-start contract, initialize_X_N_Z_M_U_optimal(G,
 * Zinit, Uinit, maxiter) (core/paradmm.c:266-375), for one instance, on the
 * device: Z from `circles`, X_e = Z_v(e) on every edge, the duals U from
 * Uinit, then `dual_iters` rounds of the reference's per-factor map
 *     X~ = prox_f(Z - U),  U <- X~ - (Z - U)
 * (its loop at core/paradmm.c:349-357), each factor on its own with its own
 * penalties, so that a dual reaching the map's fixed point makes Z a fixed
 * point of that factor's prox.  N = Z - U and M = X + U follow.  Uinit:
 *   pair_duals    6 per pair i < j, row-major: [u_cx_i, u_cy_i, u_r_i,
 *                 u_cx_j, u_cy_j, u_r_j];
 *   wall_duals    3 per wall factor [u_cx, u_cy, u_r], circle by circle,
 *                 each circle's walls in the order they were given;
 *   radius_duals  1 per circle;
 * any of them NULL = 0.  dual_iters = 0 takes Uinit as it is (unlike the
 * reference, whose U is left unset then, core/paradmm.c:278).  The state is
 * kept in FP32.  Resets the instance's penalty scale to 1. */
int paradmm_gpu_warm_start_duals(paradmm_gpu *h, int instance, const double *circles, const double *pair_duals,
                                 const double *wall_duals, const double *radius_duals, int dual_iters);

/* Residual balancing of the penalties (adaptive rho).  The reference has a
 * hook for it and nothing in it: update_outgoing_rhos (core/paradmm.c:564-566,
 * called at the end of updateZ, :671 and :893) is empty; the drop-in
 * update_outgoing_rhos of this library stays empty too, and the paradmm.h
 * sweep functions never balance.  On a handle, after this call, every
 * `period` iterates (counted from the state the handle was created, uploaded
 * or warm-started with; ages a = period, 2 period, ...) the residuals r, s of
 * that iterate decide: r > mu s doubles every penalty of the instance (as long
 * as its scale stays <= 2^log2_max), s > mu r halves them (scale >=
 * 2^log2_min), else nothing.  A decision on the iterate of age a applies
 * right after the sweep of age a + 2: RHOS times t (t = 2 or 1/2) and the
 * scaled duals U divided by t (N = Z - U follows), so rho U is unchanged.
 * Power-of-two scaling is exact, and the pair and wall operators and the
 * consensus weights are homogeneous in the penalties, so only the radius
 * operator and the duals feel it: the FP64 generic engine reproduces the
 * same rule applied to the reference's own updateG bit for bit.  period = 0
 * switches it off (the default); otherwise period >= 3 and mu >= 1.  A new
 * state (upload, warm start, fallback restart) returns the scale to 1.
 * Downloads give U in the current scale; RHOS of the host graph is not
 * written (the current penalties are RHOS x 2^scale, paradmm_gpu_rho_scale).
 * In the grid schedule, an instance resumed by a later call after it had
 * stopped skips the decisions that fall on its first two sweeps of that
 * call.  With exponent-2 radius rewards keep rho_radius 2^log2_min > 2: the
 * radius operator is convex only there (packing/host.c:10-29). */
int paradmm_gpu_set_rho_balance(paradmm_gpu *h, int period, double mu, int log2_min, int log2_max);

/* log2 of the penalty scale instance `instance` will use in its next sweep. */
int paradmm_gpu_rho_scale(const paradmm_gpu *h, int instance, int *log2_scale);

/* In-call fallback for warm starts (per-instance schedule only; no reference
 * counterpart).  With after_sweeps > 0, every later paradmm_gpu_solve call
 * restarts an instance that has not converged after after_sweeps sweeps of
 * that call (or whose residual became NaN/Inf before then) from its plain
 * start -- the circles given at creation, X = Z on every edge, every dual 0 --
 * and continues it for the rest of the call's maxiter, inside the same
 * launch.  0 (the default) switches it off.  EINVAL on a grid-schedule handle. */
int paradmm_gpu_set_fallback(paradmm_gpu *h, int64_t after_sweeps);

/* restarted[i] = 1 if instance i fell back to its plain start in the last
 * solve call, else 0. */
int paradmm_gpu_instance_fallbacks(const paradmm_gpu *h, int *restarted);

/* Schedule autotuner (no reference counterpart).  Times each candidate
 * configuration of the handle -- the grid-wide schedule, and for batches of
 * instances with N <= 1024 the per-instance schedule with clusters of 1, 2
 * or 4 CTAs for instances of at least 120, 200 or 300 circles -- on a probe
 * solve from the handle's current state, restores that state after each
 * probe, and keeps the fastest.  The probe is paradmm_gpu_solve(h, sweeps,
 * tol): with tol < 0 every instance runs `sweeps` sweeps (a throughput
 * probe); with tol >= 0 instances stop on their residual as in a real solve,
 * which also weighs how long each instance runs.  The state, iteration
 * counters and fallback setting are as before the call.  Device memory for
 * one copy of the state is allocated for the duration. */
typedef struct paradmm_gpu_tuning {
    int schedule;      /* PARADMM_SCHEDULE_GRID or PARADMM_SCHEDULE_INSTANCE  */
    int cluster_size;  /* per-instance schedule: CTAs per large instance      */
    int coop_min_n;    /* per-instance schedule: smallest N given a cluster   */
    int candidates;    /* configurations timed                                */
    double ms;         /* device time of the chosen configuration's probe     */
    double worst_ms;   /* slowest candidate's probe                           */
    int block_width;   /* paradmm_gpu_create_packing_tuned: chosen tile side  */
    int reserved[3];
} paradmm_gpu_tuning;
int paradmm_gpu_autotune(paradmm_gpu *h, int sweeps, double tol, paradmm_gpu_tuning *out);

/* paradmm_gpu_create_packing plus the tile shape: builds the instances with
 * tile sides (block widths) 64 and 128 (or only opts->block_width when it is
 * set), autotunes each handle's schedule with the same probe as
 * paradmm_gpu_autotune(h, sweeps, tol), and returns the fastest handle in
 * its initial state (the others are destroyed).  No reference counterpart. */
int paradmm_gpu_create_packing_tuned(const paradmm_packing_desc *descs, int count, const paradmm_gpu_opts *opts,
                                     int sweeps, double tol, paradmm_gpu **out, paradmm_gpu_tuning *tuning);

/* Failure-detection self-test (no reference counterpart): launches a
 * two-block grid barrier that one block never reaches, with a wait limit of
 * timeout_ms.  The waiting block gives up after the limit, records the
 * device-side error and returns, as the packing kernels do when a block
 * stops making progress; the call then returns PARADMM_ETIMEOUT, the status
 * paradmm_gpu_solve reports in that case.  The device stays usable. */
int paradmm_gpu_selftest_barrier_timeout(int device, int timeout_ms);

/* Device memory the handle holds, in bytes. */
int64_t paradmm_gpu_device_bytes(const paradmm_gpu *h);

/* Per-instance schedule: device-clock start and stop of every instance in
 * the last solve/iterate call, in ms from the earliest start. */
int paradmm_gpu_instance_times(const paradmm_gpu *h, double *begin_ms, double *end_ms);

/* Kernels the handle has launched so far. */
int64_t paradmm_gpu_launches(const paradmm_gpu *h);

/* Packing engine: when on, later sweeps record how long the average block
 * spends per sweep in the pass, the first grid barrier, the consensus
 * finalisation and the second barrier (per-instance schedule: the pass, the
 * block/cluster barrier after it, the consensus, and the barrier plus stop
 * test); paradmm_gpu_phase_times returns those four means (microseconds)
 * for the last solve/iterate call. */
/* Tail hand-off of the per-instance schedule: once every instance of a
 * solve call has started and at most `instances` are unfinished, those stop
 * at a sweep boundary and finish together on the grid-wide schedule (one
 * pass over all their tiles by every CTA per sweep, instead of one pass per
 * instance by its own few CTAs); each keeps its own budget of maxiter sweeps
 * and its own stop test.  0 (default): off.  Not combined with a fallback
 * budget (paradmm_gpu_set_fallback) that can restart an instance within the
 * call.  The per-instance device timestamps (paradmm_gpu_instance_times)
 * of a handed-over instance end at the hand-off.  paradmm_gpu_tail_handoffs:
 * instances the last solve call handed over. */
int paradmm_gpu_set_tail_handoff(paradmm_gpu *h, int instances);
int paradmm_gpu_tail_handoffs(const paradmm_gpu *h);

int paradmm_gpu_set_profiling(paradmm_gpu *h, int on);
int paradmm_gpu_phase_times(const paradmm_gpu *h, double out[4]);

/* Page-locks G's X, M, N, U and Z arrays so uploads and downloads run at
 * full PCIe/C2C rate.  The paradmm.h sweep functions do this by themselves
 * for graphs whose edge state is >= 64 MiB; closeG (or unpin) releases it. */
int paradmm_gpu_pin_graph(const graph *G);
int paradmm_gpu_unpin_graph(const graph *G);

/* Appends the factors of the reference demo's packing graph to G (which
 * must be fresh from startG(G, 2)): one radius factor per circle on var 2i+1,
 * each of the n_walls half-planes on every circle (vars 2i, 2i+1), and every
 * pair i < j (vars 2i, 2i+1, 2j, 2j+1), by addNode, in packing/host.c's order
 * (order = 0: radius, walls, pairs) or packing/gpu.cu's (order = 1: walls,
 * radius, pairs).  walls (n_walls x 4 doubles) and exponent (1 double) are
 * borrowed by the graph like any addNode parameter and must outlive it.
 * A fast bulk replacement for the reference demo's construction loops
 * (packing/host.c:299-335). */
int paradmm_add_packing_factors(graph *G, int n_circles, int n_walls, double *walls, double *exponent, int order);

/* ---- one packing instance sharded over ranks ----
 *
 * No reference counterpart: the reference runs one graph on one device
 * (core/paradmm-gpu.cu).  An instance is split by circle-block rows: rank r
 * of nranks stores and sweeps the pair tiles (I, J >= I) of rows
 * [bounds[r], bounds[r+1]) and the wall and radius factors of those rows'
 * circles, with bounds from paradmm_gpu_shard_rows (rows balanced by pair
 * count; block width opts->block_width, 64 by default).  Every rank keeps
 * the whole consensus Z.  One sweep is
 *     paradmm_gpu_shard_begin(h, exchange, stream)   pass + this rank's partial sums
 *     <sum `exchange` over all ranks, in place>      e.g. an NCCL all-reduce (float64 sum)
 *     paradmm_gpu_shard_end(h, exchange, stream)     consensus + residuals + stop test
 * where `exchange` is a device buffer of exchange_bytes (32 bytes per
 * circle, 16-byte aligned) owned by the caller.  Every rank derives Z from
 * the same summed buffer, so all ranks hold identical Z and take the same
 * stop decision; with one rank the sweep equals the unsharded engine's bit
 * for bit.  `stream` is a cudaStream_t (NULL: the default stream); all
 * three steps must be ordered on it.  A run is armed by shard_start
 * (maxiter sweeps at most, stop when primal + dual <= tol, tol < 0: never);
 * shard_poll synchronises the stream and says whether the instance still
 * runs (all ranks see the same answer after the same sweep); shard_finish
 * ends the run and fills stats (iterations, converged, residuals).  The
 * handle answers paradmm_gpu_get_circles / instance_stats / warm_start like
 * a one-instance packing handle; paradmm_gpu_solve/iterate and the
 * autotuner refuse it. */
int paradmm_gpu_shard_rows(int n_circles, int block_width, int nranks, int *bounds /* nranks + 1 */);
int paradmm_gpu_create_packing_shard(const paradmm_packing_desc *desc, int rank, int nranks,
                                     const paradmm_gpu_opts *opts, paradmm_gpu **out);
int paradmm_gpu_shard_info(const paradmm_gpu *h, int *row_lo, int *row_hi, int64_t *exchange_bytes);
int paradmm_gpu_shard_start(paradmm_gpu *h, int maxiter, double tol, int check_every);
int paradmm_gpu_shard_begin(paradmm_gpu *h, void *exchange, void *stream);
int paradmm_gpu_shard_end(paradmm_gpu *h, const void *exchange, void *stream);
int paradmm_gpu_shard_poll(paradmm_gpu *h, void *stream, int *active);
int paradmm_gpu_shard_finish(paradmm_gpu *h, void *stream, paradmm_stats *stats);

/* The whole armed run in ONE persistent launch per device, with the exchange
 * fused into it: each rank writes its partial sums straight into slot r of
 * every rank's exchange buffer (peer stores over NVLink), raises its flag in
 * every rank's flag array, waits (bounded) for all ranks' flags of the sweep
 * and sums the slots in rank order, so every rank holds the same Z and takes
 * the same stop decision; no host round trip, no collective library call.
 *
 * paradmm_gpu_shard_fused_buffers allocates (once) and returns this rank's
 * exchange buffer (2 x nranks x n_circles x 32 bytes) and flag array
 * (nranks x 8 bytes) on its device; a multi-process caller shares them
 * between processes (CUDA IPC) and maps the peers' into each process.
 *
 * paradmm_gpu_shard_run_fused(hs, nlocal, exchanges, flags, wait_ms, stream)
 * runs ranks hs[0 .. nlocal) -- consecutive ranks of one split, on one
 * device, each armed by paradmm_gpu_shard_start and not yet stepped -- in
 * one cooperative launch; exchanges[q] and flags[q] are rank q's buffers as
 * this device addresses them, for every q < nranks.  One process per GPU
 * passes nlocal = 1; every rank must launch (all ranks' kernels run at the
 * same time, one per GPU), or, on one device, all ranks go in one call.  A
 * flag that does not arrive within wait_ms (0: 4 s) ends the launch with
 * PARADMM_ETIMEOUT.  It returns when the run has ended (stop test or
 * maxiter); paradmm_gpu_shard_finish then reads the statistics.  At most 8
 * ranks. */
int paradmm_gpu_shard_fused_buffers(paradmm_gpu *h, void **exchange, void **flags);
int paradmm_gpu_shard_run_fused(paradmm_gpu *const *hs, int nlocal, void *const *exchanges, void *const *flags,
                                int wait_ms, void *stream);

/* Process-to-process sharing of those buffers (CUDA IPC; the handle is 64
 * bytes): export a device allocation's base pointer, import it on `device`
 * (peer access enabled on first use), close an imported pointer. */
int paradmm_gpu_ipc_export(const void *dev_ptr, void *handle /* 64 bytes */);
int paradmm_gpu_ipc_import(int device, const void *handle, void **dev_ptr);
int paradmm_gpu_ipc_close(int device, void *dev_ptr);

/* ---- allocation-free packing sweeps ----
 *
 * Some callers cannot allocate device memory while they run: services that
 * reserve their whole device-memory budget up front and forbid any later
 * cudaMalloc, and latency-critical loops (a planner re-solving a packing
 * every control tick, for instance), where cudaMalloc/cudaFree can
 * synchronise the device and stall every other stream.  This entry point
 * serves them: it allocates nothing.  (It has no counterpart in the
 * reference, which allocates per factor.)
 *
 * It runs `sweeps` fused sweeps (stopping early once primal + dual <= tol,
 * tol < 0: never) of ONE packing instance described by `desc` (desc->init
 * is ignored).  The caller passes, in device memory it owns:
 *   d_circles  n_circles x [cx, cy, r] doubles: the consensus, read at the
 *              start and written back at the end;
 *   d_state    paradmm_noalloc_state_bytes(n_circles, n_walls) bytes,
 *              16-byte aligned: the FP32 edge state in the engine's layout
 *              (opaque to the caller).  With init_state = 1 it is first set to the plain
 *              start X_e = Z_v(e), U = 0; with init_state = 0 it must hold
 *              the state a previous successful (or NaN/Inf-stopped) call
 *              left, so consecutive calls continue one solve.  A buffer this
 *              entry point never initialised (zero-filled, say) is refused
 *              with PARADMM_EINVAL, and so is one whose last call ended in
 *              any other error: the state then has to start again with
 *              init_state = 1.
 * All scratch (tables, consensus partial sums, residual slots, barrier
 * control) lives in one fixed array of PARADMM_NOALLOC_SCRATCH_BYTES inside
 * this library, present on every GPU that loads it until the process exits.
 * Limits: n_circles <= PARADMM_NOALLOC_MAX_CIRCLES, n_walls <=
 * PARADMM_NOALLOC_MAX_WALLS; larger problems are rejected with PARADMM_EINVAL.
 * The first call on a device looks up that array's device address (a
 * one-time set-up); make that first call before any stream capture.  Every
 * call reuses the same array and overwrites what the previous call left, so
 * calls whose work overlaps on the GPU (other threads or streams) race: run
 * them one after another.  `stream` is a cudaStream_t (NULL: the default
 * stream); the call returns after the work on it has finished.  stats may be
 * NULL; its device_ms is host-measured. */
#define PARADMM_NOALLOC_MAX_CIRCLES 512
#define PARADMM_NOALLOC_MAX_WALLS 8
#define PARADMM_NOALLOC_SCRATCH_BYTES (512 * 1024)
int64_t paradmm_noalloc_state_bytes(int n_circles, int n_walls);
int paradmm_gpu_packing_iterate_noalloc(const paradmm_packing_desc *desc, double *d_circles, void *d_state,
                                        int init_state, int sweeps, double tol, paradmm_stats *stats,
                                        int device, void *stream);

/* ---- errors ---- */
int paradmm_last_status(void);
const char *paradmm_last_error_string(void);

/* ---- engine used by the paradmm.h sweep functions (updateG, ...) ----
 * The drop-in sweep functions build (and cache, per graph pointer, until
 * closeG) a handle with these options. */
void paradmm_set_sweep_options(const paradmm_gpu_opts *opts);

#ifdef __cplusplus
}
#endif

#endif /* PARADMM_B200_PARADMM_GPU_H */
