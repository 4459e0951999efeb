/*
 * ORACLE -- test infrastructure only (see paradmm_port.c).
 *
 * Packing-problem harness shared by the two oracle builds:
 *   oracle/libparadmm_port.so       harness + the C restatement
 *   oracle/_ref/libparadmm_ref.so   harness + the reference's own sources
 * It builds the circle-packing factor graph through addNode in the order the
 * reference demo uses (packing/host.c:299-335: radius factors, then walls,
 * then pairs), seeds the initial state deterministically (the reference's
 * initialize_X_N_Z_M_U_rand is time-seeded, core/paradmm.c:247, so it is
 * never used), and computes the residuals and packing metrics.
 */
#ifndef ORACLE_HARNESS_H
#define ORACLE_HARNESS_H

#include <stdint.h>
#include "paradmm.h"

#define ORC_MAX_WALLS 8

typedef struct orc_packing {
    graph G;
    int N;                       /* circles: var 2i = centre, 2i+1 = radius */
    int nwalls;
    int order;                   /* 0: radius, walls, pairs (packing/host.c) */
                                 /* 1: walls, radius, pairs (packing/gpu.cu) */
    double walls[ORC_MAX_WALLS][4];  /* [v_x, v_y, p_x, p_y] per half-plane */
    double exponent[1];          /* radius-reward exponent (params[0])      */
} orc_packing;

/* splitmix64 stream; u01 = top 53 bits / 2^53. */
uint64_t orc_splitmix64(uint64_t *state);
double orc_u01(uint64_t *state);

orc_packing *orc_packing_new(int N, int nwalls, const double *walls, double exponent, int order);
void orc_packing_free(orc_packing *P);
graph *orc_packing_graph(orc_packing *P);

/* Seeded plain init: circle i draws cx = W u, cy = H u, r = rmax u (in that
 * order).  Z <- those, X_e = N_e = M_e = Z_v(e), U = 0 (both dims of a
 * radius variable hold r).  RHOS = rho, ALPHAS = alpha, and the edges of the
 * radius factors get rho_radius. */
void orc_packing_init(orc_packing *P, uint64_t seed, double W, double H, double rmax,
                      double rho, double rho_radius, double alpha);

/* out[0] primal r = RMS over all (edge, dim) of X - Z_v(e)
 * out[1] dual   s = RMS over all (edge, dim) of Z_v(e) - Zprev_v(e)  (NaN if Zprev NULL)
 * out[2] max violation (>= 0): pair overlap, wall penetration, negative radius
 * out[3] total radius = sum of Z radius dim 0 */
void orc_packing_metrics(orc_packing *P, const double *Zprev, double out[4]);

/* Runs up to `iters` sweeps (nthreads == 0: updateG, else updateGOpenMP(G,1,nthreads)).
 * trace (iters x 4, may be NULL) gets the metrics after every sweep.  Stops
 * early when tol > 0 and r + s <= tol.  Returns the sweeps done. */
int orc_packing_run(orc_packing *P, int iters, int nthreads, double tol, double *trace);

/* Residual balancing of the penalties between sweeps.  The reference has a
 * hook for it and nothing in it: update_outgoing_rhos (core/paradmm.c:564-566,
 * called at the end of updateZ, :671) is empty.  This is the rule the engine
 * implements (paradmm_gpu_set_rho_balance), restated over the reference's
 * own updateG:
 *   - sweeps are counted from the state this call starts from (the sweep
 *     that produces iterate a has age a = 1, 2, ...);
 *   - after every sweep the residuals r_a, s_a are computed (out[0..1] of
 *     orc_packing_metrics, without the O(N^2) packing metrics);
 *   - at ages a with a % period == 0 the rule decides from (r_a, s_a):
 *     r_a > mu s_a and log2 scale < lmax: double every penalty;
 *     s_a > mu r_a and log2 scale > lmin: halve every penalty; else nothing;
 *   - a decision made at age a is applied after the sweep of age a + 2:
 *     every RHOS entry times t (t = 2 or 1/2), every U entry divided by t
 *     (the scaled dual keeps rho U fixed), N = Z - U.
 * Scaling by a power of two is exact, and the pair and wall operators and
 * the consensus weights are homogeneous in the penalties, so only the radius
 * operator (absolute rho) and the dual scale see the change.  period >= 3.
 * trace (iters x 4, may be NULL): r, s, log2 scale in force for the next
 * sweep, and +1 / -1 / 0 for a doubling / halving / nothing applied after
 * that sweep.  Returns the sweeps done (stops when tol > 0 and r + s <= tol). */
int orc_packing_run_balanced(orc_packing *P, int iters, double tol, int period, double mu, int lmin, int lmax,
                             double *trace);

/* Wall-clock seconds of `iters` sweeps: updateG (nthreads == 0) or one
 * updateGOpenMP(G, iters, nthreads) call. */
double orc_time_sweeps(graph *G, int iters, int nthreads);

/* Host threads available to OpenMP in this build. */
int orc_max_threads(void);

#endif
