/*
 * ORACLE -- test infrastructure only (see harness.h).
 */
#define _POSIX_C_SOURCE 199309L
#include "harness.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>
#ifdef _OPENMP
#include <omp.h>
#endif

uint64_t orc_splitmix64(uint64_t *s)
{
    uint64_t z = (*s += 0x9E3779B97F4A7C15ULL);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

double orc_u01(uint64_t *s) { return (double)(orc_splitmix64(s) >> 11) * (1.0 / 9007199254740992.0); }

static void add_radius_factors(orc_packing *P)
{
    for (int i = 0; i < P->N; i++) {
        int v[1] = {2 * i + 1};
        addNode(&P->G, maximize_sum_of_squared_disk_radii_alpha, P->exponent, 1, v);
    }
}

static void add_wall_factors(orc_packing *P)
{
    for (int w = 0; w < P->nwalls; w++)
        for (int i = 0; i < P->N; i++) {
            int v[2] = {2 * i, 2 * i + 1};
            addNode(&P->G, disk_plane_collision_variable_radius, P->walls[w], 2, v);
        }
}

static void add_pair_factors(orc_packing *P)
{
    for (int i = 0; i + 1 < P->N; i++)
        for (int j = i + 1; j < P->N; j++) {
            int v[4] = {2 * i, 2 * i + 1, 2 * j, 2 * j + 1};
            addNode(&P->G, disk_collision_variable_radius, NULL, 4, v);
        }
}

orc_packing *orc_packing_new(int N, int nwalls, const double *walls, double exponent, int order)
{
    if (N < 1 || nwalls < 0 || nwalls > ORC_MAX_WALLS) return NULL;
    orc_packing *P = calloc(1, sizeof(orc_packing));
    if (!P) return NULL;
    P->N = N;
    P->nwalls = nwalls;
    P->order = order;
    P->exponent[0] = exponent;
    memcpy(P->walls, walls, sizeof(double) * 4 * (size_t)nwalls);
    startG(&P->G, 2);
    if (order == 0) { add_radius_factors(P); add_wall_factors(P); }
    else { add_wall_factors(P); add_radius_factors(P); }
    add_pair_factors(P);
    return P;
}

void orc_packing_free(orc_packing *P)
{
    if (!P) return;
    closeG(&P->G);
    free(P);
}

graph *orc_packing_graph(orc_packing *P) { return &P->G; }

void orc_packing_init(orc_packing *P, uint64_t seed, double W, double H, double rmax,
                      double rho, double rho_radius, double alpha)
{
    graph *G = &P->G;
    initialize_X_N_Z_M_U_zeros(G);
    initialize_RHOS_APHAS(G, rho, alpha);
    for (int f = 0; f < G->num_opts; f++)
        if (G->list_of_operators_functions_pointers[f] == maximize_sum_of_squared_disk_radii_alpha)
            for (int k = 0; k < G->operatorix_to_numedges[f]; k++)
                G->RHOS[G->operatorix_to_edgelistix[f][k]] = rho_radius;
    uint64_t s = seed;
    for (int i = 0; i < P->N; i++) {
        double cx = W * orc_u01(&s), cy = H * orc_u01(&s), r = rmax * orc_u01(&s);
        G->Z[4 * i + 0] = cx; G->Z[4 * i + 1] = cy;
        G->Z[4 * i + 2] = r;  G->Z[4 * i + 3] = r;
    }
    const int d = G->num_dims;
    for (int e = 0; e < G->num_edges; e++) {
        const int v = G->edgeix_to_varlistix[e];
        for (int k = 0; k < d; k++) {
            const double z = G->Z[d * v + k];
            G->X[d * e + k] = z; G->N[d * e + k] = z; G->M[d * e + k] = z; G->U[d * e + k] = 0.0;
        }
    }
}

void orc_packing_metrics(orc_packing *P, const double *Zprev, double out[4])
{
    graph *G = &P->G;
    const int d = G->num_dims;
    double sp = 0, sd = 0;
    for (int e = 0; e < G->num_edges; e++) {
        const int v = G->edgeix_to_varlistix[e];
        for (int k = 0; k < d; k++) {
            const double t = G->X[d * e + k] - G->Z[d * v + k];
            sp += t * t;
            if (Zprev) { const double q = G->Z[d * v + k] - Zprev[d * v + k]; sd += q * q; }
        }
    }
    const double n = (double)G->num_edges * d;
    out[0] = sqrt(sp / n);
    out[1] = Zprev ? sqrt(sd / n) : NAN;
    const double *Z = G->Z;
    double viol = 0, total = 0;
    for (int i = 0; i < P->N; i++) {
        const double cx = Z[4 * i], cy = Z[4 * i + 1], r = Z[4 * i + 2];
        total += r;
        if (-r > viol) viol = -r;
        for (int w = 0; w < P->nwalls; w++) {
            const double *W = P->walls[w];
            const double g = W[0] * (cx - W[2]) + W[1] * (cy - W[3]) + r;
            if (g > viol) viol = g;
        }
        for (int j = i + 1; j < P->N; j++) {
            const double dx = cx - Z[4 * j], dy = cy - Z[4 * j + 1];
            const double g = r + Z[4 * j + 2] - sqrt(dx * dx + dy * dy);
            if (g > viol) viol = g;
        }
    }
    out[2] = viol;
    out[3] = total;
}

/* The reference's updateGOpenMP splits its loops as id * N / numthreads in
 * int (core/paradmm.c:964-965, 990-991, ...), N up to num_edges * num_dims:
 * more threads than INT_MAX / N overflow and write outside the arrays, so
 * the harness never asks for more. */
static int orc_safe_threads(const graph *G, int nthreads)
{
    long long n = (long long)G->num_edges * G->num_dims;
    if (G->num_opts > n) n = G->num_opts;
    if (G->num_vars > n) n = G->num_vars;
    if (n < 1) n = 1;
    const long long cap = 2147483647LL / n;
    if (nthreads > cap) nthreads = (int)(cap < 1 ? 1 : cap);
    return nthreads;
}

int orc_packing_run(orc_packing *P, int iters, int nthreads, double tol, double *trace)
{
    graph *G = &P->G;
    if (nthreads > 0) nthreads = orc_safe_threads(G, nthreads);
    const size_t zn = (size_t)G->num_dims * G->num_vars;
    double *Zprev = malloc(sizeof(double) * zn);
    int done = 0;
    for (int it = 0; it < iters; it++) {
        memcpy(Zprev, G->Z, sizeof(double) * zn);
        if (nthreads == 0) updateG(G); else updateGOpenMP(G, 1, nthreads);
        done++;
        if (trace || tol > 0) {
            double m[4];
            orc_packing_metrics(P, Zprev, m);
            if (trace) memcpy(trace + 4 * (size_t)it, m, sizeof m);
            if (tol > 0 && m[0] + m[1] <= tol) break;
        }
    }
    free(Zprev);
    return done;
}

static void orc_residuals(const graph *G, const double *Zprev, double *r, double *s)
{
    const int d = G->num_dims;
    double sp = 0, sd = 0;
    for (int e = 0; e < G->num_edges; e++) {
        const int v = G->edgeix_to_varlistix[e];
        for (int k = 0; k < d; k++) {
            const double t = G->X[d * e + k] - G->Z[d * v + k];
            const double q = G->Z[d * v + k] - Zprev[d * v + k];
            sp += t * t;
            sd += q * q;
        }
    }
    const double n = (double)G->num_edges * d;
    *r = sqrt(sp / n);
    *s = sqrt(sd / n);
}

int orc_packing_run_balanced(orc_packing *P, int iters, double tol, int period, double mu, int lmin, int lmax,
                             double *trace)
{
    graph *G = &P->G;
    if (period < 3) return -1;
    const int d = G->num_dims;
    const size_t zn = (size_t)d * G->num_vars;
    double *Zprev = malloc(sizeof(double) * zn);
    int done = 0, log2s = 0, pending = 0, apply_age = -1;
    for (int it = 0; it < iters; it++) {
        const int age = it + 1;
        memcpy(Zprev, G->Z, sizeof(double) * zn);
        updateG(G);
        done++;
        double r, s;
        orc_residuals(G, Zprev, &r, &s);
        int applied = 0;
        if (age == apply_age && pending != 0) {
            const double t = pending > 0 ? 2.0 : 0.5;
            for (int e = 0; e < G->num_edges; e++) G->RHOS[e] *= t;
            for (int e = 0; e < G->num_edges; e++) {
                const int v = G->edgeix_to_varlistix[e];
                for (int k = 0; k < d; k++) {
                    G->U[d * e + k] /= t;
                    G->N[d * e + k] = G->Z[d * v + k] - G->U[d * e + k];
                }
            }
            log2s += pending;
            applied = pending;
            pending = 0;
        }
        if (age % period == 0) {
            if (r > mu * s && log2s < lmax) pending = 1;
            else if (s > mu * r && log2s > lmin) pending = -1;
            else pending = 0;
            apply_age = age + 2;
        }
        if (trace) {
            trace[4 * (size_t)it + 0] = r;
            trace[4 * (size_t)it + 1] = s;
            trace[4 * (size_t)it + 2] = log2s;
            trace[4 * (size_t)it + 3] = applied;
        }
        if (tol > 0 && r + s <= tol) break;
    }
    free(Zprev);
    return done;
}

static double now_s(void)
{
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return ts.tv_sec + 1e-9 * ts.tv_nsec;
}

double orc_time_sweeps(graph *G, int iters, int nthreads)
{
    if (nthreads > 0) nthreads = orc_safe_threads(G, nthreads);
    const double t0 = now_s();
    if (nthreads == 0) for (int it = 0; it < iters; it++) updateG(G);
    else updateGOpenMP(G, iters, nthreads);
    return now_s() - t0;
}

int orc_max_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
