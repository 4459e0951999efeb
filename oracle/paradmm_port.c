/*
 * ORACLE -- test infrastructure only.  Nothing in the shipped library links,
 * loads or calls this file; only tests/, __graft_entry__.smoke() and the CPU
 * baseline leg of bench.py may use it, and only as the checker.
 *
 * A plain-C restatement of the reference parADMM CPU path, written from the
 * reference's behaviour:
 *   graph construction  core/paradmm.c:79-120, 381-466
 *   initialisation      core/paradmm.c:188-226, 266-375 (optimal)
 *   sweep               core/paradmm.c:569-741  (updateXM, updateZ, updateUN)
 *   OpenMP sweep        core/paradmm.c:949-1092 (same arithmetic, threads)
 *   packing operators   packing/host.c:10-132
 *
 * Every floating-point expression is evaluated in the same order as the
 * reference so that, built with -ffp-contract=off and without fast-math, the
 * results are bit-identical to the reference compiled the same way.  This is
 * pinned by tests/test_oracle.py against oracle/_ref (the reference compiled
 * from its own sources) and against the committed golden fixtures.
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "paradmm.h"

/* ------------------------------------------------------------------ utils */

double abs_d(double x) { return x >= 0 ? x : -x; }

void quicksort(int *a, int n)
{
    /* Only the effect matters (ascending order, core/paradmm.c:28-60). */
    for (int i = 1; i < n; i++) {
        int v = a[i], j = i - 1;
        while (j >= 0 && a[j] > v) { a[j + 1] = a[j]; j--; }
        a[j + 1] = v;
    }
}

double get_random(double lo, double hi) { return ((double)rand() / RAND_MAX) * (hi - lo) + lo; }

void *realloc2(void *p, size_t before, size_t now) { return before == 0 ? malloc(now) : realloc(p, now); }

/* ------------------------------------------------------- graph lifetime */

void startG(graph *G, int numdims)
{
    G->num_dims = numdims;
    G->num_edges = 0;
    G->num_opts = 0;
    G->num_vars = 0;
}

void closeG(graph *G)
{
    free(G->X); free(G->M); free(G->N); free(G->U); free(G->Z);
    free(G->RHOS); free(G->ALPHAS);
    for (int f = 0; f < G->num_opts; f++) free(G->operatorix_to_edgelistix[f]);
    free(G->operatorix_to_edgelistix);
    free(G->list_of_operators_param_pointers);
    free(G->list_of_operators_param_sizes);
    free(G->operatorix_to_numedges);
    free(G->list_of_operators_functions_pointers);
    for (int v = 0; v < G->num_vars; v++) free(G->varix_to_edgelistix[v]);
    free(G->varix_to_edgelistix);
    free(G->varix_to_numedges);
    free(G->edgeix_to_varlistix);
}

void printG(graph *G) { printf("graph: %d factors, %d vars, %d dims, %d edges\n", G->num_opts, G->num_vars, G->num_dims, G->num_edges); }

/* Growth helper: the oracle grows every list one element at a time, which
 * reproduces the reference's resulting structure (core/paradmm.c:405-465). */
static void *grow(void *p, size_t elem, int old_count, int new_count)
{
    void *q = old_count == 0 ? malloc(elem * (size_t)new_count) : realloc(p, elem * (size_t)new_count);
    if (!q) { fprintf(stderr, "oracle: out of memory\n"); exit(EXIT_FAILURE); }
    return q;
}

static void add_factor(graph *G, paradmm_op_fn op, void *params, int param_size, int with_size,
                       int nv, int *vars)
{
    quicksort(vars, nv);
    int f = G->num_opts++;
    int maxv = 0;
    for (int i = 0; i < nv; i++) if (vars[i] > maxv) maxv = vars[i];
    int old_vars = G->num_vars;
    if (G->num_vars < maxv + 1) G->num_vars = maxv + 1;

    G->list_of_operators_functions_pointers = grow(G->list_of_operators_functions_pointers, sizeof(paradmm_op_fn), f, f + 1);
    G->list_of_operators_param_pointers = grow(G->list_of_operators_param_pointers, sizeof(void *), f, f + 1);
    if (with_size) {
        G->list_of_operators_param_sizes = grow(G->list_of_operators_param_sizes, sizeof(int), f, f + 1);
        G->list_of_operators_param_sizes[f] = param_size;
    }
    G->list_of_operators_functions_pointers[f] = op;
    G->list_of_operators_param_pointers[f] = params;

    G->operatorix_to_numedges = grow(G->operatorix_to_numedges, sizeof(int), f, f + 1);
    G->operatorix_to_numedges[f] = nv;
    G->operatorix_to_edgelistix = grow(G->operatorix_to_edgelistix, sizeof(int *), f, f + 1);
    G->operatorix_to_edgelistix[f] = grow(NULL, sizeof(int), 0, nv);
    for (int i = 0; i < nv; i++) G->operatorix_to_edgelistix[f][i] = G->num_edges + i;

    if (G->num_vars > old_vars) {
        G->varix_to_numedges = grow(G->varix_to_numedges, sizeof(int), old_vars, G->num_vars);
        G->varix_to_edgelistix = grow(G->varix_to_edgelistix, sizeof(int *), old_vars, G->num_vars);
        for (int v = old_vars; v < G->num_vars; v++) { G->varix_to_numedges[v] = 0; G->varix_to_edgelistix[v] = NULL; }
    }
    for (int i = 0; i < nv; i++) {
        int v = vars[i];
        int k = G->varix_to_numedges[v]++;
        G->varix_to_edgelistix[v] = grow(G->varix_to_edgelistix[v], sizeof(int), k, k + 1);
        G->varix_to_edgelistix[v][k] = G->num_edges + i;
    }
    G->edgeix_to_varlistix = grow(G->edgeix_to_varlistix, sizeof(int), G->num_edges, G->num_edges + nv);
    for (int i = 0; i < nv; i++) G->edgeix_to_varlistix[G->num_edges + i] = vars[i];
    G->num_edges += nv;
}

void addNode(graph *G, void (*op)(double *, double *, double *, int, int, void *), void *params, int nv, int *vars)
{
    add_factor(G, op, params, 0, 0, nv, vars);
}

void addNodeWithParamSize(graph *G, void (*op)(double *, double *, double *, int, int, void *), void *params,
                          int param_size, int nv, int *vars)
{
    add_factor(G, op, params, param_size, 1, nv, vars);
}

/* ------------------------------------------------------- initialisation */

void initialize_RHOS_APHAS(graph *G, double rho0, double alpha0)
{
    G->RHOS = malloc(sizeof(double) * (size_t)G->num_edges);
    G->ALPHAS = malloc(sizeof(double) * (size_t)G->num_edges);
    for (int e = 0; e < G->num_edges; e++) { G->RHOS[e] = rho0; G->ALPHAS[e] = alpha0; }
}

void initialize_X_N_Z_M_U_zeros(graph *G)
{
    size_t le = (size_t)G->num_dims * G->num_edges, lv = (size_t)G->num_dims * G->num_vars;
    G->X = calloc(le, sizeof(double));
    G->N = calloc(le, sizeof(double));
    G->M = calloc(le, sizeof(double));
    G->U = calloc(le, sizeof(double));
    G->Z = calloc(lv, sizeof(double));
}

/* core/paradmm.c:266-375: Z = Zinit, X_e = Z_v(e), then for every factor
 * `maxiter` rounds of  X~ = op(X - U),  U = -(X - U) + X~  from U = Uinit;
 * N = X - U, M = X + U.  Allocates the state arrays as the reference does.
 * With maxiter = 0 the reference leaves U unset; here it is then 0. */
void initialize_X_N_Z_M_U_optimal(graph *G, double Zinit[], double Uinit[], int maxiter)
{
    const int d = G->num_dims;
    size_t le = (size_t)d * G->num_edges, lv = (size_t)d * G->num_vars;
    G->X = malloc(sizeof(double) * le);
    G->N = malloc(sizeof(double) * le);
    G->M = malloc(sizeof(double) * le);
    G->U = calloc(le, sizeof(double));
    G->Z = malloc(sizeof(double) * lv);
    for (size_t i = 0; i < lv; i++) G->Z[i] = Zinit[i];
    for (int v = 0; v < G->num_vars; v++)
        for (int q = 0; q < G->varix_to_numedges[v]; q++) {
            const int e = G->varix_to_edgelistix[v][q];
            for (int k = 0; k < d; k++) G->X[(size_t)e * d + k] = Zinit[(size_t)v * d + k];
        }
    double *xmu = malloc(sizeof(double) * le), *xi = malloc(sizeof(double) * le);
    double *rh = malloc(sizeof(double) * (size_t)G->num_edges);
    for (size_t i = 0; i < le; i++) { xmu[i] = G->X[i] - Uinit[i]; xi[i] = G->X[i]; }
    for (int e = 0; e < G->num_edges; e++) rh[e] = G->RHOS[e];
    for (int f = 0; f < G->num_opts; f++) {
        const int ne = G->operatorix_to_numedges[f], e0 = G->operatorix_to_edgelistix[f][0];
        const size_t o = (size_t)d * e0;
        for (int it = 0; it < maxiter; it++) {
            G->list_of_operators_functions_pointers[f](&xi[o], &xmu[o], &rh[e0], ne, d,
                                                       G->list_of_operators_param_pointers[f]);
            for (int j = 0; j < d * ne; j++) {
                G->U[o + j] = -xmu[o + j] + xi[o + j];
                xmu[o + j] = G->X[o + j] - G->U[o + j];
            }
        }
    }
    for (size_t i = 0; i < le; i++) { G->M[i] = G->X[i] + G->U[i]; G->N[i] = xmu[i]; }
    free(xi);
    free(rh);
    free(xmu);
}

/* ---------------------------------------------------- packing operators */

/* packing/host.c:10-29: ten Newton steps on the prox of -r^a. */
double max_alpha_radius(double n, double rho, double a)
{
    double r = abs_d(n / 2.0);
    for (int it = 0; it < 10; it++) {
        const double num = -pow(r, a - 1) + (rho / a) * (r - n);
        const double den = -(a - 1) * pow(r, a - 2) + (rho / a);
        r -= num / den;
        if (r < 0) return 0.0;
    }
    return r;
}

/* packing/host.c:31-65: circle (centre edge 0, radius edge 1) kept on the
 * feasible side of the half-plane v.(c - p) + r <= 0, params = [v, p]. */
void disk_plane_collision_variable_radius(double *x, double *n, double *rhos, int numvars, int d, void *params)
{
    const double *v = (const double *)params, *p = v + d;
    double inner = 0;
    for (int k = 0; k < d; k++) inner += v[k] * (n[k] - p[k]);
    if (inner + n[d] > 0) {
        double r = (-inner * rhos[0] + n[d] * rhos[1]) / (rhos[0] + rhos[1]);
        if (r < 0) r = 0;
        for (int k = 0; k < d; k++) {
            x[k] = n[k] - (inner * v[k]) + (-v[k] * r);
            x[k + d] = r;
        }
    } else {
        for (int k = 0; k < d * numvars; k++) x[k] = n[k];
    }
}

/* packing/host.c:67-81: per radius edge, x = argmax of r^a - rho/2 (r-n)^2. */
void maximize_sum_of_squared_disk_radii_alpha(double *x, double *n, double *rhos, int numvars, int d, void *params)
{
    const double a = ((const double *)params)[0];
    for (int i = 0; i < numvars; i++) {
        double r = max_alpha_radius(n[i * d], rhos[i], a);
        for (int k = 0; k < d; k++) x[i * d + k] = r;
    }
}

/* packing/host.c:83-132: two circles [c1, r1, c2, r2] pushed apart along the
 * centre line until r1 + r2 = |c1 - c2| (weighted by the edge penalties). */
void disk_collision_variable_radius(double *x, double *n, double *rhos, int numvars, int d, void *params)
{
    (void)params;
    const double nr1 = n[d], nr2 = n[3 * d];
    double sum2 = (nr1 + nr2);
    sum2 *= sum2;
    double dist2 = 0.0;
    for (int k = 0; k < d; k++) { double t = (n[k] - n[k + 2 * d]); dist2 += (t * t); }
    for (int k = 0; k < d * numvars; k++) x[k] = n[k];
    if (dist2 < sum2) {
        const double nx1 = 0, nx2 = sqrt(dist2);
        const double rx1 = rhos[0], rr1 = rhos[1], rx2 = rhos[2], rr2 = rhos[3];
        const double den = (rr1 * rr2 * rx1 + rr2 * rx1 * rx2 + rr1 * (rr2 + rx1) * rx2);
        const double x1lin = ((-nr1 - nr2 + nx2) * rr1 * rr2 * rx2 + nx1 * rx1 * (rr2 * rx2 + rr1 * (rr2 + rx2))) / den;
        const double x2lin = ((nr1 + nr2 + nx1) * rr1 * rr2 * rx1 + nx2 * (rr2 * rx1 + rr1 * (rr2 + rx1)) * rx2) / den;
        const double r1lin = ((-nr2 - nx1 + nx2) * rr2 * rx1 * rx2 + nr1 * rr1 * (rx1 * rx2 + rr2 * (rx1 + rx2))) / den;
        const double r2lin = ((-nr1 - nx1 + nx2) * rr1 * rx1 * rx2 + nr2 * rr2 * (rx1 * rx2 + rr1 * (rx1 + rx2))) / den;
        for (int k = 0; k < d; k++) {
            const double dir = (n[k + 2 * d] - n[k]) / (nx2);
            x[k + d] = r1lin;
            x[k + 3 * d] = r2lin;
            x[k] += dir * x1lin;
            x[k + 2 * d] += dir * (x2lin - nx2);
        }
    }
}

/* -------------------------------------------------------------- sweep */

static void call_factor(graph *G, int f)
{
    const int d = G->num_dims;
    const int e0 = G->operatorix_to_edgelistix[f][0];
    G->list_of_operators_functions_pointers[f](&G->X[d * e0], &G->N[d * e0], &G->RHOS[e0],
                                               G->operatorix_to_numedges[f], d,
                                               G->list_of_operators_param_pointers[f]);
}

static void z_of_var(graph *G, int v)
{
    const int d = G->num_dims, deg = G->varix_to_numedges[v];
    const int *el = G->varix_to_edgelistix[v];
    double den = 0;
    for (int i = 0; i < deg; i++) den += G->RHOS[el[i]];
    for (int k = 0; k < d; k++) {
        double acc = 0;
        for (int i = 0; i < deg; i++) acc = acc + G->M[d * el[i] + k] * (G->RHOS[el[i]]);
        G->Z[d * v + k] = acc / den;
    }
}

static void u_of_var(graph *G, int v)
{
    const int d = G->num_dims;
    for (int i = 0; i < G->varix_to_numedges[v]; i++) {
        const int e = G->varix_to_edgelistix[v][i];
        const double a = G->ALPHAS[e];
        for (int k = 0; k < d; k++) G->U[e * d + k] += a * (G->X[d * e + k] - G->Z[d * v + k]);
    }
}

static void n_of_var(graph *G, int v)
{
    const int d = G->num_dims;
    for (int i = 0; i < G->varix_to_numedges[v]; i++) {
        const int e = G->varix_to_edgelistix[v][i];
        for (int k = 0; k < d; k++) G->N[e * d + k] = G->Z[d * v + k] - G->U[e * d + k];
    }
}

void update_outgoing_rhos(graph *G) { (void)G; }

void updateX(graph *G) { for (int f = 0; f < G->num_opts; f++) call_factor(G, f); }

void updateM(graph *G)
{
    const long n = (long)G->num_edges * G->num_dims;
    for (long i = 0; i < n; i++) G->M[i] = G->X[i] + G->U[i];
}

void updateXM(graph *G) { updateX(G); updateM(G); }

void updateZ(graph *G)
{
    for (int v = 0; v < G->num_vars; v++) z_of_var(G, v);
    update_outgoing_rhos(G);
}

void updateU(graph *G) { for (int v = 0; v < G->num_vars; v++) u_of_var(G, v); }
void updateN(graph *G) { for (int v = 0; v < G->num_vars; v++) n_of_var(G, v); }

void updateUN(graph *G)
{
    /* core/paradmm.c:675-694 interleaves U then N per edge; per edge the two
     * are independent of other edges, so doing U for a var's edges and then
     * N for the same edges gives identical values. */
    for (int v = 0; v < G->num_vars; v++) { u_of_var(G, v); n_of_var(G, v); }
}

void updateG(graph *G) { updateXM(G); updateZ(G); updateUN(G); }

/* Threaded sweep: every output element is owned by one thread, so the result
 * equals the serial sweep (core/paradmm.c:949-1092). */
void updateGOpenMP(graph *G, int maxiter, int nthreads)
{
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#else
    (void)nthreads;
#endif
    for (int it = 0; it < maxiter; it++) {
        const long ncomp = (long)G->num_edges * G->num_dims;
#pragma omp parallel
        {
#pragma omp for schedule(static)
            for (int f = 0; f < G->num_opts; f++) call_factor(G, f);
#pragma omp for schedule(static)
            for (long i = 0; i < ncomp; i++) G->M[i] = G->X[i] + G->U[i];
#pragma omp for schedule(static)
            for (int v = 0; v < G->num_vars; v++) z_of_var(G, v);
#pragma omp for schedule(static)
            for (int v = 0; v < G->num_vars; v++) u_of_var(G, v);
#pragma omp for schedule(static)
            for (int v = 0; v < G->num_vars; v++) n_of_var(G, v);
        }
    }
}
