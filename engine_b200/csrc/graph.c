/*
 * Host side of the paradmm.h API: graph construction, initialisation,
 * utilities, and the plain-C form of the three packing operators.
 *
 * Builds exactly the data structures of the reference (core/paradmm.c):
 *   - addNode sorts the factor's variable list ascending (core/paradmm.c:383),
 *     gives the factor the next contiguous edge ids (:424-427), appends each
 *     edge to its variable's list in insertion order (:442-453) and records
 *     edge -> variable (:460-465);
 *   - every list is a separate malloc block freed by closeG (:91-120).
 * Lists grow geometrically (capacity = next power of two >= count, derived
 * from the count the struct already holds), so building an N-circle packing
 * graph is O(E) instead of one realloc per edge.
 *
 * The sweep functions (updateX ... updateGOpenMP) live in engine.cu and run
 * on the GPU.
 */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include "paradmm.h"
#include "paradmm_gpu.h"

/* engine.cu: drops the cached sweep handle of a graph being closed */
void paradmm_internal_forget_graph(const graph *G);
/* engine.cu: records a status for paradmm_last_status() */
void paradmm_internal_set_error(int status, const char *msg);

/* ------------------------------------------------------------ utilities */

double abs_d(double x) { return x >= 0 ? x : -x; }

static void isort(int *a, int n)
{
    for (int i = 1; i < n; i++) {
        int v = a[i], j = i - 1;
        while (j >= 0 && a[j] > v) { a[j + 1] = a[j]; j--; }
        a[j + 1] = v;
    }
}

static int cmp_int(const void *x, const void *y)
{
    int a = *(const int *)x, b = *(const int *)y;
    return (a > b) - (a < b);
}

void quicksort(int *array, int n)
{
    if (n <= 16) isort(array, n);
    else qsort(array, (size_t)n, sizeof(int), cmp_int);
}

double get_random(double lo, double hi) { return ((double)rand() / RAND_MAX) * (hi - lo) + lo; }

void *realloc2(void *p, size_t before, size_t now) { return before == 0 ? malloc(now) : realloc(p, now); }

/* ------------------------------------------------------------- growth */

static size_t cap_of(size_t count)
{
    if (count == 0) return 0;
    size_t c = 8;
    while (c < count) c <<= 1;
    return c;
}

/* Makes *pp hold at least new_count elements, given it holds old_count. */
static int ensure(void **pp, size_t elem, size_t old_count, size_t new_count)
{
    size_t oc = cap_of(old_count), nc = cap_of(new_count);
    if (new_count <= oc && old_count > 0) return 0;
    if (nc == oc && old_count > 0) return 0;
    void *q = old_count == 0 ? malloc(elem * nc) : realloc(*pp, elem * nc);
    if (!q) return -1;
    *pp = q;
    return 0;
}

/* --------------------------------------------------------------- graph */

void startG(graph *G, int numdims)
{
    memset(G, 0, sizeof(*G));
    G->num_dims = numdims;
}

void closeG(graph *G)
{
    paradmm_internal_forget_graph(G);
    free(G->X); free(G->M); free(G->N); free(G->U); free(G->Z);
    free(G->RHOS); free(G->ALPHAS);
    if (G->operatorix_to_edgelistix)
        for (int f = 0; f < G->num_opts; f++) free(G->operatorix_to_edgelistix[f]);
    free(G->operatorix_to_edgelistix);
    free(G->list_of_operators_param_pointers);
    free(G->list_of_operators_param_sizes);
    free(G->operatorix_to_numedges);
    free(G->list_of_operators_functions_pointers);
    if (G->varix_to_edgelistix)
        for (int v = 0; v < G->num_vars; v++) free(G->varix_to_edgelistix[v]);
    free(G->varix_to_edgelistix);
    free(G->varix_to_numedges);
    free(G->edgeix_to_varlistix);
    /* leave counts and pointers harmless for a second closeG */
    int d = G->num_dims;
    memset(G, 0, sizeof(*G));
    G->num_dims = d;
}

void printG(graph *G)
{
    printf("number of operator in G is %d\n\n", G->num_opts);
    printf("number of global variables in G is %d\n\n", G->num_vars);
    printf("Dimension of each variable in G is %d\n\n", G->num_dims);
    printf("number of edges in G is %d\n\n", G->num_edges);
    if (G->RHOS) { printf("RHOS\n"); for (int e = 0; e < G->num_edges; e++) printf("%f\n", G->RHOS[e]); printf("\n"); }
    if (G->ALPHAS) { printf("ALPHAS\n"); for (int e = 0; e < G->num_edges; e++) printf("%f\n", G->ALPHAS[e]); printf("\n"); }
    printf("List of operators_pointers\n");
    for (int f = 0; f < G->num_opts; f++) printf("%p\n", (void *)G->list_of_operators_functions_pointers[f]);
    printf("\nList of operatorix_to_numedges\n");
    for (int f = 0; f < G->num_opts; f++) printf("%d\n", G->operatorix_to_numedges[f]);
    printf("\nList of operatorix_to_edgelistin\n");
    for (int f = 0; f < G->num_opts; f++) {
        printf("edge list of operator %d : ", f);
        for (int k = 0; k < G->operatorix_to_numedges[f]; k++) printf("\t%d", G->operatorix_to_edgelistix[f][k]);
        printf("\n");
    }
    printf("\nList of varix_to_numedges\n");
    for (int v = 0; v < G->num_vars; v++) printf("%d\n", G->varix_to_numedges[v]);
    printf("\nList of varix_to_edgelistix\n");
    for (int v = 0; v < G->num_vars; v++) {
        printf("edge list of variable %d : ", v);
        for (int k = 0; k < G->varix_to_numedges[v]; k++) printf("\t%d", G->varix_to_edgelistix[v][k]);
        printf("\n");
    }
    printf("\nList of edgeix_to_varlistix:\n");
    for (int e = 0; e < G->num_edges; e++) printf("%d ", G->edgeix_to_varlistix[e]);
    printf("\n");
}

static void oom(void)
{
    /* The reference prints and exits on allocation failure
     * (core/paradmm.c:196-200); construction keeps that contract because
     * addNode has no way to report an error. */
    fprintf(stderr, "paradmm: out of host memory while building the graph\n");
    exit(EXIT_FAILURE);
}

static void add_factor(graph *G, paradmm_op_fn op, void *params, int param_size, int nv, int *vars)
{
    if (nv < 1 || !vars) { paradmm_internal_set_error(PARADMM_EINVAL, "addNode: a factor needs at least one variable"); return; }
    quicksort(vars, nv);
    for (int i = 0; i < nv; i++)
        if (vars[i] < 0) { paradmm_internal_set_error(PARADMM_EINVAL, "addNode: negative variable index"); return; }
    const int f = G->num_opts;
    const int maxv = vars[nv - 1];
    const int old_vars = G->num_vars;
    const int new_vars = maxv + 1 > old_vars ? maxv + 1 : old_vars;
    const int e0 = G->num_edges;

    if (ensure((void **)&G->list_of_operators_functions_pointers, sizeof(paradmm_op_fn), f, f + 1) ||
        ensure((void **)&G->list_of_operators_param_pointers, sizeof(void *), f, f + 1) ||
        ensure((void **)&G->list_of_operators_param_sizes, sizeof(int), f, f + 1) ||
        ensure((void **)&G->operatorix_to_numedges, sizeof(int), f, f + 1) ||
        ensure((void **)&G->operatorix_to_edgelistix, sizeof(int *), f, f + 1) ||
        ensure((void **)&G->edgeix_to_varlistix, sizeof(int), e0, e0 + nv))
        oom();
    if (new_vars > old_vars) {
        if (ensure((void **)&G->varix_to_numedges, sizeof(int), old_vars, new_vars) ||
            ensure((void **)&G->varix_to_edgelistix, sizeof(int *), old_vars, new_vars))
            oom();
        for (int v = old_vars; v < new_vars; v++) { G->varix_to_numedges[v] = 0; G->varix_to_edgelistix[v] = NULL; }
    }
    int *el = malloc(sizeof(int) * (size_t)nv);
    if (!el) oom();
    for (int i = 0; i < nv; i++) el[i] = e0 + i;

    G->list_of_operators_functions_pointers[f] = op;
    G->list_of_operators_param_pointers[f] = params;
    G->list_of_operators_param_sizes[f] = param_size;
    G->operatorix_to_numedges[f] = nv;
    G->operatorix_to_edgelistix[f] = el;
    for (int i = 0; i < nv; i++) {
        const int v = vars[i];
        const int k = G->varix_to_numedges[v];
        if (ensure((void **)&G->varix_to_edgelistix[v], sizeof(int), (size_t)k, (size_t)k + 1)) oom();
        G->varix_to_edgelistix[v][k] = e0 + i;
        G->varix_to_numedges[v] = k + 1;
        G->edgeix_to_varlistix[e0 + i] = v;
    }
    G->num_opts = f + 1;
    G->num_vars = new_vars;
    G->num_edges = e0 + nv;
}

void addNode(graph *G, void (*op)(double *, double *, double *, int, int, void *), void *params, int nv, int *vars)
{
    add_factor(G, op, params, 0, nv, vars);
}

void addNodeWithParamSize(graph *G, void (*op)(double *, double *, double *, int, int, void *), void *params,
                          int param_size, int nv, int *vars)
{
    add_factor(G, op, params, param_size, nv, vars);
}

/* ---------------------------------------------- bulk packing construction */

int paradmm_add_packing_factors(graph *G, int n, int nw, double *walls, double *exponent, int order)
{
    if (!G || n < 1 || nw < 0 || (nw > 0 && !walls) || !exponent || G->num_dims != 2 || G->num_opts != 0) {
        paradmm_internal_set_error(PARADMM_EINVAL, "paradmm_add_packing_factors: bad arguments or graph not fresh");
        return PARADMM_EINVAL;
    }
    if ((long long)n * (n - 1) / 2 * 4 + (long long)n * (1 + 2 * nw) > 2147483647LL) {
        paradmm_internal_set_error(PARADMM_EINVAL, "paradmm_add_packing_factors: edge count overflows int");
        return PARADMM_EINVAL;
    }
    int v[4];
    for (int pass = 0; pass < 2; ++pass) {
        const int radius_now = (order == 0) ? pass == 0 : pass == 1;
        if (radius_now) {
            for (int i = 0; i < n; i++) { v[0] = 2 * i + 1; addNode(G, maximize_sum_of_squared_disk_radii_alpha, exponent, 1, v); }
        } else {
            for (int w = 0; w < nw; w++)
                for (int i = 0; i < n; i++) { v[0] = 2 * i; v[1] = 2 * i + 1; addNode(G, disk_plane_collision_variable_radius, walls + 4 * w, 2, v); }
        }
    }
    for (int i = 0; i + 1 < n; i++)
        for (int j = i + 1; j < n; j++) {
            v[0] = 2 * i; v[1] = 2 * i + 1; v[2] = 2 * j; v[3] = 2 * j + 1;
            addNode(G, disk_collision_variable_radius, NULL, 4, v);
        }
    return PARADMM_OK;
}

/* ----------------------------------------------------- initialisation */

void initialize_RHOS_APHAS(graph *G, double rho0, double alpha0)
{
    const size_t n = (size_t)G->num_edges;
    G->RHOS = malloc(sizeof(double) * (n ? n : 1));
    G->ALPHAS = malloc(sizeof(double) * (n ? n : 1));
    if (!G->RHOS || !G->ALPHAS) oom();
    for (size_t e = 0; e < n; e++) { G->RHOS[e] = rho0; G->ALPHAS[e] = alpha0; }
}

void initialize_X_N_Z_M_U_zeros(graph *G)
{
    const size_t le = (size_t)G->num_dims * G->num_edges, lv = (size_t)G->num_dims * G->num_vars;
    G->X = calloc(le ? le : 1, sizeof(double));
    G->N = calloc(le ? le : 1, sizeof(double));
    G->M = calloc(le ? le : 1, sizeof(double));
    G->U = calloc(le ? le : 1, sizeof(double));
    G->Z = calloc(lv ? lv : 1, sizeof(double));
    if (!G->X || !G->N || !G->M || !G->U || !G->Z) oom();
}

void initialize_X_N_Z_M_U_rand(graph *G, double X_l, double X_u, double N_l, double N_u, double Z_l, double Z_u,
                               double M_l, double M_u, double U_l, double U_u)
{
    const size_t le = (size_t)G->num_dims * G->num_edges, lv = (size_t)G->num_dims * G->num_vars;
    G->X = malloc(sizeof(double) * (le ? le : 1));
    G->N = malloc(sizeof(double) * (le ? le : 1));
    G->M = malloc(sizeof(double) * (le ? le : 1));
    G->U = malloc(sizeof(double) * (le ? le : 1));
    G->Z = malloc(sizeof(double) * (lv ? lv : 1));
    if (!G->X || !G->N || !G->M || !G->U || !G->Z) oom();
    /* time-seeded like core/paradmm.c:247; draw order X, N, M, U per slot */
    srand((unsigned)time(NULL));
    for (size_t i = 0; i < le; i++) {
        G->X[i] = get_random(X_l, X_u);
        G->N[i] = get_random(N_l, N_u);
        G->M[i] = get_random(M_l, M_u);
        G->U[i] = get_random(U_l, U_u);
    }
    for (size_t i = 0; i < lv; i++) G->Z[i] = get_random(Z_l, Z_u);
}

/* Warm start from a consensus guess (core/paradmm.c:266-375): X_e = Zinit_v(e);
 * each factor's prox is iterated maxiter times on n = X - U, updating
 * U = Xiter - (X - U); then M = X + U and N = X - U.  With maxiter = 0 the
 * reference leaves U uninitialised; here U = Uinit in that case. */
void initialize_X_N_Z_M_U_optimal(graph *G, double Zinit[], double Uinit[], int maxiter)
{
    const int d = G->num_dims;
    const size_t le = (size_t)d * G->num_edges, lv = (size_t)d * G->num_vars;
    G->X = malloc(sizeof(double) * (le ? le : 1));
    G->N = malloc(sizeof(double) * (le ? le : 1));
    G->M = malloc(sizeof(double) * (le ? le : 1));
    G->U = malloc(sizeof(double) * (le ? le : 1));
    G->Z = malloc(sizeof(double) * (lv ? lv : 1));
    double *xmu = malloc(sizeof(double) * (le ? le : 1));
    double *xit = malloc(sizeof(double) * (le ? le : 1));
    double *rh = malloc(sizeof(double) * (G->num_edges ? G->num_edges : 1));
    if (!G->X || !G->N || !G->M || !G->U || !G->Z || !xmu || !xit || !rh) oom();
    memcpy(G->Z, Zinit, sizeof(double) * lv);
    for (int e = 0; e < G->num_edges; e++)
        for (int k = 0; k < d; k++) G->X[(size_t)e * d + k] = Zinit[(size_t)G->edgeix_to_varlistix[e] * d + k];
    for (size_t i = 0; i < le; i++) { xmu[i] = G->X[i] - Uinit[i]; xit[i] = G->X[i]; G->U[i] = Uinit[i]; }
    memcpy(rh, G->RHOS, sizeof(double) * (size_t)G->num_edges);
    for (int f = 0; f < G->num_opts; f++) {
        const int nv = G->operatorix_to_numedges[f];
        const size_t s = (size_t)d * G->operatorix_to_edgelistix[f][0];
        for (int it = 0; it < maxiter; it++) {
            G->list_of_operators_functions_pointers[f](&xit[s], &xmu[s], &rh[s / d], nv, d,
                                                       G->list_of_operators_param_pointers[f]);
            for (int j = 0; j < d * nv; j++) {
                G->U[s + j] = -xmu[s + j] + xit[s + j];
                xmu[s + j] = G->X[s + j] - G->U[s + j];
            }
        }
    }
    for (size_t i = 0; i < le; i++) { G->M[i] = G->X[i] + G->U[i]; G->N[i] = xmu[i]; }
    free(xit); free(rh); free(xmu);
}

/* ---------------------------------------- packing operators, plain C form */

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

void disk_plane_collision_variable_radius(double *x, double *n, double *rhos, int numvars, int d, void *params)
{
    const double *v = (const double *)params, *p = v + d;
    double inner = 0;
    for (int k = 0; k < d; k++) inner += v[k] * (n[k] - p[k]);
    if (inner + n[d] > 0) {
        double r = (-inner * rhos[0] + n[d] * rhos[1]) / (rhos[0] + rhos[1]);
        if (r < 0) r = 0;
        for (int k = 0; k < d; k++) { x[k] = n[k] - (inner * v[k]) + (-v[k] * r); x[k + d] = r; }
    } else {
        for (int k = 0; k < d * numvars; k++) x[k] = n[k];
    }
}

void maximize_sum_of_squared_disk_radii_alpha(double *x, double *n, double *rhos, int numvars, int d, void *params)
{
    const double a = ((const double *)params)[0];
    for (int i = 0; i < numvars; i++) {
        const double r = max_alpha_radius(n[i * d], rhos[i], a);
        for (int k = 0; k < d; k++) x[i * d + k] = r;
    }
}

void disk_collision_variable_radius(double *x, double *n, double *rhos, int numvars, int d, void *params)
{
    (void)params;
    const double nr1 = n[d], nr2 = n[3 * d];
    double s2 = nr1 + nr2;
    s2 *= s2;
    double d2 = 0.0;
    for (int k = 0; k < d; k++) { const double t = n[k] - n[k + 2 * d]; d2 += t * t; }
    for (int k = 0; k < d * numvars; k++) x[k] = n[k];
    if (d2 < s2) {
        const double nx1 = 0, nx2 = sqrt(d2);
        const double rx1 = rhos[0], rr1 = rhos[1], rx2 = rhos[2], rr2 = rhos[3];
        const double den = (rr1 * rr2 * rx1 + rr2 * rx1 * rx2 + rr1 * (rr2 + rx1) * rx2);
        const double x1 = ((-nr1 - nr2 + nx2) * rr1 * rr2 * rx2 + nx1 * rx1 * (rr2 * rx2 + rr1 * (rr2 + rx2))) / den;
        const double x2 = ((nr1 + nr2 + nx1) * rr1 * rr2 * rx1 + nx2 * (rr2 * rx1 + rr1 * (rr2 + rx1)) * rx2) / den;
        const double r1 = ((-nr2 - nx1 + nx2) * rr2 * rx1 * rx2 + nr1 * rr1 * (rx1 * rx2 + rr2 * (rx1 + rx2))) / den;
        const double r2 = ((-nr1 - nx1 + nx2) * rr1 * rx1 * rx2 + nr2 * rr2 * (rx1 * rx2 + rr1 * (rx1 + rx2))) / den;
        for (int k = 0; k < d; k++) {
            const double dir = (n[k + 2 * d] - n[k]) / nx2;
            x[k + d] = r1;
            x[k + 3 * d] = r2;
            x[k] += dir * x1;
            x[k + 2 * d] += dir * (x2 - nx2);
        }
    }
}
