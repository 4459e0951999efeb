/*
 * paradmm.h -- drop-in factor-graph ADMM API of the B200 engine.
 *
 * Source- and binary-compatible with the reference engine's public header
 * (core/paradmm.h:20-115 in parADMM/engine): the `graph` struct keeps the
 * same fields in the same order with the same types, and every function keeps
 * its name, argument list and meaning, so code written against the reference
 * (e.g. packing/host.c) links against libparadmm_b200.so unchanged.
 *
 * What differs is where the work runs.  In this library the sweep functions
 * (updateX ... updateG and the *OpenMP variants) execute on the GPU through
 * the engine in paradmm_gpu.h: the graph's host state is uploaded, the sweeps
 * run as sm_100a kernels, and X, M, N, U and Z are written back in the
 * reference's FP64 [edge][dim] layout.  They return void like the reference;
 * a failure leaves the graph unchanged and is reported by
 * paradmm_last_status() / paradmm_last_error_string() (paradmm_gpu.h).
 *
 * Graph construction (startG, addNode, ...) and initialisation are host code
 * that builds exactly the reference's data structures (edge ids assigned
 * contiguously per factor in insertion order, variable lists sorted
 * ascending, var->edge lists in insertion order).
 */
#ifndef PARADMM_B200_PARADMM_H
#define PARADMM_B200_PARADMM_H

#include <stddef.h>

#ifdef __cplusplus
#define MY_EXTERN_C extern "C"
#else
#define MY_EXTERN_C
#endif

/* Proximal-operator plugin ABI (reference core/paradmm.h:41):
 *   op(x_out, n_in, rhos, numvars, numdims, params)
 * x_out/n_in point at the factor's contiguous edge slice (numvars edges of
 * numdims components each), rhos at the slice's per-edge penalties. */
typedef void (*paradmm_op_fn)(double *, double *, double *, int, int, void *);

/* Unused parameter holder kept for source compatibility
 * (reference core/paradmm.h:22-31). */
typedef struct params_matrix
{
    int flag_1stiter;
    int rows;
    double *A;
    double *B;
    double *R;
    double *ATB;
    double *ATA;
} mparams;

/* Factor graph (reference core/paradmm.h:33-63).  Field order, names and
 * types are part of the ABI. */
typedef struct graphs
{
    int num_opts;   /* number of factors (proximal operators)            */
    int num_vars;   /* number of consensus variables                     */
    int num_dims;   /* components per variable (same for all variables)  */
    int num_edges;  /* number of factor-variable edges                   */

    void (**list_of_operators_functions_pointers)(double *, double *, double *, int, int, void *);
    void **list_of_operators_param_pointers;   /* borrowed, caller-owned   */
    int *list_of_operators_param_sizes;        /* bytes, addNodeWithParamSize */

    int *operatorix_to_numedges;    /* edges per factor                      */
    int **operatorix_to_edgelistix; /* factor -> its (contiguous) edge ids   */

    int *varix_to_numedges;         /* edges per variable                    */
    int **varix_to_edgelistix;      /* variable -> edge ids, insertion order */

    int *edgeix_to_varlistix;       /* edge -> variable                      */

    double *X;  /* num_dims * num_edges, [edge][dim] */
    double *M;  /* num_dims * num_edges              */
    double *N;  /* num_dims * num_edges              */
    double *U;  /* num_dims * num_edges              */

    double *Z;  /* num_dims * num_vars,  [var][dim]  */

    double *RHOS;   /* one penalty per edge     */
    double *ALPHAS; /* one step size per edge   */
} graph;

/* ---- utilities (reference core/paradmm.c:21-73) ---- */
MY_EXTERN_C double abs_d(double x);
MY_EXTERN_C void quicksort(int *array, int n);
MY_EXTERN_C double get_random(double lowerbound, double upperbound);
MY_EXTERN_C void *realloc2(void *ptr, size_t sizesbefore, size_t sizesnow);

/* ---- graph lifetime (reference core/paradmm.c:79-182) ---- */
MY_EXTERN_C void startG(graph *G, int numdims);
MY_EXTERN_C void closeG(graph *G);
MY_EXTERN_C void printG(graph *G);

/* ---- initialisation (reference core/paradmm.c:188-375) ---- */
MY_EXTERN_C void initialize_RHOS_APHAS(graph *G, double rho0, double alpha0);
MY_EXTERN_C void initialize_X_N_Z_M_U_zeros(graph *G);
MY_EXTERN_C void initialize_X_N_Z_M_U_rand(graph *G, double X_l, double X_u, double N_l, double N_u,
                                           double Z_l, double Z_u, double M_l, double M_u,
                                           double U_l, double U_u);
MY_EXTERN_C void initialize_X_N_Z_M_U_optimal(graph *G, double Zinit[], double Uinit[], int maxiter);

/* ---- construction (reference core/paradmm.c:381-558) ---- */
MY_EXTERN_C void addNode(graph *G, void (*op)(double *, double *, double *, int, int, void *),
                         void *op_params, int op_numvars, int *listvarix);
MY_EXTERN_C void addNodeWithParamSize(graph *G, void (*op)(double *, double *, double *, int, int, void *),
                                      void *op_params, int op_param_size, int op_numvars, int *listvarix);

/* ---- the sweep (reference core/paradmm.c:564-741), GPU-backed here ---- */
MY_EXTERN_C void update_outgoing_rhos(graph *G);

MY_EXTERN_C void updateXM(graph *G);
MY_EXTERN_C void updateX(graph *G);
MY_EXTERN_C void updateM(graph *G);

MY_EXTERN_C void updateZ(graph *G);

MY_EXTERN_C void updateUN(graph *G);
MY_EXTERN_C void updateU(graph *G);
MY_EXTERN_C void updateN(graph *G);

MY_EXTERN_C void updateG(graph *G);

/* ---- multi-sweep entry points (reference core/paradmm.c:812-1092) ----
 * Declared unconditionally: in this library they run on the GPU and
 * `numthreads` only sizes the host-side staging threads. */
MY_EXTERN_C void updateXOpenMP(graph *G);
MY_EXTERN_C void updateMOpenMP(graph *G);
MY_EXTERN_C void updateZOpenMP(graph *G);
MY_EXTERN_C void updateUOpenMP(graph *G);
MY_EXTERN_C void updateNOpenMP(graph *G);
MY_EXTERN_C void updateGOpenMP(graph *G, int maxiter, int numthreads);

/* ---- circle-packing proximal operators (reference packing/host.c:10-132) ----
 * Exported with the reference names and the plugin ABI so packing graphs can
 * be built against this library.  The engine recognises these (and any
 * operator registered with paradmm_gpu_register_op) and runs its own fused
 * device kernels for them; the host bodies are the operators' plain-C form
 * for callers that invoke an operator directly. */
MY_EXTERN_C double max_alpha_radius(double n, double rho, double alpha);
MY_EXTERN_C void disk_plane_collision_variable_radius(double *x, double *n, double *rhos, int numvars, int numdims, void *params);
MY_EXTERN_C void maximize_sum_of_squared_disk_radii_alpha(double *x, double *n, double *rhos, int numvars, int numdims, void *params);
MY_EXTERN_C void disk_collision_variable_radius(double *x, double *n, double *rhos, int numvars, int numdims, void *params);

#endif /* PARADMM_B200_PARADMM_H */
