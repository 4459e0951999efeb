// Generic CSR engine: device view and launchers (generic_kernels.cu).
#pragma once

#include <cuda_runtime.h>

enum { GEN_PHASE_X = 0, GEN_PHASE_M, GEN_PHASE_XM, GEN_PHASE_Z, GEN_PHASE_U, GEN_PHASE_N, GEN_PHASE_UN };

struct GenDev {
    int num_dims, num_vars, num_edges, num_opts;
    int fp64;               // state type: 1 double, 0 float
    int pad;
    // factors
    const int *f_kind;      // PARADMM_OP_*
    const long long *f_e0;  // first edge of the factor's contiguous slice
    const int *f_nv;        // edges of the factor
    const long long *f_param;  // offset into params (doubles), -1 if none
    const double *params;
    // incidence
    const int *e2v;         // edge -> variable
    const long long *v_off; // var -> [v_off[v], v_off[v+1]) in v_edges
    const int *v_edges;     // edges of each variable in insertion order
    // state: [edge][dim] arrays of T, Z [var][dim] double
    void *X, *M, *N, *U;
    double *Z;
    const double *RHOS, *ALPHAS;
};

cudaError_t gen_launch_phase(const GenDev &G, int phase, cudaStream_t s);
cudaError_t gen_launch_resid(const GenDev &G, const double *Zprev, double *out, cudaStream_t s);
cudaError_t gen_launch_violation(const GenDev &G, unsigned long long *out, cudaStream_t s);
cudaError_t gen_launch_rescale(const GenDev &G, double t, cudaStream_t s);
