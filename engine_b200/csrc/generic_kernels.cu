// Generic CSR engine: any graph built from the three packing operators, any
// number of dimensions, per-edge penalties and steps, FP64 or FP32 state.
//
// It keeps the reference data layout ([edge][dim] arrays X, M, N, U, Z) and
// restates each phase of the reference sweep as one kernel:
//   gen_x   updateX / updateXM  (core/paradmm.c:569-623): one thread per factor
//   gen_m   updateM             (core/paradmm.c:625-634)
//   gen_z   updateZ             (core/paradmm.c:637-672): one thread per
//           variable, edges summed in insertion order (CSR of var -> edges)
//   gen_u / gen_n / gen_un  updateU / updateN / updateUN (core/paradmm.c:675-734)
// This file is compiled with -fmad=false, and every expression keeps the
// reference's evaluation order, so in FP64 the results are bit-identical to
// the reference built without fast-math and with -ffp-contract=off.
#include "common.cuh"
#include "generic.cuh"

// ---------------------------------------------------------------------------
// Operators on the factor's edge slice (packing/host.c:10-132), in T.
// ---------------------------------------------------------------------------
template <typename T>
__device__ T gen_pow(T r, T e)
{
    // exact for the exponents the radius reward uses (r^1 = r, r^0 = 1)
    if (e == (T)1) return r;
    if (e == (T)0) return (T)1;
    if (e == (T)-1) return (T)1 / r;
    return (T)pow((double)r, (double)e);
}

template <typename T>
__device__ T gen_max_alpha_radius(T n, T rho, T a)
{
    T r = n / (T)2.0;
    r = r >= 0 ? r : -r;
    for (int it = 0; it < 10; ++it) {
        const T num = -gen_pow(r, a - 1) + (rho / a) * (r - n);
        const T den = -(a - 1) * gen_pow(r, a - 2) + (rho / a);
        r -= num / den;
        if (r < 0) return (T)0.0;
    }
    return r;
}

template <typename T>
__device__ void gen_op_radius(T *x, const T *n, const double *rhos, int nv, int d, const double *params)
{
    const T a = (T)params[0];
    for (int i = 0; i < nv; ++i) {
        const T r = gen_max_alpha_radius(n[i * d], (T)rhos[i], a);
        for (int k = 0; k < d; ++k) x[i * d + k] = r;
    }
}

template <typename T>
__device__ void gen_op_wall(T *x, const T *n, const double *rhos, int nv, int d, const double *params)
{
    const double *v = params, *p = params + d;
    T inner = 0;
    for (int k = 0; k < d; ++k) inner += (T)v[k] * (n[k] - (T)p[k]);
    if (inner + n[d] > 0) {
        const T r0 = (T)rhos[0], r1 = (T)rhos[1];
        T r = (-inner * r0 + n[d] * r1) / (r0 + r1);
        if (r < 0) r = 0;
        for (int k = 0; k < d; ++k) {
            const T vk = (T)v[k];
            x[k] = n[k] - (inner * vk) + (-vk * r);
            x[k + d] = r;
        }
    } else {
        for (int k = 0; k < d * nv; ++k) x[k] = n[k];
    }
}

template <typename T>
__device__ void gen_op_pair(T *x, const T *n, const double *rhos, int nv, int d)
{
    const T nr1 = n[d], nr2 = n[3 * d];
    T s2 = (nr1 + nr2);
    s2 *= s2;
    T d2 = 0.0;
    for (int k = 0; k < d; ++k) { const T t = (n[k] - n[k + 2 * d]); d2 += (t * t); }
    for (int k = 0; k < d * nv; ++k) x[k] = n[k];
    if (d2 < s2) {
        const T nx1 = 0, nx2 = sqrt(d2);
        const T rx1 = (T)rhos[0], rr1 = (T)rhos[1], rx2 = (T)rhos[2], rr2 = (T)rhos[3];
        const T den = (rr1 * rr2 * rx1 + rr2 * rx1 * rx2 + rr1 * (rr2 + rx1) * rx2);
        const T x1 = ((-nr1 - nr2 + nx2) * rr1 * rr2 * rx2 + nx1 * rx1 * (rr2 * rx2 + rr1 * (rr2 + rx2))) / den;
        const T x2 = ((nr1 + nr2 + nx1) * rr1 * rr2 * rx1 + nx2 * (rr2 * rx1 + rr1 * (rr2 + rx1)) * rx2) / den;
        const T r1 = ((-nr2 - nx1 + nx2) * rr2 * rx1 * rx2 + nr1 * rr1 * (rx1 * rx2 + rr2 * (rx1 + rx2))) / den;
        const T r2 = ((-nr1 - nx1 + nx2) * rr1 * rx1 * rx2 + nr2 * rr2 * (rx1 * rx2 + rr1 * (rx1 + rx2))) / den;
        for (int k = 0; k < d; ++k) {
            const T dir = (n[k + 2 * d] - n[k]) / (nx2);
            x[k + d] = r1;
            x[k + 3 * d] = r2;
            x[k] += dir * x1;
            x[k + 2 * d] += dir * (x2 - nx2);
        }
    }
}

// ---------------------------------------------------------------------------
// Phase kernels.
// ---------------------------------------------------------------------------
template <typename T>
__global__ void gen_x(GenDev G, int with_m)
{
    T *X = (T *)G.X;
    const T *Nn = (const T *)G.N, *U = (const T *)G.U;
    T *M = (T *)G.M;
    const int d = G.num_dims;
    for (int f = blockIdx.x * blockDim.x + threadIdx.x; f < G.num_opts; f += gridDim.x * blockDim.x) {
        const long long e0 = G.f_e0[f];
        const int nv = G.f_nv[f];
        const int kind = G.f_kind[f];
        const double *prm = G.f_param[f] >= 0 ? G.params + G.f_param[f] : nullptr;
        T *x = X + e0 * d;
        const T *n = Nn + e0 * d;
        const double *rh = G.RHOS + e0;
        if (kind == PARADMM_OP_USER) continue;  // run-time compiled operators: their own kernel
        if (kind == PARADMM_OP_PAIR) gen_op_pair<T>(x, n, rh, nv, d);
        else if (kind == PARADMM_OP_WALL) gen_op_wall<T>(x, n, rh, nv, d, prm);
        else gen_op_radius<T>(x, n, rh, nv, d, prm);
        if (with_m)
            for (int k = 0; k < nv * d; ++k) M[e0 * d + k] = x[k] + U[e0 * d + k];
    }
}

template <typename T>
__global__ void gen_m(GenDev G)
{
    const T *X = (const T *)G.X, *U = (const T *)G.U;
    T *M = (T *)G.M;
    const long long n = (long long)G.num_edges * G.num_dims;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        M[i] = X[i] + U[i];
}

template <typename T>
__global__ void gen_z(GenDev G)
{
    const T *M = (const T *)G.M;
    const int d = G.num_dims;
    for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < G.num_vars; v += gridDim.x * blockDim.x) {
        const long long b = G.v_off[v], e = G.v_off[v + 1];
        double den = 0;
        for (long long i = b; i < e; ++i) den += G.RHOS[G.v_edges[i]];
        for (int k = 0; k < d; ++k) {
            double acc = 0;
            for (long long i = b; i < e; ++i) {
                const long long ed = G.v_edges[i];
                acc = acc + (double)M[d * ed + k] * (G.RHOS[ed]);
            }
            G.Z[(long long)d * v + k] = acc / den;
        }
    }
}

template <typename T>
__global__ void gen_un(GenDev G, int do_u, int do_n)
{
    T *U = (T *)G.U, *Nn = (T *)G.N;
    const T *X = (const T *)G.X;
    const int d = G.num_dims;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < G.num_edges; e += (long long)gridDim.x * blockDim.x) {
        const long long v = G.e2v[e];
        const T a = (T)G.ALPHAS[e];
        for (int k = 0; k < d; ++k) {
            const T z = (T)G.Z[d * v + k];
            if (do_u) U[e * d + k] += a * (X[d * e + k] - z);
            if (do_n) Nn[e * d + k] = z - U[e * d + k];
        }
    }
}

// A balancing step of the penalties (no reference counterpart: its hook,
// update_outgoing_rhos, is empty, core/paradmm.c:564-566): every penalty
// times t (t = 2 or 1/2: exact), every scaled dual U divided by t so that
// rho U is unchanged, and N = Z - U again.
template <typename T>
__global__ void gen_rescale(GenDev G, double t)
{
    T *U = (T *)G.U, *Nn = (T *)G.N;
    double *R = const_cast<double *>(G.RHOS);
    const int d = G.num_dims;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < G.num_edges; e += (long long)gridDim.x * blockDim.x) {
        R[e] *= t;
        const long long v = G.e2v[e];
        for (int k = 0; k < d; ++k) {
            U[e * d + k] /= (T)t;
            Nn[e * d + k] = (T)G.Z[d * v + k] - U[e * d + k];
        }
    }
}

// Sum of squares of X - Z_v(e) and of Z_v(e) - Zprev_v(e) over all (edge,
// dim), accumulated into out[0], out[1].
template <typename T>
__global__ void gen_resid(GenDev G, const double *Zprev, double *out)
{
    const T *X = (const T *)G.X;
    const int d = G.num_dims;
    double sp = 0, sd = 0;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < G.num_edges; e += (long long)gridDim.x * blockDim.x) {
        const long long v = G.e2v[e];
        for (int k = 0; k < d; ++k) {
            const double z = G.Z[d * v + k];
            const double t = (double)X[d * e + k] - z;
            sp += t * t;
            if (Zprev) { const double q = z - Zprev[d * v + k]; sd += q * q; }
        }
    }
    sp = block_sum(sp);
    sd = block_sum(sd);
    if (threadIdx.x == 0) { atomicAdd(&out[0], sp); atomicAdd(&out[1], sd); }
}

// Max violation over the factors (pair overlap, wall penetration, -r) from Z.
__global__ void gen_violation(GenDev G, unsigned long long *out)
{
    const int d = G.num_dims;
    double m = 0.0;
    for (int f = blockIdx.x * blockDim.x + threadIdx.x; f < G.num_opts; f += gridDim.x * blockDim.x) {
        const long long e0 = G.f_e0[f];
        const int kind = G.f_kind[f];
        if (kind == PARADMM_OP_PAIR) {
            const long long c1 = G.e2v[e0], r1 = G.e2v[e0 + 1], c2 = G.e2v[e0 + 2], r2 = G.e2v[e0 + 3];
            double dd = 0;
            for (int k = 0; k < d; ++k) { const double t = G.Z[d * c1 + k] - G.Z[d * c2 + k]; dd += t * t; }
            m = fmax(m, G.Z[d * r1] + G.Z[d * r2] - sqrt(dd));
        } else if (kind == PARADMM_OP_WALL) {
            const double *prm = G.params + G.f_param[f];
            const long long c = G.e2v[e0], r = G.e2v[e0 + 1];
            double g = 0;
            for (int k = 0; k < d; ++k) g += prm[k] * (G.Z[d * c + k] - prm[d + k]);
            m = fmax(m, g + G.Z[d * r]);
        } else if (kind == PARADMM_OP_RADIUS) {
            for (int i = 0; i < G.f_nv[f]; ++i) m = fmax(m, -G.Z[d * (long long)G.e2v[e0 + i]]);
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) atomicMax(out, (unsigned long long)__double_as_longlong(m));
}

// ---------------------------------------------------------------------------
// Launchers.
// ---------------------------------------------------------------------------
static int grid_for(long long n, int threads)
{
    long long g = (n + threads - 1) / threads;
    if (g < 1) g = 1;
    if (g > 148 * 32) g = 148 * 32;
    return (int)g;
}

cudaError_t gen_launch_phase(const GenDev &G, int phase, cudaStream_t s)
{
    const int th = 256;
    const bool f64 = G.fp64 != 0;
    switch (phase) {
    case GEN_PHASE_X:
    case GEN_PHASE_XM:
        if (f64) gen_x<double><<<grid_for(G.num_opts, th), th, 0, s>>>(G, phase == GEN_PHASE_XM);
        else gen_x<float><<<grid_for(G.num_opts, th), th, 0, s>>>(G, phase == GEN_PHASE_XM);
        break;
    case GEN_PHASE_M:
        if (f64) gen_m<double><<<grid_for((long long)G.num_edges * G.num_dims, th), th, 0, s>>>(G);
        else gen_m<float><<<grid_for((long long)G.num_edges * G.num_dims, th), th, 0, s>>>(G);
        break;
    case GEN_PHASE_Z:
        if (f64) gen_z<double><<<grid_for(G.num_vars, 128), 128, 0, s>>>(G);
        else gen_z<float><<<grid_for(G.num_vars, 128), 128, 0, s>>>(G);
        break;
    case GEN_PHASE_U:
    case GEN_PHASE_N:
    case GEN_PHASE_UN: {
        const int du = phase != GEN_PHASE_N, dn = phase != GEN_PHASE_U;
        if (f64) gen_un<double><<<grid_for(G.num_edges, th), th, 0, s>>>(G, du, dn);
        else gen_un<float><<<grid_for(G.num_edges, th), th, 0, s>>>(G, du, dn);
        break;
    }
    default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

cudaError_t gen_launch_resid(const GenDev &G, const double *Zprev, double *out, cudaStream_t s)
{
    if (G.fp64) gen_resid<double><<<grid_for(G.num_edges, 256), 256, 0, s>>>(G, Zprev, out);
    else gen_resid<float><<<grid_for(G.num_edges, 256), 256, 0, s>>>(G, Zprev, out);
    return cudaGetLastError();
}

cudaError_t gen_launch_rescale(const GenDev &G, double t, cudaStream_t s)
{
    if (G.fp64) gen_rescale<double><<<grid_for(G.num_edges, 256), 256, 0, s>>>(G, t);
    else gen_rescale<float><<<grid_for(G.num_edges, 256), 256, 0, s>>>(G, t);
    return cudaGetLastError();
}

cudaError_t gen_launch_violation(const GenDev &G, unsigned long long *out, cudaStream_t s)
{
    gen_violation<<<grid_for(G.num_opts, 256), 256, 0, s>>>(G, out);
    return cudaGetLastError();
}
