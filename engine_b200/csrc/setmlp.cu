// Learned proposal for circle packing: a permutation-equivariant set MLP that
// maps each instance's plain start (and geometric context) to a guess of the
// converged packing, used to warm-start the ADMM engine.
//
// Per circle i of an instance with N circles in a W x H box, features
// (device kernel sm_features): the plain start (cx0/W, cy0/H, r0/rmax), the
// distances to the 4 nearest other centres, to the 4 walls and a
// neighbour-repulsion vector, all in units of the mean spacing
// s = sqrt(W H / N), counts of neighbours within s and 2 s, N / 400, W / H.
// Network (weights BF16, activations and accumulation FP32):
//     h1 = relu(W1 f + b1)                       32 -> 128
//     g  = mean over the instance's circles of h1
//     h2 = relu(W2 [h1; g] + b2)                 256 -> 128
//     o  = W3 h2 + b3                            128 -> 3 (padded to 4)
// Output: cx = cx0 + s o0, cy = cy0 + s o1, r = s max(o2, 0).
// Training: mean squared error against converged packings produced by the
// plain solver, Adam on FP32 master weights, BF16 copies for the GEMMs.
// Every kernel here is this file's own (tensor-core GEMM with TF32 inputs,
// BF16 weights and FP32 accumulation, segment mean/sum, fused epilogues,
// Adam).
#include <cuda_bf16.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "engine_internal.h"
#include "paradmm_gpu.h"

#define SM_F 32     // padded feature width
#define SM_H 128    // hidden width
#define SM_O 4      // outputs (3 used)
#define SM_NF 21    // features actually used

// parameter layout (FP32 master copy)
#define SM_W1 0
#define SM_B1 (SM_W1 + SM_H * SM_F)
#define SM_W2 (SM_B1 + SM_H)
#define SM_B2 (SM_W2 + SM_H * 2 * SM_H)
#define SM_W3 (SM_B2 + SM_H)
#define SM_B3 (SM_W3 + SM_O * SM_H)
#define SM_NPARAM (SM_B3 + SM_O)

// ---------------------------------------------------------------------------
// Features and targets
// ---------------------------------------------------------------------------
struct SmInst {  // one instance of a data set (device)
    int N, row0;      // circles, first row in the row arrays
    float W, H;       // box
};

__global__ void sm_features(const SmInst *inst, int n_inst, const double *init, float rmax, float *F)
{
    // one block per instance, threads over its circles
    for (int b = blockIdx.x; b < n_inst; b += gridDim.x) {
        const SmInst I = inst[b];
        const float s = sqrtf(I.W * I.H / (float)I.N);
        for (int i = threadIdx.x; i < I.N; i += blockDim.x) {
            const double *ci = init + 3LL * (I.row0 + i);
            const float x = (float)ci[0], y = (float)ci[1], r = (float)ci[2];
            float d[4] = {1e30f, 1e30f, 1e30f, 1e30f};
            float rx = 0.f, ry = 0.f, n1 = 0.f, n2 = 0.f;
            for (int j = 0; j < I.N; ++j) {
                if (j == i) continue;
                const double *cj = init + 3LL * (I.row0 + j);
                const float dx = x - (float)cj[0], dy = y - (float)cj[1];
                const float dd = sqrtf(dx * dx + dy * dy) + 1e-9f;
                if (dd < d[3]) {
                    d[3] = dd;
                    for (int q = 3; q > 0 && d[q] < d[q - 1]; --q) { const float t = d[q]; d[q] = d[q - 1]; d[q - 1] = t; }
                }
                if (dd < 3.f * s) { const float w = s * s / (dd * dd); rx += dx / dd * w; ry += dy / dd * w; }
                if (dd < s) n1 += 1.f;
                if (dd < 2.f * s) n2 += 1.f;
            }
            float f[SM_F];
            for (int q = 0; q < SM_F; ++q) f[q] = 0.f;
            f[0] = x / I.W; f[1] = y / I.H; f[2] = r / rmax;
            for (int q = 0; q < 4; ++q) f[3 + q] = fminf(d[q] / s, 4.f);
            f[7] = fminf(x / s, 4.f); f[8] = fminf((I.W - x) / s, 4.f);
            f[9] = fminf(y / s, 4.f); f[10] = fminf((I.H - y) / s, 4.f);
            f[11] = fmaxf(fminf(rx * 0.25f, 4.f), -4.f); f[12] = fmaxf(fminf(ry * 0.25f, 4.f), -4.f);
            f[13] = n1 * 0.25f; f[14] = n2 * 0.1f;
            f[15] = (float)I.N / 400.f; f[16] = I.W / I.H;
            f[17] = r / s; f[18] = d[0] / s - r / s; f[19] = 1.f; f[20] = sqrtf((float)I.N) / 20.f;
            float *o = F + (long long)(I.row0 + i) * SM_F;
            for (int q = 0; q < SM_F; ++q) o[q] = f[q];
        }
    }
}

__global__ void sm_targets(const SmInst *inst, int n_inst, const double *init, const double *target, float *T)
{
    for (int b = blockIdx.x; b < n_inst; b += gridDim.x) {
        const SmInst I = inst[b];
        const float s = sqrtf(I.W * I.H / (float)I.N);
        for (int i = threadIdx.x; i < I.N; i += blockDim.x) {
            const long long m = I.row0 + i;
            float *o = T + m * SM_O;
            o[0] = (float)((target[3 * m] - init[3 * m]) / s);
            o[1] = (float)((target[3 * m + 1] - init[3 * m + 1]) / s);
            o[2] = (float)(target[3 * m + 2] / s);
            o[3] = 0.f;
        }
    }
}

// ---------------------------------------------------------------------------
// GEMM on the tensor cores: C[M x N] = op(A) op(B) (+ C) with FP32
// accumulation (mma.sync m16n8k8, TF32 inputs).  A is FP32 [M][K] (or [K][M]
// when TA), B is T [K][N] (or [N][K] when TB), T = float or bf16.  FP32
// operands are split into two TF32 numbers (hi + lo) and the product is
// taken as the sum of the two or three significant partial products, so the
// result has FP32 accuracy; BF16 weights are exact in TF32.
// 64 x 64 block tiles, K in chunks of 16, 4 warps of 32 x 32 (2 x 4 mma
// tiles each).  split > 1 splits K over blockIdx.z: every split writes its
// partial tile to its own slice of the workspace and sm_gemm_reduce adds the
// slices in order, so the result does not depend on timing.
// ---------------------------------------------------------------------------
template <typename TB>
PDM_D float ld_b(const TB *p);
template <>
PDM_D float ld_b<float>(const float *p) { return *p; }
template <>
PDM_D float ld_b<__nv_bfloat16>(const __nv_bfloat16 *p) { return __bfloat162float(*p); }

PDM_D unsigned to_tf32(float x)
{
    unsigned r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return r;
}

PDM_D void split_tf32(float x, unsigned &hi, unsigned &lo)
{
    hi = to_tf32(x);
    lo = to_tf32(x - __uint_as_float(hi));
}

PDM_D void mma_tf32(float (&d)[4], const unsigned (&a)[4], const unsigned (&b)[2])
{
    asm volatile("mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0, %1, %2, %3}, {%4, %5, %6, %7}, {%8, %9}, "
                 "{%0, %1, %2, %3};"
                 : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
                 : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

#define SM_KC 16       // K chunk
#define SM_LD (SM_KC + 4)  // padded row of the staged tiles (conflict-free fragment loads)

template <bool TA, bool TB, typename BT>
__global__ void __launch_bounds__(128) sm_gemm_tc(int M, int N, int K, const float *A, int lda, const BT *B, int ldb,
                                                  float *C, int ldc, int accumulate, int split, float *ws)
{
    __shared__ float As[64][SM_LD];  // [m][k]
    __shared__ float Bs[64][SM_LD];  // [n][k]
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    const int gid = lane >> 2, tig = lane & 3;
    const int wm = (w >> 1) * 32, wn = (w & 1) * 32;
    const int m0 = blockIdx.y * 64, n0 = blockIdx.x * 64;
    constexpr bool B_EXACT_TF32 = sizeof(BT) == 2;  // BF16 has 8 significand bits, TF32 11
    const int kper = (K + split - 1) / split;
    const int kbeg = blockIdx.z * kper, kend = min(K, kbeg + kper);
    float acc[2][4][4] = {};
    for (int k0 = kbeg; k0 < kend; k0 += SM_KC) {
        for (int e = tid; e < 64 * SM_KC; e += 128) {
            int mm, kk;
            if (TA) { kk = e / 64; mm = e % 64; } else { mm = e / SM_KC; kk = e % SM_KC; }  // coalesced along memory
            const int gm = m0 + mm, gk = k0 + kk;
            As[mm][kk] = (gm < M && gk < kend) ? (TA ? A[(long long)gk * lda + gm] : A[(long long)gm * lda + gk]) : 0.f;
        }
        for (int e = tid; e < 64 * SM_KC; e += 128) {
            int nn, kk;
            if (TB) { nn = e / SM_KC; kk = e % SM_KC; } else { kk = e / 64; nn = e % 64; }
            const int gn = n0 + nn, gk = k0 + kk;
            Bs[nn][kk] = (gn < N && gk < kend) ? (TB ? ld_b<BT>(B + (long long)gn * ldb + gk) : ld_b<BT>(B + (long long)gk * ldb + gn))
                                               : 0.f;
        }
        __syncthreads();
#pragma unroll
        for (int ks = 0; ks < SM_KC; ks += 8) {
            // each operand as a sum of two TF32 numbers, hi + lo, so that the
            // products keep FP32 accuracy: a_hi b + a_lo b when B is BF16 (exact
            // in TF32), a_hi b_hi + a_hi b_lo + a_lo b_hi when B is FP32
            unsigned ah[2][4], al[2][4], bh[4][2], bl[4][2];
#pragma unroll
            for (int i = 0; i < 2; ++i) {
                const int r = wm + i * 16 + gid;
                split_tf32(As[r][ks + tig], ah[i][0], al[i][0]);
                split_tf32(As[r + 8][ks + tig], ah[i][1], al[i][1]);
                split_tf32(As[r][ks + tig + 4], ah[i][2], al[i][2]);
                split_tf32(As[r + 8][ks + tig + 4], ah[i][3], al[i][3]);
            }
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const int c = wn + j * 8 + gid;
                split_tf32(Bs[c][ks + tig], bh[j][0], bl[j][0]);
                split_tf32(Bs[c][ks + tig + 4], bh[j][1], bl[j][1]);
            }
#pragma unroll
            for (int i = 0; i < 2; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    mma_tf32(acc[i][j], al[i], bh[j]);
                    if (!B_EXACT_TF32) mma_tf32(acc[i][j], ah[i], bl[j]);
                    mma_tf32(acc[i][j], ah[i], bh[j]);
                }
        }
        __syncthreads();
    }
    // epilogue: element (r, c) of mma tile (i, j) is acc[i][j][q] with
    // r = gid (+ 8 for q >= 2), c = 2 tig + (q & 1)
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const int gm = m0 + wm + i * 16 + gid + (q >= 2 ? 8 : 0);
                const int gn = n0 + wn + j * 8 + 2 * tig + (q & 1);
                if (gm >= M || gn >= N) continue;
                if (split > 1) ws[((long long)blockIdx.z * M + gm) * N + gn] = acc[i][j][q];
                else {
                    float *c = C + (long long)gm * ldc + gn;
                    *c = accumulate ? *c + acc[i][j][q] : acc[i][j][q];
                }
            }
}

// C[M x N] (+)= sum over the split slices of the workspace, in slice order.
__global__ void sm_gemm_reduce(int M, int N, int split, const float *ws, float *C, int ldc, int accumulate)
{
    const long long n = (long long)M * N;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
        float s = 0.f;
        for (int z = 0; z < split; ++z) s += ws[z * n + e];
        float *c = C + (e / N) * ldc + e % N;
        *c = accumulate ? *c + s : s;
    }
}

#define SM_WS_FLOATS (64LL * SM_H * SM_H)  // split-K workspace: up to 64 slices of a 128 x 128 product

template <bool TA, bool TB, typename BT>
static void gemm(cudaStream_t s, int M, int N, int K, const float *A, int lda, const BT *B, int ldb, float *C, int ldc,
                 bool accumulate, int split = 1, float *ws = nullptr)
{
    if (split > 1 && (!ws || (long long)split * M * N > SM_WS_FLOATS)) split = 1;
    dim3 grid((N + 63) / 64, (M + 63) / 64, split);
    sm_gemm_tc<TA, TB, BT><<<grid, 128, 0, s>>>(M, N, K, A, lda, B, ldb, C, ldc, accumulate ? 1 : 0, split, ws);
    if (split > 1) sm_gemm_reduce<<<64, 256, 0, s>>>(M, N, split, ws, C, ldc, accumulate ? 1 : 0);
}

// ---------------------------------------------------------------------------
// Elementwise / segment kernels
// ---------------------------------------------------------------------------
// Y = relu(Y + bias[col] + P[inst(row) - inst_base][col])  (P may be null).
// Y and P are batch-local; row_inst gives each batch row's data-set instance.
__global__ void sm_bias_relu(float *Y, int M, int N, const float *bias, const float *P, const int *row_inst,
                             int inst_base, int relu)
{
    const long long n = (long long)M * N;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
        const int m = (int)(e / N), c = (int)(e % N);
        float v = Y[e] + bias[c];
        if (P) v += P[(long long)(row_inst[m] - inst_base) * N + c];
        Y[e] = relu ? fmaxf(v, 0.f) : v;
    }
}

// G[b][c] = mean (or sum) over the rows of batch instance b of H[row][c];
// row0 are data-set rows, H starts at data-set row row_base.
__global__ void sm_seg_mean(const float *H, int N, const int *row0, const int *nrows, int n_inst, float *G, int scale_mean,
                            int row_base)
{
    for (int b = blockIdx.x; b < n_inst; b += gridDim.x) {
        const int r0 = row0[b] - row_base, nr = nrows[b];
        for (int c = threadIdx.x; c < N; c += blockDim.x) {
            float s = 0.f;
            for (int r = 0; r < nr; ++r) s += H[(long long)(r0 + r) * N + c];
            G[(long long)b * N + c] = scale_mean ? s / (float)nr : s;
        }
    }
}

// dO = 2 (O - T) / count on the first 3 columns; loss partial sums
__global__ void sm_mse(const float *O, const float *T, int M, float inv_count, float *dO, double *loss)
{
    double l = 0.0;
    for (int m = blockIdx.x * blockDim.x + threadIdx.x; m < M; m += gridDim.x * blockDim.x) {
#pragma unroll
        for (int c = 0; c < SM_O; ++c) {
            const float e = c < 3 ? O[m * SM_O + c] - T[m * SM_O + c] : 0.f;
            dO[m * SM_O + c] = 2.f * e * inv_count;
            l += (double)e * e;
        }
    }
    l = block_sum(l);
    if (threadIdx.x == 0) atomicAdd(loss, l);
}

// dH[m][c] = (dH[m][c] + (dG ? dG[inst - inst_base][c] / rows_of(inst) : 0)) * (H[m][c] > 0)
__global__ void sm_relu_back(float *dH, const float *H, int M, int N, const float *dG, const int *row_inst,
                             const int *nrows, int inst_base)
{
    const long long n = (long long)M * N;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
        const int m = (int)(e / N), c = (int)(e % N);
        float v = dH[e];
        if (dG) { const int b = row_inst[m]; v += dG[(long long)(b - inst_base) * N + c] / (float)nrows[b]; }
        dH[e] = H[e] > 0.f ? v : 0.f;
    }
}

// column sums of X[M][N] accumulated into out[N]
__global__ void sm_colsum(const float *X, int M, int N, float *out)
{
    for (int c = blockIdx.x; c < N; c += gridDim.x) {
        float s = 0.f;
        for (int m = threadIdx.x; m < M; m += blockDim.x) s += X[(long long)m * N + c];
        s = (float)block_sum((double)s);
        if (threadIdx.x == 0) out[c] += s;
    }
}

__global__ void sm_adam(float *p, const float *g, float *m1, float *m2, int n, float lr, float b1, float b2, float eps,
                        float c1, float c2, float wd)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float gi = g[i] + wd * p[i];
        m1[i] = b1 * m1[i] + (1.f - b1) * gi;
        m2[i] = b2 * m2[i] + (1.f - b2) * gi * gi;
        p[i] -= lr * (m1[i] / c1) / (sqrtf(m2[i] / c2) + eps);
    }
}

__global__ void sm_to_bf16(const float *p, __nv_bfloat16 *q, int n)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) q[i] = __float2bfloat16(p[i]);
}

// ---------------------------------------------------------------------------
// Network object
// ---------------------------------------------------------------------------
struct paradmm_setmlp {
    int device = 0;
    cudaStream_t stream = nullptr;
    float *p = nullptr, *g = nullptr, *m1 = nullptr, *m2 = nullptr;  // FP32 master, grads, Adam moments
    __nv_bfloat16 *pb = nullptr;                                      // BF16 copy of the parameters
    long long adam_t = 0;
    // data set
    int n_inst = 0;
    long long n_rows = 0;
    SmInst *d_inst = nullptr;
    int *d_row_inst = nullptr, *d_row0 = nullptr, *d_nrows = nullptr;
    float *F = nullptr, *T = nullptr;
    std::vector<int> h_row0, h_nrows;
    std::vector<SmInst> h_inst;
    // activations (capacity rows)
    long long cap = 0;
    int cap_inst = 0;
    float *H1 = nullptr, *H2 = nullptr, *O = nullptr, *dO = nullptr, *dH1 = nullptr, *dH2 = nullptr;
    float *G = nullptr, *P = nullptr, *dP = nullptr, *dG = nullptr;
    double *d_loss = nullptr;
    float *ws = nullptr;             // split-K workspace of the weight-gradient GEMMs
    std::vector<void *> allocs;
};

static int sm_alloc(paradmm_setmlp *n, void **p, size_t bytes)
{
    cudaError_t e = cudaMalloc(p, bytes ? bytes : 16);
    if (e != cudaSuccess) return pdm_cuda_fail(e, "cudaMalloc (set MLP)", __FILE__, __LINE__);
    n->allocs.push_back(*p);
    return PARADMM_OK;
}

static int sm_reserve(paradmm_setmlp *n, long long rows, int insts)
{
    if (rows <= n->cap && insts <= n->cap_inst) return PARADMM_OK;
    for (float **b : {&n->H1, &n->H2, &n->O, &n->dO, &n->dH1, &n->dH2, &n->G, &n->P, &n->dP, &n->dG}) {
        if (*b) {
            cudaFree(*b);
            n->allocs.erase(std::find(n->allocs.begin(), n->allocs.end(), (void *)*b));
            *b = nullptr;
        }
    }
    n->cap = std::max(rows, n->cap);
    n->cap_inst = std::max(insts, n->cap_inst);
    int rc;
    if ((rc = sm_alloc(n, (void **)&n->H1, sizeof(float) * n->cap * SM_H)) ||
        (rc = sm_alloc(n, (void **)&n->H2, sizeof(float) * n->cap * SM_H)) ||
        (rc = sm_alloc(n, (void **)&n->dH1, sizeof(float) * n->cap * SM_H)) ||
        (rc = sm_alloc(n, (void **)&n->dH2, sizeof(float) * n->cap * SM_H)) ||
        (rc = sm_alloc(n, (void **)&n->O, sizeof(float) * n->cap * SM_O)) ||
        (rc = sm_alloc(n, (void **)&n->dO, sizeof(float) * n->cap * SM_O)) ||
        (rc = sm_alloc(n, (void **)&n->G, sizeof(float) * n->cap_inst * SM_H)) ||
        (rc = sm_alloc(n, (void **)&n->P, sizeof(float) * n->cap_inst * SM_H)) ||
        (rc = sm_alloc(n, (void **)&n->dP, sizeof(float) * n->cap_inst * SM_H)) ||
        (rc = sm_alloc(n, (void **)&n->dG, sizeof(float) * n->cap_inst * SM_H)))
        return rc;
    return PARADMM_OK;
}

// Forward over rows [r0, r0 + rows) = instances [b0, b0 + nb) of the data set.
static void sm_forward(paradmm_setmlp *n, long long r0, long long rows, int b0, int nb)
{
    cudaStream_t s = n->stream;
    const __nv_bfloat16 *W1 = n->pb + SM_W1, *W2 = n->pb + SM_W2, *W3 = n->pb + SM_W3;
    const float *F = n->F + r0 * SM_F;
    const int M = (int)rows;
    const int blocks = 148 * 4;
    gemm<false, true>(s, M, SM_H, SM_F, F, SM_F, W1, SM_F, n->H1, SM_H, false);
    sm_bias_relu<<<blocks, 256, 0, s>>>(n->H1, M, SM_H, n->p + SM_B1, nullptr, nullptr, 0, 1);
    sm_seg_mean<<<std::min(nb, 1024), 128, 0, s>>>(n->H1, SM_H, n->d_row0 + b0, n->d_nrows + b0, nb, n->G, 1, (int)r0);
    gemm<false, true>(s, nb, SM_H, SM_H, n->G, SM_H, W2 + SM_H, 2 * SM_H, n->P, SM_H, false);
    gemm<false, true>(s, M, SM_H, SM_H, n->H1, SM_H, W2, 2 * SM_H, n->H2, SM_H, false);
    sm_bias_relu<<<blocks, 256, 0, s>>>(n->H2, M, SM_H, n->p + SM_B2, n->P, n->d_row_inst + r0, b0, 1);
    gemm<false, true>(s, M, SM_O, SM_H, n->H2, SM_H, W3, SM_H, n->O, SM_O, false);
    sm_bias_relu<<<blocks, 256, 0, s>>>(n->O, M, SM_O, n->p + SM_B3, nullptr, nullptr, 0, 0);
}

// Backward of the MSE over the same rows; gradients accumulate into n->g.
static void sm_backward(paradmm_setmlp *n, long long r0, long long rows, int b0, int nb)
{
    cudaStream_t s = n->stream;
    const __nv_bfloat16 *W2 = n->pb + SM_W2, *W3 = n->pb + SM_W3;
    const float *F = n->F + r0 * SM_F;
    const int M = (int)rows;
    const int blocks = 148 * 4;
    const int split = std::max(1, std::min(64, M / 512));
    // layer 3
    gemm<true, false>(s, SM_O, SM_H, M, n->dO, SM_O, n->H2, SM_H, n->g + SM_W3, SM_H, true, split, n->ws);
    sm_colsum<<<SM_O, 256, 0, s>>>(n->dO, M, SM_O, n->g + SM_B3);
    gemm<false, false>(s, M, SM_H, SM_O, n->dO, SM_O, W3, SM_H, n->dH2, SM_H, false);
    sm_relu_back<<<blocks, 256, 0, s>>>(n->dH2, n->H2, M, SM_H, nullptr, nullptr, nullptr, 0);
    // layer 2
    gemm<true, false>(s, SM_H, SM_H, M, n->dH2, SM_H, n->H1, SM_H, n->g + SM_W2, 2 * SM_H, true, split, n->ws);
    sm_colsum<<<SM_H, 256, 0, s>>>(n->dH2, M, SM_H, n->g + SM_B2);
    // dP = per-instance sums of dH2; dW2b += dP^T G; dG = dP W2b
    sm_seg_mean<<<std::min(nb, 1024), 128, 0, s>>>(n->dH2, SM_H, n->d_row0 + b0, n->d_nrows + b0, nb, n->dP, 0, (int)r0);
    gemm<true, false>(s, SM_H, SM_H, nb, n->dP, SM_H, n->G, SM_H, n->g + SM_W2 + SM_H, 2 * SM_H, true, 1);
    gemm<false, false>(s, nb, SM_H, SM_H, n->dP, SM_H, W2 + SM_H, 2 * SM_H, n->dG, SM_H, false);
    gemm<false, false>(s, M, SM_H, SM_H, n->dH2, SM_H, W2, 2 * SM_H, n->dH1, SM_H, false);
    sm_relu_back<<<blocks, 256, 0, s>>>(n->dH1, n->H1, M, SM_H, n->dG, n->d_row_inst + r0, n->d_nrows, b0);
    // layer 1
    gemm<true, false>(s, SM_H, SM_F, M, n->dH1, SM_H, F, SM_F, n->g + SM_W1, SM_F, true, split, n->ws);
    sm_colsum<<<SM_H, 256, 0, s>>>(n->dH1, M, SM_H, n->g + SM_B1);
}

// ---------------------------------------------------------------------------
// C-ABI
// ---------------------------------------------------------------------------
extern "C" int64_t paradmm_setmlp_num_params(void) { return SM_NPARAM; }
extern "C" void paradmm_setmlp_destroy(paradmm_setmlp *n);

extern "C" int paradmm_setmlp_create(int device, uint64_t seed, paradmm_setmlp **out)
{
    pdm_clear_status();
    if (!out) return pdm_set_error(PARADMM_EINVAL, "out is NULL");
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) {
        cudaGetLastError();
        return pdm_set_error(PARADMM_ENODEVICE, "no CUDA device %d", device);
    }
    PDM_CUDA(cudaSetDevice(device));
    paradmm_setmlp *n = new paradmm_setmlp();
    n->device = device;
    int rc = PARADMM_OK;
    if (cudaStreamCreateWithFlags(&n->stream, cudaStreamNonBlocking) != cudaSuccess) rc = pdm_set_error(PARADMM_ECUDA, "stream");
    if (!rc) rc = sm_alloc(n, (void **)&n->p, sizeof(float) * SM_NPARAM);
    if (!rc) rc = sm_alloc(n, (void **)&n->g, sizeof(float) * SM_NPARAM);
    if (!rc) rc = sm_alloc(n, (void **)&n->m1, sizeof(float) * SM_NPARAM);
    if (!rc) rc = sm_alloc(n, (void **)&n->m2, sizeof(float) * SM_NPARAM);
    if (!rc) rc = sm_alloc(n, (void **)&n->pb, sizeof(__nv_bfloat16) * SM_NPARAM);
    if (!rc) rc = sm_alloc(n, (void **)&n->d_loss, sizeof(double));
    if (!rc) rc = sm_alloc(n, (void **)&n->ws, sizeof(float) * SM_WS_FLOATS);
    if (rc) { paradmm_setmlp_destroy(n); return rc; }
    // He-style init from a splitmix64 stream (host), zero biases
    std::vector<float> h(SM_NPARAM, 0.f);
    uint64_t st = seed ^ 0x5eed5eed12345678ULL;
    auto u01 = [&]() {
        uint64_t z = (st += 0x9E3779B97F4A7C15ULL);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
        z ^= z >> 31;
        return (double)(z >> 11) * (1.0 / 9007199254740992.0);
    };
    auto fill = [&](int off, int cnt, int fan_in) {
        const double a = std::sqrt(6.0 / fan_in);
        for (int i = 0; i < cnt; ++i) h[off + i] = (float)((2.0 * u01() - 1.0) * a);
    };
    fill(SM_W1, SM_H * SM_F, SM_NF);
    fill(SM_W2, SM_H * 2 * SM_H, 2 * SM_H);
    fill(SM_W3, SM_O * SM_H, SM_H);
    for (int i = 0; i < SM_O * SM_H; ++i) h[SM_W3 + i] *= 0.1f;
    PDM_CUDA(cudaMemcpy(n->p, h.data(), sizeof(float) * SM_NPARAM, cudaMemcpyHostToDevice));
    PDM_CUDA(cudaMemset(n->m1, 0, sizeof(float) * SM_NPARAM));
    PDM_CUDA(cudaMemset(n->m2, 0, sizeof(float) * SM_NPARAM));
    sm_to_bf16<<<64, 256, 0, n->stream>>>(n->p, n->pb, SM_NPARAM);
    PDM_CUDA(cudaStreamSynchronize(n->stream));
    *out = n;
    return PARADMM_OK;
}

extern "C" void paradmm_setmlp_destroy(paradmm_setmlp *n)
{
    if (!n) return;
    int prev = -1;
    cudaGetDevice(&prev);
    cudaSetDevice(n->device);
    for (void *p : n->allocs) cudaFree(p);
    if (n->stream) cudaStreamDestroy(n->stream);
    if (prev >= 0) cudaSetDevice(prev);
    delete n;
}

extern "C" int paradmm_setmlp_get_params(paradmm_setmlp *n, float *out)
{
    pdm_clear_status();
    if (!n || !out) return pdm_set_error(PARADMM_EINVAL, "NULL argument");
    PDM_CUDA(cudaSetDevice(n->device));
    PDM_CUDA(cudaMemcpy(out, n->p, sizeof(float) * SM_NPARAM, cudaMemcpyDeviceToHost));
    return PARADMM_OK;
}

extern "C" int paradmm_setmlp_set_params(paradmm_setmlp *n, const float *in)
{
    pdm_clear_status();
    if (!n || !in) return pdm_set_error(PARADMM_EINVAL, "NULL argument");
    PDM_CUDA(cudaSetDevice(n->device));
    PDM_CUDA(cudaMemcpy(n->p, in, sizeof(float) * SM_NPARAM, cudaMemcpyHostToDevice));
    sm_to_bf16<<<64, 256, 0, n->stream>>>(n->p, n->pb, SM_NPARAM);
    PDM_CUDA(cudaStreamSynchronize(n->stream));
    return PARADMM_OK;
}

// Data set: n_inst instances, n_circles[b], box[2b..2b+1] = (W, H), init and
// (optional) target circles [cx, cy, r] per circle, instance-major.
extern "C" int paradmm_setmlp_set_data(paradmm_setmlp *n, int n_inst, const int *n_circles, const double *box,
                                       const double *init, const double *target, double rmax)
{
    pdm_clear_status();
    if (!n || n_inst < 1 || !n_circles || !box || !init) return pdm_set_error(PARADMM_EINVAL, "bad data set");
    PDM_CUDA(cudaSetDevice(n->device));
    std::vector<SmInst> inst(n_inst);
    std::vector<int> row_inst;
    n->h_row0.assign(n_inst, 0);
    n->h_nrows.assign(n_inst, 0);
    long long rows = 0;
    for (int b = 0; b < n_inst; ++b) {
        if (n_circles[b] < 2) return pdm_set_error(PARADMM_EINVAL, "instance %d has fewer than 2 circles", b);
        inst[b].N = n_circles[b];
        inst[b].row0 = (int)rows;
        inst[b].W = (float)box[2 * b];
        inst[b].H = (float)box[2 * b + 1];
        n->h_row0[b] = (int)rows;
        n->h_nrows[b] = n_circles[b];
        for (int i = 0; i < n_circles[b]; ++i) row_inst.push_back(b);
        rows += n_circles[b];
    }
    // drop the previous data set
    for (void **b : {(void **)&n->d_inst, (void **)&n->d_row_inst, (void **)&n->d_row0, (void **)&n->d_nrows,
                     (void **)&n->F, (void **)&n->T}) {
        if (*b) {
            cudaFree(*b);
            n->allocs.erase(std::find(n->allocs.begin(), n->allocs.end(), *b));
            *b = nullptr;
        }
    }
    n->n_inst = n_inst;
    n->n_rows = rows;
    n->h_inst = inst;
    int rc;
    if ((rc = sm_alloc(n, (void **)&n->d_inst, sizeof(SmInst) * n_inst)) ||
        (rc = sm_alloc(n, (void **)&n->d_row_inst, sizeof(int) * rows)) ||
        (rc = sm_alloc(n, (void **)&n->d_row0, sizeof(int) * n_inst)) ||
        (rc = sm_alloc(n, (void **)&n->d_nrows, sizeof(int) * n_inst)) ||
        (rc = sm_alloc(n, (void **)&n->F, sizeof(float) * rows * SM_F)) ||
        (rc = sm_alloc(n, (void **)&n->T, sizeof(float) * rows * SM_O)))
        return rc;
    double *d_init = nullptr, *d_target = nullptr;
    PDM_CUDA(cudaMalloc(&d_init, sizeof(double) * 3 * rows));
    cudaMemcpy(d_init, init, sizeof(double) * 3 * rows, cudaMemcpyHostToDevice);
    if (target) {
        cudaMalloc(&d_target, sizeof(double) * 3 * rows);
        cudaMemcpy(d_target, target, sizeof(double) * 3 * rows, cudaMemcpyHostToDevice);
    }
    cudaMemcpy(n->d_inst, inst.data(), sizeof(SmInst) * n_inst, cudaMemcpyHostToDevice);
    cudaMemcpy(n->d_row_inst, row_inst.data(), sizeof(int) * rows, cudaMemcpyHostToDevice);
    cudaMemcpy(n->d_row0, n->h_row0.data(), sizeof(int) * n_inst, cudaMemcpyHostToDevice);
    cudaMemcpy(n->d_nrows, n->h_nrows.data(), sizeof(int) * n_inst, cudaMemcpyHostToDevice);
    sm_features<<<std::min(n_inst, 4096), 256, 0, n->stream>>>(n->d_inst, n_inst, d_init, (float)rmax, n->F);
    if (target) sm_targets<<<std::min(n_inst, 4096), 256, 0, n->stream>>>(n->d_inst, n_inst, d_init, d_target, n->T);
    else cudaMemsetAsync(n->T, 0, sizeof(float) * rows * SM_O, n->stream);
    cudaError_t e = cudaStreamSynchronize(n->stream);
    cudaFree(d_init);
    if (d_target) cudaFree(d_target);
    if (e != cudaSuccess) return pdm_cuda_fail(e, "set MLP data", __FILE__, __LINE__);
    return PARADMM_OK;
}

// One pass over instances [b0, b0 + nb): loss (and, when train, gradients
// and one Adam step).  Returns the mean squared error per output.
static int sm_step(paradmm_setmlp *n, int b0, int nb, bool train, float lr, double *loss)
{
    const long long r0 = n->h_row0[b0];
    const long long rows = (long long)n->h_row0[b0 + nb - 1] + n->h_nrows[b0 + nb - 1] - r0;
    int rc = sm_reserve(n, rows, nb);
    if (rc) return rc;
    cudaStream_t s = n->stream;
    sm_forward(n, r0, rows, b0, nb);
    PDM_CUDA(cudaMemsetAsync(n->d_loss, 0, sizeof(double), s));
    sm_mse<<<148 * 2, 256, 0, s>>>(n->O, n->T + r0 * SM_O, (int)rows, 1.f / (3.f * (float)rows), n->dO, n->d_loss);
    if (train) {
        PDM_CUDA(cudaMemsetAsync(n->g, 0, sizeof(float) * SM_NPARAM, s));
        sm_backward(n, r0, rows, b0, nb);
        n->adam_t++;
        const float b1 = 0.9f, b2 = 0.999f;
        sm_adam<<<64, 256, 0, s>>>(n->p, n->g, n->m1, n->m2, SM_NPARAM, lr, b1, b2, 1e-8f,
                                    1.f - powf(b1, (float)n->adam_t), 1.f - powf(b2, (float)n->adam_t), 0.f);
        sm_to_bf16<<<64, 256, 0, s>>>(n->p, n->pb, SM_NPARAM);
    }
    double l = 0;
    PDM_CUDA(cudaMemcpyAsync(&l, n->d_loss, sizeof(double), cudaMemcpyDeviceToHost, s));
    PDM_CUDA(cudaStreamSynchronize(s));
    if (loss) *loss = l / (3.0 * (double)rows);
    return PARADMM_OK;
}

// Gradients of the MSE over instances [b0, b0 + nb) (no update): into grads.
extern "C" int paradmm_setmlp_gradients(paradmm_setmlp *n, int b0, int nb, float *grads, double *loss)
{
    pdm_clear_status();
    if (!n || !grads || b0 < 0 || nb < 1 || b0 + nb > n->n_inst) return pdm_set_error(PARADMM_EINVAL, "bad range");
    PDM_CUDA(cudaSetDevice(n->device));
    const long long r0 = n->h_row0[b0];
    const long long rows = (long long)n->h_row0[b0 + nb - 1] + n->h_nrows[b0 + nb - 1] - r0;
    int rc = sm_reserve(n, rows, nb);
    if (rc) return rc;
    cudaStream_t s = n->stream;
    sm_forward(n, r0, rows, b0, nb);
    PDM_CUDA(cudaMemsetAsync(n->d_loss, 0, sizeof(double), s));
    sm_mse<<<148 * 2, 256, 0, s>>>(n->O, n->T + r0 * SM_O, (int)rows, 1.f / (3.f * (float)rows), n->dO, n->d_loss);
    PDM_CUDA(cudaMemsetAsync(n->g, 0, sizeof(float) * SM_NPARAM, s));
    sm_backward(n, r0, rows, b0, nb);
    double l = 0;
    PDM_CUDA(cudaMemcpyAsync(&l, n->d_loss, sizeof(double), cudaMemcpyDeviceToHost, s));
    PDM_CUDA(cudaMemcpyAsync(grads, n->g, sizeof(float) * SM_NPARAM, cudaMemcpyDeviceToHost, s));
    PDM_CUDA(cudaStreamSynchronize(s));
    if (loss) *loss = l / (3.0 * (double)rows);
    return PARADMM_OK;
}

// Features of the current data set (rows x 32 floats) -- for checks.
extern "C" int paradmm_setmlp_features(paradmm_setmlp *n, float *out)
{
    pdm_clear_status();
    if (!n || !out || !n->F) return pdm_set_error(PARADMM_EINVAL, "no data set");
    PDM_CUDA(cudaSetDevice(n->device));
    PDM_CUDA(cudaMemcpy(out, n->F, sizeof(float) * n->n_rows * SM_F, cudaMemcpyDeviceToHost));
    return PARADMM_OK;
}

// Trains for `epochs` passes over the data set in mini-batches of
// batch_inst instances (the instance order of the data set); losses gets
// one mean loss per epoch.  Learning rate decays linearly to lr_end.
extern "C" int paradmm_setmlp_train(paradmm_setmlp *n, int epochs, int batch_inst, float lr, float lr_end,
                                    double *losses)
{
    pdm_clear_status();
    if (!n || epochs < 1 || batch_inst < 1 || !n->F) return pdm_set_error(PARADMM_EINVAL, "bad training call");
    PDM_CUDA(cudaSetDevice(n->device));
    const int nbatch = (n->n_inst + batch_inst - 1) / batch_inst;
    const long long total = (long long)epochs * nbatch;
    long long step = 0;
    for (int ep = 0; ep < epochs; ++ep) {
        double sum = 0;
        long long cnt = 0;
        for (int bi = 0; bi < nbatch; ++bi, ++step) {
            const int b0 = bi * batch_inst, nb = std::min(batch_inst, n->n_inst - b0);
            const float a = (float)step / (float)std::max(1LL, total - 1);
            double l = 0;
            int rc = sm_step(n, b0, nb, true, lr + (lr_end - lr) * a, &l);
            if (rc) return rc;
            const long long rows = (long long)n->h_row0[b0 + nb - 1] + n->h_nrows[b0 + nb - 1] - n->h_row0[b0];
            sum += l * rows;
            cnt += rows;
        }
        if (losses) losses[ep] = sum / (double)cnt;
    }
    return PARADMM_OK;
}

extern "C" int paradmm_setmlp_eval(paradmm_setmlp *n, double *loss)
{
    pdm_clear_status();
    if (!n || !n->F) return pdm_set_error(PARADMM_EINVAL, "no data set");
    PDM_CUDA(cudaSetDevice(n->device));
    double sum = 0;
    long long cnt = 0;
    for (int b0 = 0; b0 < n->n_inst; b0 += 256) {
        const int nb = std::min(256, n->n_inst - b0);
        double l = 0;
        int rc = sm_step(n, b0, nb, false, 0.f, &l);
        if (rc) return rc;
        const long long rows = (long long)n->h_row0[b0 + nb - 1] + n->h_nrows[b0 + nb - 1] - n->h_row0[b0];
        sum += l * rows;
        cnt += rows;
    }
    if (loss) *loss = sum / (double)cnt;
    return PARADMM_OK;
}

// Proposal for the current data set: circles [cx, cy, r] per row (host out).
extern "C" int paradmm_setmlp_predict(paradmm_setmlp *n, const double *init, double *out)
{
    pdm_clear_status();
    if (!n || !init || !out || !n->F) return pdm_set_error(PARADMM_EINVAL, "no data set");
    PDM_CUDA(cudaSetDevice(n->device));
    std::vector<float> o;
    for (int b0 = 0; b0 < n->n_inst; b0 += 256) {
        const int nb = std::min(256, n->n_inst - b0);
        const long long r0 = n->h_row0[b0];
        const long long rows = (long long)n->h_row0[b0 + nb - 1] + n->h_nrows[b0 + nb - 1] - r0;
        int rc = sm_reserve(n, rows, nb);
        if (rc) return rc;
        sm_forward(n, r0, rows, b0, nb);
        if ((long long)o.size() < rows * SM_O) o.resize(rows * SM_O);
        PDM_CUDA(cudaMemcpyAsync(o.data(), n->O, sizeof(float) * rows * SM_O, cudaMemcpyDeviceToHost, n->stream));
        PDM_CUDA(cudaStreamSynchronize(n->stream));
        for (int b = b0; b < b0 + nb; ++b) {
            const SmInst &I = n->h_inst[b];
            const double sc = std::sqrt((double)I.W * I.H / I.N);
            for (int i = 0; i < I.N; ++i) {
                const long long m = I.row0 + i;
                const float *om = o.data() + (m - r0) * SM_O;
                out[3 * m] = init[3 * m] + sc * om[0];
                out[3 * m + 1] = init[3 * m + 1] + sc * om[1];
                out[3 * m + 2] = sc * std::max(0.0f, om[2]);
            }
        }
    }
    return PARADMM_OK;
}
