// Shared device/host helpers of the B200 parADMM engine.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "paradmm_gpu.h"

#define PDM_HD __host__ __device__ __forceinline__
#define PDM_D __device__ __forceinline__

// ----------------------------------------------------------------------------
// Device-side error codes (written to DevCtl::err, read by the host).
// ----------------------------------------------------------------------------
enum : int {
    DEV_OK = 0,
    DEV_BARRIER_TIMEOUT = 1,
    DEV_PEER_TIMEOUT = 2,  // a rank's flag for a sweep did not arrive (sharded instance)
};

static inline const char *pdm_dev_err_name(int e)
{
    return e == DEV_BARRIER_TIMEOUT ? "grid barrier" : e == DEV_PEER_TIMEOUT ? "exchange with another rank" : "unknown";
}

// Control block of one persistent launch: grid barrier, error flag, work
// counters.  Lives in device memory owned by the handle; zeroed before each
// launch.
struct DevCtl {
    unsigned int bar_count;   // grid-barrier arrivals in this launch
    unsigned int n_done;      // per-instance schedule: instances whose solve in this launch has ended
    int err;                  // DEV_* error, first writer wins
    int n_active;             // instances still iterating
    unsigned int item_ctr[2]; // dynamic work counters, one per iteration parity
    unsigned int pad[2];      // pad[0]: sweeps completed by the launch
    unsigned long long prof[4];  // optional: summed block time in pass, barrier 1, finalise, barrier 2 (ns)
    unsigned long long timeout_ns;  // barrier wait limit (0: PDM_BARRIER_TIMEOUT_NS)
};

// Barrier waits give up after this long; the kernel then records
// DEV_BARRIER_TIMEOUT and every block returns.  A full sweep of the largest
// supported problem is a few milliseconds, so a wait this long only ends a
// launch that can no longer make progress.
#define PDM_BARRIER_TIMEOUT_NS (4000ull * 1000ull * 1000ull)
#define PDM_BARRIER_MAX_POLLS (400ull * 1000ull * 1000ull)

PDM_D uint64_t globaltimer_ns()
{
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

PDM_D unsigned ld_acquire_u32(const unsigned *p)
{
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

PDM_D void st_release_u32(unsigned *p, unsigned v)
{
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

PDM_D unsigned atom_add_acq_rel_u32(unsigned *p, unsigned v)
{
    unsigned old;
    asm volatile("atom.acq_rel.gpu.global.add.u32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(v) : "memory");
    return old;
}

PDM_D int ld_volatile_i32(const int *p) { return *(const volatile int *)p; }

// Barrier of `nblocks` co-resident blocks that share `ctl` (the whole grid of
// a cooperative launch, or one rank's blocks of a launch that holds several
// ranks).  One counter
// that only grows within a launch (the host zeroes it): a block's arrival
// returns its position, which fixes the count that ends this round (the next
// multiple of the grid size), and the block waits until the counter reaches
// it.  One atomic per block and polling of one cache line: 1.45 us per
// barrier with 296 blocks on B200, against 3.5 us for a two-level tree with
// a generation flag.  Every wait is bounded by ctl->timeout_ns (default
// PDM_BARRIER_TIMEOUT_NS) and PDM_BARRIER_MAX_POLLS; on timeout, or when
// another block has already recorded an error, it returns false and the
// caller leaves its loop.  All threads of the block get the same answer.
PDM_D bool grid_barrier_n(DevCtl *ctl, unsigned nblocks)
{
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        const unsigned pos = atom_add_acq_rel_u32(&ctl->bar_count, 1u);
        const unsigned target = (pos / nblocks + 1u) * nblocks;
        int ok = 1;
        if ((int)(ld_acquire_u32(&ctl->bar_count) - target) < 0) {
            const uint64_t limit = ctl->timeout_ns ? ctl->timeout_ns : PDM_BARRIER_TIMEOUT_NS;
            const uint64_t t0 = globaltimer_ns();
            uint64_t polls = 0;
            while ((int)(ld_acquire_u32(&ctl->bar_count) - target) < 0) {
                if ((++polls & 63) == 0) {
                    if (ld_volatile_i32(&ctl->err) != DEV_OK) { ok = 0; break; }
                    if (polls > PDM_BARRIER_MAX_POLLS || globaltimer_ns() - t0 > limit) {
                        atomicCAS(&ctl->err, DEV_OK, DEV_BARRIER_TIMEOUT);
                        ok = 0;
                        break;
                    }
                }
            }
        }
        if (ld_volatile_i32(&ctl->err) != DEV_OK) ok = 0;
        s_ok = ok;
    }
    __syncthreads();
    const int ok = s_ok;
    __syncthreads();
    return ok != 0;
}

// The barrier over every block of the launch.
PDM_D bool grid_barrier(DevCtl *ctl) { return grid_barrier_n(ctl, gridDim.x * gridDim.y * gridDim.z); }

// System-scope flag accesses (flags another GPU writes or reads over NVLink).
PDM_D unsigned long long ld_acquire_sys_u64(const unsigned long long *p)
{
    unsigned long long v;
    asm volatile("ld.acquire.sys.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}

PDM_D void st_release_sys_u64(unsigned long long *p, unsigned long long v)
{
    asm volatile("st.release.sys.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

// Shared-memory address of a generic pointer into this CTA's shared memory.
PDM_D unsigned smem_u32(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }

// Loads/stores of data that other blocks of the same launch write: through
// L2 only (the per-SM L1 is not coherent within a launch).
PDM_D double4 ldcg_d4(const double4 *p)
{
    const double2 *q = reinterpret_cast<const double2 *>(p);
    double2 a = __ldcg(q), b = __ldcg(q + 1);
    return make_double4(a.x, a.y, b.x, b.y);
}
PDM_D void stcg_d4(double4 *p, double4 v)
{
    double2 *q = reinterpret_cast<double2 *>(p);
    __stcg(q, make_double2(v.x, v.y));
    __stcg(q + 1, make_double2(v.z, v.w));
}

PDM_D double warp_sum(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Block-wide sum (any blockDim multiple of 32, <= 1024); result valid in all
// threads.  Fixed reduction order, so the result is deterministic.
// Sums two values over the block (every thread gets both sums).
PDM_D double2 block_sum2(double a, double b)
{
    __shared__ double s_p[2][32];
    __shared__ double2 s_t;
    a = warp_sum(a);
    b = warp_sum(b);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    __syncthreads();
    if (l == 0) { s_p[0][w] = a; s_p[1][w] = b; }
    __syncthreads();
    if (w == 0) {
        const int nw = (blockDim.x + 31) >> 5;
        double x = l < nw ? s_p[0][l] : 0.0, y = l < nw ? s_p[1][l] : 0.0;
        x = warp_sum(x);
        y = warp_sum(y);
        if (l == 0) s_t = make_double2(x, y);
    }
    __syncthreads();
    return s_t;
}

PDM_D double block_sum(double v)
{
    __shared__ double s_part[32];
    __shared__ double s_total;
    v = warp_sum(v);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    __syncthreads();
    if (l == 0) s_part[w] = v;
    __syncthreads();
    if (w == 0) {
        const int nw = (blockDim.x + 31) >> 5;
        double t = l < nw ? s_part[l] : 0.0;
        t = warp_sum(t);
        if (l == 0) s_total = t;
    }
    __syncthreads();
    const double r = s_total;
    __syncthreads();
    return r;
}

// Host-side CUDA check used by the engine: records the error and returns.
int pdm_cuda_fail(cudaError_t e, const char *what, const char *file, int line);
#define PDM_CUDA(call)                                                                   \
    do {                                                                                 \
        cudaError_t e__ = (call);                                                        \
        if (e__ != cudaSuccess) return pdm_cuda_fail(e__, #call, __FILE__, __LINE__);    \
    } while (0)
