// Host-side launchers of the packing kernels (packing_kernels.cu).
#pragma once

#include <cuda_runtime.h>

#include "packing.cuh"

cudaError_t pk_launch_persistent(int V, bool stream_hint, const PkDev &D, const PkRun &R, int grid, cudaStream_t s);
cudaError_t pk_max_blocks_per_sm(int V, bool stream_hint, int *blocks);
cudaError_t pk_launch_instances(int V, bool stream_hint, const PkDev &D, const PkRun &R, const int *order, int n_coop,
                                int n_early, unsigned *queue, int grid, int cluster, cudaStream_t s);
cudaError_t pk_instances_max_clusters(int V, bool stream_hint, int cluster, int *clusters);
cudaError_t pk_instances_blocks_per_sm(int V, bool stream_hint, int *blocks);
cudaError_t pk_launch_init(int V, const PkDev &D, int inst, const PkInitArgs &A, int grid, cudaStream_t s);
cudaError_t pk_launch_scatter(int V, const PkDev &D, int inst, const int2 *pmap, long long npairs, const int *wmap,
                              int wall0, int nwall, const int *rmap, int rad0, int nrad, const int2 *cmap,
                              const double *Nd, const double *Ud, const double *Zd, int *flag, int grid, cudaStream_t s);
cudaError_t pk_launch_gather(int V, const PkDev &D, int inst, const int2 *pmap, long long npairs, const int *wmap,
                             int wall0, int nwall, const int *rmap, int rad0, int nrad, const int2 *cmap,
                             const int *wcirc, const int *rcirc, int nmode, float uf, double *Xo, double *Mo,
                             double *No, double *Uo, double *Zo, int grid, cudaStream_t s);
cudaError_t pk_launch_violation(const PkDev &D, unsigned long long *out, int grid, cudaStream_t s);
cudaError_t pk_shard_prepare(int V, bool stream_hint, int *blocks_per_sm);
cudaError_t pk_launch_shard_begin(int V, bool stream_hint, const PkDev &D, const PkRun &R, int grid, int nb,
                                  int row_lo, int row_hi, double4 *exch, cudaStream_t s);
cudaError_t pk_launch_shard_end(int V, const PkDev &D, const PkRun &R, long long k, int nb, const double4 *exch,
                                unsigned *done, cudaStream_t s);

// The sharded instance's fused sweep loop (pk_shard_fused): ranks
// [rank0, rank0 + nlocal) of `nranks` run in one cooperative launch on this
// device, `blocks` CTAs each; every rank's exchange buffer and flag array
// is given as this device sees it (its own memory, or a peer GPU's mapped
// into this process).
#define PK_XCH_MAX 8
struct PkXch {
    int nranks, rank0, nlocal, blocks;
    unsigned long long epoch;                    // flag epoch of this launch (the same on every rank)
    double4 *exch[PK_XCH_MAX];                   // rank q's exchange buffer: [2][nranks][N] double4
    unsigned long long *flag[PK_XCH_MAX];        // rank q's flags: [nranks]
    int row_lo[PK_XCH_MAX], row_hi[PK_XCH_MAX];  // block rows of the local ranks
};
cudaError_t pk_shard_fused_blocks(int V, bool stream_hint, int *blocks_per_sm);
cudaError_t pk_launch_shard_fused(int V, bool stream_hint, const PkDev *devs, const PkRun &R, const PkXch &X,
                                  cudaStream_t s);

// Cluster-resident solver (onchip_kernels.cu).  Instances of size class c
// need a group of 2^c CTAs (c = 0 .. OC_CLASSES - 1).
#define OC_MAX_WALLS 4    // walls per circle the solver holds on chip
#define OC_MAX_GROUP 16   // CTAs of the largest group (one whole cluster)
#define OC_CLASSES 5      // group sizes 1, 2, 4, 8, 16
struct OcArgs {
    const int *queue;              // instances by class, each class largest first
    int qoff[OC_CLASSES + 1];      // class c is queue[qoff[c] .. qoff[c + 1])
    unsigned *ctr;                 // [OC_CLASSES] grab counters, zeroed before each launch
    const unsigned char *glog2;    // per cluster: log2 of its group size
};
long long pk_onchip_bytes(int n_circles, int group);
cudaError_t pk_onchip_max_clusters(int V, int csize, int smem, int *clusters);
cudaError_t pk_launch_onchip(int V, const PkDev &D, const PkRun &R, const OcArgs &A, int n_clusters, int csize,
                             int smem, cudaStream_t s);
