// Host-side internals of the engine shared by engine.cu and the drop-in
// sweep functions.
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <string>
#include <vector>

#include "common.cuh"
#include "generic.cuh"
#include "packing.cuh"
#include "packing_launch.h"

int pdm_set_error(int status, const char *fmt, ...);
void pdm_clear_status();  // marks the calling thread's last call as successful

// Result of classifying a host graph.
struct GraphInfo {
    int ok = 0;                    // all factors known and well-formed
    std::vector<int> kind;         // per factor PARADMM_OP_*
    // packing structure (valid when packing_ok)
    int packing_ok = 0;
    std::string packing_why;       // why the packing engine cannot run it
    int N = 0;                     // circles
    std::vector<int> centre_var, radius_var;  // per circle
    std::vector<int> circle_of_var;           // -1 if none
};

// Parameters a captured per-instance launch was built for.
struct PkGraphKey {
    int n_iter;
    double tol;
    int check_every, fallback_after, prof, cluster, n_coop, inst_grid, n_early;
    int bal_period, bal_lmin, bal_lmax;
    double bal_mu;
    int schedule, bal_any, yield_below;
};

struct PkHost {
    int V = 2, BW = 64;
    bool stream_hint = true;
    int dynamic = 1;
    int grid = 0;
    int n_inst = 0, n_items = 0, n_circ = 0;
    long long n_tiles = 0;
    int n_wall = 0, n_rad = 0;
    std::vector<PkInst> inst;
    std::vector<int4> items;
    std::vector<PkCircle> circ;
    std::vector<float4> wall_vp, wall_coef;
    std::vector<double2> wall_rho;
    std::vector<int> wall_circle;   // local circle of each wall (within its instance)
    std::vector<float4> rad_coef;
    std::vector<double> rad_rho;
    std::vector<int> rad_circle;
    std::vector<int> wall_base, rad_base;  // per instance
    std::vector<double> init_Z;      // per global circle (cx, cy, r)
    PkDev D{};
    long long it_next = 0;           // global sweep counter
    std::vector<long long> upload_iter;
    std::vector<long long> age;        // per instance: sweeps run since its state was set (balancing ages)
    std::vector<long long> last_swept; // per instance: global index of its last sweep (grid schedule; -1: none)
    int bal_period = 0;              // residual balancing of the penalties (paradmm_gpu_set_rho_balance)
    double bal_mu = 10.0;
    int bal_lmin = -1, bal_lmax = 4;
    std::vector<int> nmode;
    std::vector<PkStatus> status;    // host copy after the last launch
    std::vector<long long> iters_last_call;
    int schedule = PARADMM_SCHEDULE_GRID;  // resolved schedule
    int inst_grid = 0;               // CTAs of the per-instance schedule
    int cluster = 1;                 // CTAs per large instance in the per-instance schedule
    int coop_min_n = 0;              // instances with N >= this are solved by a whole cluster
    int n_coop = 0;                  // how many instances that is (the first n_coop of the order)
    int n_early = 0;                 // clusters that start on the on-chip-solver instances (after the coop part of the order)
    // cluster-resident schedule (PARADMM_SCHEDULE_ONCHIP)
    int oc_csize = 0, oc_clusters = 0, oc_smem = 0;
    int *d_oc_queue = nullptr;
    unsigned *d_oc_ctr = nullptr;
    unsigned char *d_oc_glog2 = nullptr;
    OcArgs oc_args{};
    std::vector<int> order;          // instances, largest first (per-instance schedule)
    int *d_order = nullptr;          // the same on the device
    int prof = 0;                    // per-phase timing requested
    int fallback_after = 0;          // per-instance schedule: restart from the plain start after this many sweeps
    int tail_yield = 0;              // per-instance schedule: hand the last this-many instances to the grid schedule
    int yielded_last_call = 0;       // instances the last solve call handed over
    std::vector<int> claim_order;    // the grid schedule's item claim order (host copy of D.claim)
    std::vector<int2> fin_list;      // consensus items (host copy of D.fin_items)
    int *d_claim_tail = nullptr;     // claim order / consensus items of the handed-over instances
    int2 *d_fin_tail = nullptr;
    // per-instance schedule: the solve call's launch sequence as a CUDA graph
    int use_graphs = 1;
    cudaGraphExec_t graph_exec = nullptr;
    PkGraphKey graph_key{};
    PkStatus *h_status = nullptr;    // pinned status staging
    DevCtl *h_ctl = nullptr;         // pinned control-block copy
    double phase_us[4] = {0, 0, 0, 0};  // last call: mean block time per sweep (us)
    // reference-layout maps (graph handles)
    int2 *d_pmap = nullptr; long long n_pmap = 0;
    int *d_wmap = nullptr, *d_rmap = nullptr, *d_wcirc = nullptr, *d_rcirc = nullptr;
    int2 *d_cmap = nullptr;
    int *d_flag = nullptr;
    unsigned long long *d_viol = nullptr;
    // shard of one instance (paradmm_gpu_create_packing_shard): this rank
    // stores the pair tiles of circle-block rows [row_lo, row_hi)
    int shard_n = 0, shard_rank = 0, row_lo = 0, row_hi = -1;
    int shard_running = 0, shard_phase = 0;  // a run is armed; 1 = the exchange of sweep shard_k is pending
    long long shard_it0 = 0, shard_k = 0, shard_stop = 0;  // first sweep of the run, next sweep, end of the run
    // fused exchange (paradmm_gpu_shard_run_fused)
    double4 *d_fx_exch = nullptr;              // [2][shard_n][N] partial sums, by sweep parity and rank
    unsigned long long *d_fx_flags = nullptr;  // [shard_n] each rank's (epoch, sweep) flag
    PkDev *d_fx_devs = nullptr;                // [PK_XCH_MAX] the local ranks' device views for one launch
    unsigned long long fx_epoch = 0;           // fused launches run so far (the flag epoch)
    double shard_tol = -1.0;
    int shard_check_every = 1;
    unsigned *d_done = nullptr;      // CTAs of the running consensus launch that finished
};

struct GenHost {
    GenDev D{};
    // factors with run-time compiled operators (PARADMM_OP_USER)
    int n_user = 0;
    int *d_user_f = nullptr;         // their factor ids
    int *d_user_id = nullptr;        // [factor] index of the operator in the compiled module
    long long *d_user_poff = nullptr;  // [factor] byte offset into d_user_params, -1 if none
    unsigned char *d_user_params = nullptr;
    const void *user_kernel = nullptr;  // cudaKernel_t of the compiled X-phase
    std::vector<int> radius_vars;    // for the total-radius metric
    double *d_Zprev = nullptr;
    double *d_acc = nullptr;         // residual sums
    unsigned long long *d_viol = nullptr;
    int zprev_valid = 0;
    double last_primal = -1, last_dual = -1;
    // residual balancing of the penalties (paradmm_gpu_set_rho_balance)
    int bal_period = 0, bal_lmin = -1, bal_lmax = 4;
    double bal_mu = 10.0;
    long long age = 0;               // sweeps since the state was set
    int bal_log2 = 0;                // log2 of the current penalty scale
    int bal_pending = 0;             // +1 / -1: a doubling / halving decided, not applied yet
    long long bal_apply_age = -1;    // age of the sweep after which it applies
};

// Run-time compiled operators (userops.cu): the X-phase kernel for operators
// given as (device source, function name), and its launch over the handle's
// user factors.
int pdm_user_kernel(const std::vector<std::pair<std::string, std::string>> &ops, int device, const void **kernel);
cudaError_t pdm_launch_user_x(const void *kernel, const GenDev &D, const GenHost &Gh, int with_m, cudaStream_t s);

struct paradmm_gpu {
    int engine = PARADMM_ENGINE_AUTO;
    int device = 0;
    int num_sms = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    paradmm_gpu_opts opts{};
    int from_graph = 0;
    int num_dims = 0, num_vars = 0, num_edges = 0, num_opts = 0;
    GenHost *gen = nullptr;
    PkHost *pk = nullptr;
    DevCtl *ctl = nullptr;
    double *d_stage[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};  // X M N U Z in reference layout
    std::vector<void *> allocs;
    long long device_bytes = 0;
    long long launches = 0;          // kernels launched by this handle
};
