// Host side of the B200 parADMM engine: the C-ABI of paradmm_gpu.h and the
// GPU-backed sweep functions of paradmm.h.
//
// Replaces the reference GPU back-end's host code (core/paradmm-gpu.cu:424-532
// copyGraphFromCPUtoGPU and the launch loop of packing/gpu.cu:257-291).
#include <ctype.h>
#include <dlfcn.h>
#include <stdarg.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <climits>
#include <cstddef>
#include <cmath>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "engine_internal.h"
#include "packing_launch.h"
#include "paradmm.h"
#include "paradmm_gpu.h"
#include "paradmm_learned.h"

// ===========================================================================
// Errors
// ===========================================================================
static thread_local int t_status = PARADMM_OK;
static thread_local char t_msg[512] = "";

int pdm_set_error(int status, const char *fmt, ...)
{
    t_status = status;
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(t_msg, sizeof t_msg, fmt, ap);
    va_end(ap);
    return status;
}

int pdm_cuda_fail(cudaError_t e, const char *what, const char *file, int line)
{
    int st = PARADMM_ECUDA;
    if (e == cudaErrorMemoryAllocation) st = PARADMM_ENOMEM;
    if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver || e == cudaErrorInvalidDevice) st = PARADMM_ENODEVICE;
    cudaGetLastError();  // clear a sticky-free error so the next call starts clean
    return pdm_set_error(st, "%s failed: %s (%s:%d)", what, cudaGetErrorString(e), file, line);
}

extern "C" void paradmm_internal_set_error(int status, const char *msg) { pdm_set_error(status, "%s", msg); }
extern "C" int paradmm_last_status(void) { return t_status; }
extern "C" const char *paradmm_last_error_string(void) { return t_msg; }

static inline void ok_status() { t_status = PARADMM_OK; }
void pdm_clear_status() { t_status = PARADMM_OK; }

struct DevGuard {
    int prev = -1;
    explicit DevGuard(int d)
    {
        if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
        if (prev != d) cudaSetDevice(d);
    }
    ~DevGuard()
    {
        int cur = -1;
        cudaGetDevice(&cur);
        if (prev >= 0 && cur != prev) cudaSetDevice(prev);
    }
};

// ===========================================================================
// Operator registry
// ===========================================================================
static std::mutex g_reg_mu;
static std::vector<std::pair<void *, int>> g_reg;

extern "C" int paradmm_gpu_register_op(paradmm_op_fn op, int kind)
{
    ok_status();
    if (!op || kind < PARADMM_OP_PAIR || kind > PARADMM_OP_RADIUS)
        return pdm_set_error(PARADMM_EINVAL, "paradmm_gpu_register_op: bad operator or kind %d", kind);
    std::lock_guard<std::mutex> lk(g_reg_mu);
    for (auto &p : g_reg)
        if (p.first == (void *)op) { p.second = kind; return PARADMM_OK; }
    g_reg.emplace_back((void *)op, kind);
    return PARADMM_OK;
}

// Operators with a device twin given as source, compiled at run time.
struct UserOp {
    void *host;
    std::string src, name;
    unsigned long long gen;  // registration generation (a re-registration changes it)
};
static std::vector<UserOp> g_user_ops;
static unsigned long long g_user_gen = 0;

extern "C" int paradmm_gpu_register_op_source(paradmm_op_fn op, const char *device_source, const char *function_name)
{
    ok_status();
    if (!op || !device_source || !function_name || !*function_name)
        return pdm_set_error(PARADMM_EINVAL, "paradmm_gpu_register_op_source: NULL argument");
    for (const char *c = function_name; *c; ++c)
        if (!(isalnum((unsigned char)*c) || *c == '_'))
            return pdm_set_error(PARADMM_EINVAL, "paradmm_gpu_register_op_source: '%s' is not an identifier", function_name);
    std::lock_guard<std::mutex> lk(g_reg_mu);
    for (UserOp &u : g_user_ops)
        if (u.host == (void *)op) {
            u.src = device_source;
            u.name = function_name;
            u.gen = ++g_user_gen;
            return PARADMM_OK;
        }
    g_user_ops.push_back({(void *)op, device_source, function_name, ++g_user_gen});
    return PARADMM_OK;
}

static int user_op_index(paradmm_op_fn f)
{
    std::lock_guard<std::mutex> lk(g_reg_mu);
    for (size_t i = 0; i < g_user_ops.size(); ++i)
        if (g_user_ops[i].host == (void *)f) return (int)i;
    return -1;
}

static int kind_of_name(const char *s)
{
    if (!s) return PARADMM_OP_UNKNOWN;
    if (!strcmp(s, "disk_collision_variable_radius")) return PARADMM_OP_PAIR;
    if (!strcmp(s, "disk_plane_collision_variable_radius")) return PARADMM_OP_WALL;
    if (!strcmp(s, "maximize_sum_of_squared_disk_radii_alpha")) return PARADMM_OP_RADIUS;
    return PARADMM_OP_UNKNOWN;
}

// Known by identity with this library's operators, by registration, or by
// the exported symbol name of the function the pointer refers to (a caller's
// own copy of a reference operator, e.g. packing/host.c compiled into a
// shared object or an executable linked with -rdynamic).
static int op_kind(paradmm_op_fn f)
{
    if (f == disk_collision_variable_radius) return PARADMM_OP_PAIR;
    if (f == disk_plane_collision_variable_radius) return PARADMM_OP_WALL;
    if (f == maximize_sum_of_squared_disk_radii_alpha) return PARADMM_OP_RADIUS;
    {
        std::lock_guard<std::mutex> lk(g_reg_mu);
        for (auto &p : g_reg)
            if (p.first == (void *)f) return p.second;
        for (const UserOp &u : g_user_ops)
            if (u.host == (void *)f) return PARADMM_OP_USER;
    }
    Dl_info info;
    if (f && dladdr((void *)f, &info) && info.dli_saddr == (void *)f) return kind_of_name(info.dli_sname);
    return PARADMM_OP_UNKNOWN;
}

// ===========================================================================
// Graph analysis
// ===========================================================================
static int analyze_graph(const graph *G, GraphInfo &gi, bool need_state)
{
    if (!G) return pdm_set_error(PARADMM_EINVAL, "graph is NULL");
    if (G->num_dims < 1 || G->num_edges < 1 || G->num_opts < 1 || G->num_vars < 1)
        return pdm_set_error(PARADMM_EINVAL, "empty graph (%d factors, %d vars, %d edges, %d dims)", G->num_opts,
                             G->num_vars, G->num_edges, G->num_dims);
    if (!G->list_of_operators_functions_pointers || !G->operatorix_to_numedges || !G->operatorix_to_edgelistix ||
        !G->varix_to_numedges || !G->varix_to_edgelistix || !G->edgeix_to_varlistix)
        return pdm_set_error(PARADMM_EINVAL, "graph topology arrays are not built");
    if (need_state && (!G->X || !G->M || !G->N || !G->U || !G->Z || !G->RHOS || !G->ALPHAS))
        return pdm_set_error(PARADMM_EINVAL, "graph state is not initialised (call initialize_RHOS_APHAS and initialize_X_N_Z_M_U_*)");
    const int d = G->num_dims;
    gi.kind.assign(G->num_opts, PARADMM_OP_UNKNOWN);
    long long edges_seen = 0;
    for (int f = 0; f < G->num_opts; ++f) {
        const int k = op_kind(G->list_of_operators_functions_pointers[f]);
        if (k == PARADMM_OP_UNKNOWN)
            return pdm_set_error(PARADMM_EUNSUPPORTED_OP,
                                 "factor %d: operator %p is not one of the packing operators "
                                 "(register the caller's copy with paradmm_gpu_register_op, or give its device "
                                 "twin with paradmm_gpu_register_op_source)",
                                 f, (void *)G->list_of_operators_functions_pointers[f]);
        const int nv = G->operatorix_to_numedges[f];
        const int *el = G->operatorix_to_edgelistix[f];
        if (nv < 1 || !el) return pdm_set_error(PARADMM_EINVAL, "factor %d has no edges", f);
        for (int q = 0; q < nv; ++q)
            if (el[q] != el[0] + q || el[q] < 0 || el[q] >= G->num_edges)
                return pdm_set_error(PARADMM_EINVAL, "factor %d: edge ids are not a contiguous in-range slice", f);
        edges_seen += nv;
        void *prm = G->list_of_operators_param_pointers ? G->list_of_operators_param_pointers[f] : nullptr;
        if (k == PARADMM_OP_PAIR && nv < 4) return pdm_set_error(PARADMM_EINVAL, "pair factor %d has %d edges (needs 4)", f, nv);
        if (k == PARADMM_OP_WALL && (nv < 2 || !prm))
            return pdm_set_error(PARADMM_EINVAL, "wall factor %d needs 2 edges and a [v, p] parameter block", f);
        if (k == PARADMM_OP_RADIUS && !prm) return pdm_set_error(PARADMM_EINVAL, "radius factor %d has no exponent parameter", f);
        gi.kind[f] = k;
    }
    if (edges_seen != G->num_edges) return pdm_set_error(PARADMM_EINVAL, "factor edge counts do not add up to num_edges");
    for (int e = 0; e < G->num_edges; ++e)
        if (G->edgeix_to_varlistix[e] < 0 || G->edgeix_to_varlistix[e] >= G->num_vars)
            return pdm_set_error(PARADMM_EINVAL, "edge %d: variable index out of range", e);
    gi.ok = 1;

    // ---- packing structure ----
    auto no = [&](const char *why) { gi.packing_ok = 0; gi.packing_why = why; return PARADMM_OK; };
    if (d != 2) return no("num_dims is not 2");
    for (int f = 0; f < G->num_opts; ++f)
        if (gi.kind[f] == PARADMM_OP_USER) return no("a factor uses a run-time compiled operator");
    const int V = G->num_vars;
    std::vector<int> role(V, 0), partner(V, -1);  // role 1 centre, 2 radius
    auto couple = [&](int c, int r) -> bool {
        if (role[c] == 2 || role[r] == 1) return false;
        if (role[c] == 1 && partner[c] != r) return false;
        if (role[r] == 2 && partner[r] >= 0 && partner[r] != c) return false;
        role[c] = 1; role[r] = 2; partner[c] = r; partner[r] = c;
        return true;
    };
    long long npairs = 0;
    for (int f = 0; f < G->num_opts; ++f) {
        const int e0 = G->operatorix_to_edgelistix[f][0], nv = G->operatorix_to_numedges[f];
        const int *ev = G->edgeix_to_varlistix + e0;
        if (gi.kind[f] == PARADMM_OP_PAIR) {
            if (nv != 4) return no("a pair factor has more than 4 edges");
            if (!couple(ev[0], ev[1]) || !couple(ev[2], ev[3])) return no("variables do not form consistent (centre, radius) couples");
            ++npairs;
        } else if (gi.kind[f] == PARADMM_OP_WALL) {
            if (nv != 2) return no("a wall factor has more than 2 edges");
            if (!couple(ev[0], ev[1])) return no("variables do not form consistent (centre, radius) couples");
        }
    }
    for (int f = 0; f < G->num_opts; ++f) {
        if (gi.kind[f] != PARADMM_OP_RADIUS) continue;
        const int e0 = G->operatorix_to_edgelistix[f][0], nv = G->operatorix_to_numedges[f];
        for (int q = 0; q < nv; ++q) {
            const int v = G->edgeix_to_varlistix[e0 + q];
            if (role[v] != 2) return no("a radius factor acts on a variable that is not a circle's radius");
        }
    }
    gi.circle_of_var.assign(V, -1);
    gi.centre_var.clear();
    gi.radius_var.clear();
    for (int v = 0; v < V; ++v) {
        if (role[v] == 0) return no("a variable has no pair or wall factor");
        if (role[v] == 1) {
            gi.circle_of_var[v] = (int)gi.centre_var.size();
            gi.centre_var.push_back(v);
            gi.radius_var.push_back(partner[v]);
        }
    }
    for (int c = 0; c < (int)gi.centre_var.size(); ++c) gi.circle_of_var[gi.radius_var[c]] = c;
    gi.N = (int)gi.centre_var.size();
    if (gi.N < 2 || gi.N > 32767) return no("circle count outside [2, 32767]");
    if (npairs != (long long)gi.N * (gi.N - 1) / 2) return no("not every pair of circles has exactly one pair factor");
    std::vector<uint8_t> seen((size_t)gi.N * gi.N, 0);
    double rho0[4] = {0, 0, 0, 0}, al0[4] = {0, 0, 0, 0};
    bool first = true;
    for (int f = 0; f < G->num_opts; ++f) {
        if (gi.kind[f] != PARADMM_OP_PAIR) continue;
        const int e0 = G->operatorix_to_edgelistix[f][0];
        const int P = gi.circle_of_var[G->edgeix_to_varlistix[e0]], Q = gi.circle_of_var[G->edgeix_to_varlistix[e0 + 2]];
        if (P >= Q) return no("pair factor circles out of order");
        uint8_t &s = seen[(size_t)P * gi.N + Q];
        if (s) return no("a pair of circles has two pair factors");
        s = 1;
        if (need_state) {
            for (int q = 0; q < 4; ++q) {
                if (first) { rho0[q] = G->RHOS[e0 + q]; al0[q] = G->ALPHAS[e0 + q]; }
                else if (G->RHOS[e0 + q] != rho0[q] || G->ALPHAS[e0 + q] != al0[q])
                    return no("pair-edge penalties or steps differ between pair factors");
            }
            first = false;
        }
    }
    if (need_state) {
        for (int e = 0; e < G->num_edges; ++e) {
            const int v = G->edgeix_to_varlistix[e];
            if (role[v] == 2 && (G->N[2LL * e] != G->N[2LL * e + 1] || G->U[2LL * e] != G->U[2LL * e + 1]))
                return no("a radius edge holds two different components (N or U)");
        }
        for (int c = 0; c < gi.N; ++c) {
            const int r = gi.radius_var[c];
            if (G->Z[2LL * r] != G->Z[2LL * r + 1]) return no("a radius variable holds two different components (Z)");
        }
    }
    gi.packing_ok = 1;
    return PARADMM_OK;
}

// ===========================================================================
// Device memory helpers
// ===========================================================================
static int dalloc(paradmm_gpu *h, void **p, size_t bytes)
{
    if (bytes == 0) bytes = 16;
    cudaError_t e = cudaMalloc(p, bytes);
    if (e != cudaSuccess) {
        *p = nullptr;
        return pdm_cuda_fail(e, "cudaMalloc", __FILE__, __LINE__);
    }
    h->allocs.push_back(*p);
    h->device_bytes += (long long)bytes;
    return PARADMM_OK;
}

template <class T>
static int dput(paradmm_gpu *h, T **p, const std::vector<T> &v)
{
    int rc = dalloc(h, (void **)p, sizeof(T) * v.size());
    if (rc) return rc;
    if (!v.empty()) PDM_CUDA(cudaMemcpy(*p, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice));
    return PARADMM_OK;
}

static void free_handle_memory(paradmm_gpu *h)
{
    if (h->pk) {
        if (h->pk->graph_exec) cudaGraphExecDestroy(h->pk->graph_exec);
        if (h->pk->h_status) cudaFreeHost(h->pk->h_status);
        if (h->pk->h_ctl) cudaFreeHost(h->pk->h_ctl);
        h->pk->graph_exec = nullptr;
        h->pk->h_status = nullptr;
        h->pk->h_ctl = nullptr;
    }
    for (void *p : h->allocs) cudaFree(p);
    h->allocs.clear();
    if (h->ev0) cudaEventDestroy(h->ev0);
    if (h->ev1) cudaEventDestroy(h->ev1);
    if (h->stream) cudaStreamDestroy(h->stream);
    h->ev0 = h->ev1 = nullptr;
    h->stream = nullptr;
}

static int handle_init(paradmm_gpu *h, const paradmm_gpu_opts *opts)
{
    if (opts) h->opts = *opts;
    else paradmm_gpu_default_opts(&h->opts);
    h->device = h->opts.device;
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess || ndev <= 0) {
        cudaGetLastError();
        return pdm_set_error(PARADMM_ENODEVICE, "no CUDA device available (%s)", cudaGetErrorString(e));
    }
    if (h->device < 0 || h->device >= ndev) return pdm_set_error(PARADMM_ENODEVICE, "device %d does not exist", h->device);
    PDM_CUDA(cudaSetDevice(h->device));
    PDM_CUDA(cudaDeviceGetAttribute(&h->num_sms, cudaDevAttrMultiProcessorCount, h->device));
    int coop = 0;
    PDM_CUDA(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, h->device));
    if (!coop) return pdm_set_error(PARADMM_ENODEVICE, "device %d cannot run cooperative launches", h->device);
    PDM_CUDA(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
    PDM_CUDA(cudaEventCreate(&h->ev0));
    PDM_CUDA(cudaEventCreate(&h->ev1));
    int rc = dalloc(h, (void **)&h->ctl, sizeof(DevCtl));
    if (rc) return rc;
    PDM_CUDA(cudaMemset(h->ctl, 0, sizeof(DevCtl)));
    return PARADMM_OK;
}

extern "C" void paradmm_gpu_default_opts(paradmm_gpu_opts *o)
{
    if (!o) return;
    memset(o, 0, sizeof *o);
    o->engine = PARADMM_ENGINE_AUTO;
    o->check_every = 1;
}

// ===========================================================================
// Packing engine: construction
// ===========================================================================
static void pair_coefficients(PkInst &I, const double rho[4], const double alpha[4])
{
    const double rx1 = rho[0], rr1 = rho[1], rx2 = rho[2], rr2 = rho[3];
    const double den = rr1 * rr2 * rx1 + rr2 * rx1 * rx2 + rr1 * (rr2 + rx1) * rx2;
    I.A1 = (float)(rr1 * rr2 * rx2 / den);
    I.A2 = (float)(rr1 * rr2 * rx1 / den);
    I.B2m1 = (float)((rr2 * rx1 + rr1 * (rr2 + rx1)) * rx2 / den - 1.0);
    I.C1 = (float)(rr2 * rx1 * rx2 / den);
    I.D1 = (float)(rr1 * (rx1 * rx2 + rr2 * (rx1 + rx2)) / den);
    I.C2 = (float)(rr1 * rx1 * rx2 / den);
    I.D2 = (float)(rr2 * (rx1 * rx2 + rr1 * (rx1 + rx2)) / den);
    for (int q = 0; q < 4; ++q) { I.rho[q] = rho[q]; I.alpha[q] = (float)alpha[q]; }
}

// Work items of one instance: pair tiles then circle blocks.  Returns the
// number added.
static int add_items(PkHost &P, int inst_id, int N, int nb)
{
    int n = 0;
    for (int I = 0; I < nb; ++I)
        for (int J = I; J < nb; ++J) { P.items.push_back(make_int4(inst_id, 0, I, J)); ++n; }
    for (int c0 = 0; c0 < N; c0 += PK_THREADS) { P.items.push_back(make_int4(inst_id, 1, c0, std::min(PK_THREADS, N - c0))); ++n; }
    return n;
}

// Work items of a shard: the pair tiles of block rows [row_lo, row_hi),
// then the circle blocks of those rows' circles.
static int add_items_rows(PkHost &P, int inst_id, int N, int nb, int row_lo, int row_hi, int BW)
{
    int n = 0;
    for (int I = row_lo; I < row_hi; ++I)
        for (int J = I; J < nb; ++J) { P.items.push_back(make_int4(inst_id, 0, I, J)); ++n; }
    const int c_end = std::min(N, row_hi * BW);
    for (int c0 = row_lo * BW; c0 < c_end; c0 += PK_THREADS) {
        P.items.push_back(make_int4(inst_id, 1, c0, std::min(PK_THREADS, c_end - c0)));
        ++n;
    }
    return n;
}

// Tile side: 64 circles (two columns per lane) or 128 (four).
static int pick_V(const paradmm_gpu_opts &o, int maxN)
{
    if (o.block_width == 128) return 4;
    if (o.block_width == 32 || o.block_width == 64) return 2;
    (void)maxN;
    return 2;
}

// Allocates and uploads everything of a packing handle whose host tables
// (inst, items, circ, walls, rads, init_Z) are filled.
// Per-instance schedule parameters.  Large instances are queued first and
// the first n_coop of the order (N >= coop_min_n) get a whole cluster of
// `cluster` CTAs each; the rest run one per CTA, starting with the instances
// the on-chip solver takes.  Those cost little per sweep, but any of them
// that cycles runs every sweep of the call, so n_early clusters (enough for
// one each) start on them at once instead of after every large instance.
// cluster 0: default (2); a size the device cannot launch falls back to the
// next smaller one.
static bool pk_small_path(const PkHost &P, int i)
{
    const PkInst &I = P.inst[i];
    const PkCircle &C = P.circ[I.circle_base];
    return I.N <= PK_SMALL_N && I.nb == 1 && C.wall_count <= PK_SMALL_W && C.rad_count == 1;
}

static void pk_set_instance_schedule(paradmm_gpu *h, int cluster, int coop_min_n)
{
    PkHost &P = *h->pk;
    int cl = cluster;
    if (cl != 1 && cl != 2 && cl != 4 && cl != 8) cl = 2;
    int nclu = 0;
    while (cl > 1 && (pk_instances_max_clusters(P.V, P.stream_hint, cl, &nclu) != cudaSuccess || nclu < 1)) {
        cudaGetLastError();
        cl /= 2;
    }
    P.cluster = cl;
    int ib = 0;
    if (pk_instances_blocks_per_sm(P.V, P.stream_hint, &ib) != cudaSuccess || ib < 1) ib = 1;
    P.inst_grid = cl > 1 ? nclu * cl : h->num_sms * ib;
    P.coop_min_n = coop_min_n > 0 ? coop_min_n : 200;
    std::vector<int> by_n(P.n_inst);
    for (int i = 0; i < P.n_inst; ++i) by_n[i] = i;
    std::stable_sort(by_n.begin(), by_n.end(), [&](int a, int b) { return P.inst[a].N > P.inst[b].N; });
    P.n_coop = 0;
    if (cl > 1)
        for (int q = 0; q < P.n_inst && P.inst[by_n[q]].N >= P.coop_min_n; ++q) P.n_coop = q + 1;
    P.order.assign(by_n.begin(), by_n.begin() + P.n_coop);
    int n_small = 0;
    for (int q = P.n_coop; q < P.n_inst; ++q)
        if (pk_small_path(P, by_n[q])) { P.order.push_back(by_n[q]); ++n_small; }
    for (int q = P.n_coop; q < P.n_inst; ++q)
        if (!pk_small_path(P, by_n[q])) P.order.push_back(by_n[q]);
    P.n_early = 0;
    if (cl > 1 && P.n_coop > 0 && n_small > 0)
        P.n_early = std::min((n_small + cl - 1) / cl, P.inst_grid / cl / 8);  // at most 1/8 of the clusters
    if (P.d_order && cudaMemcpy(P.d_order, P.order.data(), sizeof(int) * P.n_inst, cudaMemcpyHostToDevice) != cudaSuccess)
        cudaGetLastError();  // the queue keeps its previous order; still a valid permutation
}

// The cluster-resident schedule (onchip_kernels.cu): every instance's size
// class (the smallest group of 2^c CTAs whose shared memory holds it), the
// cluster size (16 CTAs where the device co-schedules such clusters, else
// 8), and the split of the resident clusters into groups: each class gets
// clusters in proportion to its share of the pair work (sum of N^2), largest
// class first, and the clusters left over go to the smallest class (a group
// also serves smaller classes once its own queue is empty).  Returns false,
// with a reason, when some instance cannot run this way.
static bool pk_onchip_plan(paradmm_gpu *h, std::string &why)
{
    PkHost &P = *h->pk;
    int optin = 0;
    if (cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, h->device) != cudaSuccess) {
        cudaGetLastError();
        why = "device attributes";
        return false;
    }
    const int smem = std::min(optin, 232448) - 2048;  // room for the kernel's static shared memory
    if (P.shard_n > 0) { why = "a shard of an instance"; return false; }
    if (h->from_graph) { why = "a handle built from a host graph (its uploads are not held on chip)"; return false; }
    int csize = 0, nclu = 0;
    for (int c : {16, 8}) {
        int n = 0;
        if (pk_onchip_max_clusters(P.V, c, smem, &n) == cudaSuccess && n >= 1) { csize = c; nclu = n; break; }
        cudaGetLastError();
    }
    if (csize == 0) { why = "no cluster of 8 CTAs with this much shared memory fits the device"; return false; }
    int maxc = 0;
    while ((1 << (maxc + 1)) <= csize) ++maxc;
    std::vector<std::vector<int>> cls(OC_CLASSES);
    std::vector<double> work(OC_CLASSES, 0.0);
    for (int i = 0; i < P.n_inst; ++i) {
        const PkInst &I = P.inst[i];
        const PkCircle &C0 = P.circ[I.circle_base];
        if (C0.wall_count > OC_MAX_WALLS || C0.rad_count != 1) {
            why = "an instance has more than 4 walls per circle or not one radius factor per circle";
            return false;
        }
        int c = 0;
        while (c <= maxc && pk_onchip_bytes(I.N, 1 << c) > smem) ++c;
        if (c > maxc) { why = "an instance is too large for one cluster's shared memory"; return false; }
        cls[c].push_back(i);
        work[c] += (double)I.N * I.N;
    }
    std::vector<int> q, qoff(OC_CLASSES + 1, 0);
    for (int c = 0; c < OC_CLASSES; ++c) {
        std::stable_sort(cls[c].begin(), cls[c].end(), [&](int a, int b) { return P.inst[a].N > P.inst[b].N; });
        qoff[c] = (int)q.size();
        q.insert(q.end(), cls[c].begin(), cls[c].end());
    }
    qoff[OC_CLASSES] = (int)q.size();
    double total = 0.0;
    for (double x : work) total += x;
    std::vector<unsigned char> glog2;
    for (int c = maxc; c >= 0; --c) {
        if (cls[c].empty()) continue;
        int want = (int)std::lround(nclu * work[c] / total);
        if (want < 1) want = 1;
        want = std::min(want, nclu - (int)glog2.size());
        for (int n = 0; n < want; ++n) glog2.push_back((unsigned char)c);
    }
    int smallest = 0;
    while (smallest < OC_CLASSES && cls[smallest].empty()) ++smallest;
    while ((int)glog2.size() < nclu) glog2.push_back((unsigned char)std::min(smallest, maxc));
    if (!P.d_oc_queue) {
        if (dput(h, &P.d_oc_queue, q) != PARADMM_OK || dalloc(h, (void **)&P.d_oc_ctr, sizeof(unsigned) * OC_CLASSES) != PARADMM_OK ||
            dput(h, &P.d_oc_glog2, glog2) != PARADMM_OK) {
            why = "device memory";
            return false;
        }
    } else {
        cudaMemcpy(P.d_oc_queue, q.data(), sizeof(int) * q.size(), cudaMemcpyHostToDevice);
        cudaMemcpy(P.d_oc_glog2, glog2.data(), glog2.size(), cudaMemcpyHostToDevice);
    }
    P.oc_csize = csize;
    P.oc_clusters = nclu;
    P.oc_smem = smem;
    P.oc_args.queue = P.d_oc_queue;
    for (int c = 0; c <= OC_CLASSES; ++c) P.oc_args.qoff[c] = qoff[c];
    P.oc_args.ctr = P.d_oc_ctr;
    P.oc_args.glog2 = P.d_oc_glog2;
    return true;
}

static int pk_finalize_build(paradmm_gpu *h)
{
    PkHost &P = *h->pk;
    P.n_inst = (int)P.inst.size();
    P.n_circ = (int)P.circ.size();
    P.n_wall = (int)P.wall_vp.size();
    P.n_rad = (int)P.rad_coef.size();
    // Items are instance-major (the residual reduction reads each instance's
    // items as one range); blocks claim them largest first so the dynamic
    // schedule ends evenly.
    P.n_items = (int)P.items.size();
    std::vector<int> claim(P.n_items);
    std::vector<long long> cost(P.n_items);
    {
        std::vector<int> base(P.n_inst + 1, 0);
        for (int q = 0; q < P.n_items; ++q) {
            const int4 &it = P.items[q];
            base[it.x + 1]++;
            const PkInst &I = P.inst[it.x];
            if (it.y == 1) cost[q] = it.w;
            else {
                const int nI = std::min(P.BW, I.N - it.z * P.BW), nJ = std::min(P.BW, I.N - it.w * P.BW);
                cost[q] = it.z == it.w ? (long long)nI * (nI - 1) / 2 : (long long)nI * nJ;
            }
            claim[q] = q;
        }
        for (int i = 0; i < P.n_inst; ++i) base[i + 1] += base[i];
        for (int i = 0; i < P.n_inst; ++i) { P.inst[i].item_base = base[i]; P.inst[i].n_items = base[i + 1] - base[i]; }
        std::stable_sort(claim.begin(), claim.end(), [&](int a, int b) { return cost[a] > cost[b]; });
    }

    // consensus items: one per circle block of every instance
    std::vector<int2> fin;
    for (int i = 0; i < P.n_inst; ++i) {
        P.inst[i].fin_base = (int)fin.size();
        for (int b = 0; b < P.inst[i].nb; ++b) fin.push_back(make_int2(i, b));
    }

    PkDev &D = P.D;
    D.n_inst = P.n_inst;
    D.n_items = P.n_items;
    D.n_claim = P.n_items;
    D.n_circ = P.n_circ;
    D.n_fin = (int)fin.size();
    D.n_finl = D.n_fin;
    int rc;
    if ((rc = dput(h, (PkInst **)&D.inst, P.inst))) return rc;
    if ((rc = dput(h, (int4 **)&D.items, P.items))) return rc;
    if ((rc = dput(h, (int **)&D.claim, claim))) return rc;
    P.claim_order = claim;
    if ((rc = dput(h, (PkCircle **)&D.circ, P.circ))) return rc;
    const long long tile_bytes = pk_tile_floats(P.BW) * 4LL;
    if ((rc = dalloc(h, (void **)&D.tiles, (size_t)(P.n_tiles * tile_bytes)))) return rc;
    if ((rc = dalloc(h, (void **)&D.row_part, sizeof(double4) * (size_t)P.n_tiles * P.BW))) return rc;
    if ((rc = dalloc(h, (void **)&D.col_part, sizeof(double4) * (size_t)P.n_tiles * P.BW))) return rc;
    {
        std::vector<double4> z(P.n_circ);
        for (int g = 0; g < P.n_circ; ++g) z[g] = make_double4(P.init_Z[3 * g], P.init_Z[3 * g + 1], P.init_Z[3 * g + 2], 0.0);
        if ((rc = dput(h, &D.Z, z))) return rc;
        if ((rc = dput(h, (double4 **)&D.Z0, z))) return rc;
        std::vector<float4> zp(P.n_circ);
        for (int g = 0; g < P.n_circ; ++g) zp[g] = make_float4((float)z[g].x, (float)z[g].y, (float)z[g].z, 0.f);
        if ((rc = dput(h, &D.Zp, zp))) return rc;
    }
    if ((rc = dalloc(h, (void **)&D.local_part, sizeof(double4) * (size_t)P.n_circ))) return rc;
    if ((rc = dput(h, (int2 **)&D.fin_items, fin))) return rc;
    P.fin_list = fin;
    if ((rc = dalloc(h, (void **)&D.blk_primal, sizeof(double) * 4 * (size_t)D.n_fin))) return rc;
    if ((rc = dalloc(h, (void **)&D.blk_dual, sizeof(double) * 4 * (size_t)D.n_fin))) return rc;
    PDM_CUDA(cudaMemset(D.blk_primal, 0, sizeof(double) * 4 * (size_t)D.n_fin));
    PDM_CUDA(cudaMemset(D.blk_dual, 0, sizeof(double) * 4 * (size_t)D.n_fin));
    if ((rc = dalloc(h, (void **)&D.status, sizeof(PkStatus) * (size_t)P.n_inst))) return rc;
    if ((rc = dput(h, (float4 **)&D.wall_vp, P.wall_vp))) return rc;
    if ((rc = dput(h, (float4 **)&D.wall_coef, P.wall_coef))) return rc;
    if ((rc = dput(h, (double2 **)&D.wall_rho, P.wall_rho))) return rc;
    if ((rc = dalloc(h, (void **)&D.wall_X, sizeof(float4) * (size_t)std::max(P.n_wall, 1)))) return rc;
    if ((rc = dalloc(h, (void **)&D.wall_U, sizeof(float4) * (size_t)std::max(P.n_wall, 1)))) return rc;
    if ((rc = dput(h, (float4 **)&D.rad_coef, P.rad_coef))) return rc;
    if ((rc = dput(h, (double **)&D.rad_rho, P.rad_rho))) return rc;
    if ((rc = dalloc(h, (void **)&D.rad_XU, sizeof(float2) * (size_t)std::max(P.n_rad, 1)))) return rc;
    if ((rc = dalloc(h, (void **)&P.d_viol, sizeof(unsigned long long) * (size_t)P.n_inst))) return rc;
    if ((rc = dalloc(h, (void **)&P.d_flag, sizeof(int)))) return rc;
    D.ctl = h->ctl;

    // grid: co-resident blocks for the cooperative launch
    int bps = 0;
    if (pk_max_blocks_per_sm(P.V, P.stream_hint, &bps) != cudaSuccess || bps < 1)
        return pdm_set_error(PARADMM_ECUDA, "packing kernel cannot be resident on this device");
    if (h->opts.ctas_per_sm > 0) bps = std::min(bps, h->opts.ctas_per_sm);
    P.grid = h->num_sms * bps;
    // Small problems: fewer CTAs (barrier cost grows with the CTA count and
    // there is no work for the rest).
    {
        int fin_n = D.n_fin;
        const int want = std::max(std::max(P.n_items, fin_n), P.n_inst);
        if (want < P.grid) P.grid = std::max(std::min(P.grid, h->num_sms), ((want + 31) / 32) * 32);
        if (P.grid > h->num_sms * bps) P.grid = h->num_sms * bps;
    }
    // Schedule: batches of small instances run one CTA per instance (no grid
    // barrier); a few or large instances share the grid-wide persistent loop.
    {
        int maxN = 0;
        for (const PkInst &I : P.inst) maxN = std::max(maxN, I.N);
        const int req = h->opts.schedule;
        const bool small = maxN <= 1024;
        if (req == PARADMM_SCHEDULE_INSTANCE && small) P.schedule = PARADMM_SCHEDULE_INSTANCE;
        else if (req == PARADMM_SCHEDULE_GRID || !small) P.schedule = PARADMM_SCHEDULE_GRID;
        else P.schedule = P.n_inst >= 8 ? PARADMM_SCHEDULE_INSTANCE : PARADMM_SCHEDULE_GRID;
        P.order.resize(P.n_inst);
        for (int i = 0; i < P.n_inst; ++i) P.order[i] = i;
        std::stable_sort(P.order.begin(), P.order.end(), [&](int a, int b) { return P.inst[a].N > P.inst[b].N; });
        if ((rc = dput(h, &P.d_order, P.order))) return rc;
        pk_set_instance_schedule(h, h->opts.cluster_size, h->opts.reserved[0]);
        if (req == PARADMM_SCHEDULE_ONCHIP) {
            std::string why;
            if (!pk_onchip_plan(h, why))
                return pdm_set_error(PARADMM_EUNSUPPORTED_GRAPH, "the cluster-resident schedule cannot run this batch: %s",
                                     why.c_str());
            P.schedule = PARADMM_SCHEDULE_ONCHIP;
        }
    }
    P.upload_iter.assign(P.n_inst, 0);
    P.age.assign(P.n_inst, 0);
    P.last_swept.assign(P.n_inst, -1);
    P.nmode.assign(P.n_inst, PK_MODE_Z);
    P.status.assign(P.n_inst, PkStatus{});
    for (auto &s : P.status) { s.resid_iter = -1; s.primal = s.dual = NAN; pk_bal_reset(s, 0); }
    P.iters_last_call.assign(P.n_inst, 0);
    return PARADMM_OK;
}

// Whether a launch must read the penalty scale: balancing on, or some
// instance still at a scale other than 1 (or with a change pending).
static int pk_bal_any(const PkHost &P)
{
    if (P.bal_period > 0) return 1;
    for (const PkStatus &s : P.status)
        if (s.bal_pass_age > 0 || s.bal_log2_cur != 0 || s.bal_log2_new != 0) return 1;
    return 0;
}

// Instance i's state was just set (create, warm start, upload): balancing
// ages restart, the penalty scale returns to 1.
static void pk_state_set(PkHost &P, int i)
{
    P.age[i] = 0;
    P.last_swept[i] = -1;
    pk_bal_reset(P.status[i], 0);
}

// Plain/warm state of every instance from its Z: one launch over all
// instances (grid.y = instance) when the grid allows it.  Pair and wall duals
// start at 0, radius duals at 0 or (radius_duals) at the radius prox's fixed
// point; dual_iters > 0 refines them by the reference's optimal-initialisation
// map (pk_init_state).
static int pk_init_all(paradmm_gpu *h, int radius_duals, int dual_iters = 0)
{
    PkHost &P = *h->pk;
    long long slots = 0;
    for (int i = 0; i < P.n_inst; ++i) slots = std::max(slots, (long long)P.inst[i].nb * (P.inst[i].nb + 1) / 2 * P.BW * P.BW);
    const int grid = (int)std::max(1LL, std::min<long long>(h->num_sms * 4, slots / 256 + 1));
    PkInitArgs A{};
    A.radius_duals = radius_duals;
    A.dual_iters = dual_iters;
    A.row_lo = P.row_lo;
    A.row_hi = P.row_hi;
    for (int i = 0; i < P.n_inst; ++i) {
        if (P.n_inst > 65535 || i == 0) {
            cudaError_t e = pk_launch_init(P.V, P.D, P.n_inst > 65535 ? i : -1, A, grid, h->stream);
            if (e != cudaSuccess) return pdm_cuda_fail(e, "pk_init_state", __FILE__, __LINE__);
        }
        P.nmode[i] = PK_MODE_Z;
        P.upload_iter[i] = P.it_next;
        pk_state_set(P, i);
    }
    PDM_CUDA(cudaStreamSynchronize(h->stream));
    return PARADMM_OK;
}

static int pk_init_instance_state(paradmm_gpu *h, int inst, const PkInitArgs &A)
{
    PkHost &P = *h->pk;
    PkInitArgs a = A;
    a.row_lo = P.row_lo;
    a.row_hi = P.row_hi;
    cudaError_t e = pk_launch_init(P.V, P.D, inst, a, h->num_sms * 4, h->stream);
    if (e != cudaSuccess) return pdm_cuda_fail(e, "pk_init_state", __FILE__, __LINE__);
    PDM_CUDA(cudaStreamSynchronize(h->stream));
    P.nmode[inst] = PK_MODE_Z;
    P.upload_iter[inst] = P.it_next;
    pk_state_set(P, inst);
    return PARADMM_OK;
}

// One instance of the structured packing problem (paradmm_packing_desc).
static int pk_add_desc(PkHost &P, const paradmm_packing_desc &d, int inst_id)
{
    const int N = d.n_circles;
    PkInst I{};
    I.N = N;
    I.nb = (N + P.BW - 1) / P.BW;
    I.circle_base = (int)P.circ.size();
    if (P.shard_n > 0) {  // one instance; only the rows [row_lo, row_hi) are stored
        const long long t_lo = pk_tri(P.row_lo, P.row_lo, I.nb);
        I.tile_base = -t_lo;
        P.n_tiles = pk_tri(P.row_hi, P.row_hi, I.nb) - t_lo;
    } else {
        I.tile_base = P.n_tiles;
        P.n_tiles += (long long)I.nb * (I.nb + 1) / 2;
    }
    const double rho[4] = {d.rho, d.rho, d.rho, d.rho}, al[4] = {d.alpha, d.alpha, d.alpha, d.alpha};
    pair_coefficients(I, rho, al);
    const long long E = (long long)N + 2LL * d.n_walls * N + 4LL * N * (N - 1) / 2;
    I.inv_ncomp = 1.0 / (2.0 * (double)E);
    P.wall_base.push_back((int)P.wall_vp.size());
    P.rad_base.push_back((int)P.rad_coef.size());
    for (int c = 0; c < N; ++c) {
        PkCircle C{};
        const double deg_c = (N - 1) + d.n_walls, deg_r = (N - 1) + d.n_walls + 1;
        C.inv_rho_c = 1.0 / (d.rho * (N - 1) + d.rho * d.n_walls);
        C.inv_rho_r = 1.0 / (d.rho * (N - 1) + d.rho * d.n_walls + d.rho_radius);
        C.w_c = deg_c;
        C.w_r = 2.0 * deg_r;
        C.wall_start = (int)P.wall_vp.size();
        C.wall_count = d.n_walls;
        for (int w = 0; w < d.n_walls; ++w) {
            const double *W = d.walls + 4 * w;
            P.wall_vp.push_back(make_float4((float)W[0], (float)W[1], (float)W[2], (float)W[3]));
            P.wall_coef.push_back(make_float4((float)d.rho, (float)d.rho, (float)d.alpha, (float)d.alpha));
            P.wall_rho.push_back(make_double2(d.rho, d.rho));
            P.wall_circle.push_back(c);
        }
        C.rad_start = (int)P.rad_coef.size();
        C.rad_count = 1;
        P.rad_coef.push_back(make_float4((float)d.exponent, (float)d.rho_radius, (float)d.alpha, 0.f));
        P.rad_rho.push_back(d.rho_radius);
        P.rad_circle.push_back(c);
        C.inst = inst_id;
        P.circ.push_back(C);
        P.init_Z.push_back(d.init[3 * c]);
        P.init_Z.push_back(d.init[3 * c + 1]);
        P.init_Z.push_back(d.init[3 * c + 2]);
    }
    if (P.shard_n > 0) add_items_rows(P, inst_id, N, I.nb, P.row_lo, P.row_hi, P.BW);
    else add_items(P, inst_id, N, I.nb);
    P.inst.push_back(I);
    return PARADMM_OK;
}

extern "C" int paradmm_gpu_create_packing(const paradmm_packing_desc *descs, int count, const paradmm_gpu_opts *opts,
                                          paradmm_gpu **out)
{
    ok_status();
    if (!out) return pdm_set_error(PARADMM_EINVAL, "out is NULL");
    *out = nullptr;
    if (!descs || count < 1) return pdm_set_error(PARADMM_EINVAL, "no packing instances");
    int maxN = 0;
    for (int i = 0; i < count; ++i) {
        const paradmm_packing_desc &d = descs[i];
        if (d.n_circles < 2 || d.n_circles > 32767 || d.n_walls < 0 || d.n_walls > 8 || (d.n_walls && !d.walls) || !d.init)
            return pdm_set_error(PARADMM_EINVAL, "instance %d: bad description (n_circles %d, n_walls %d)", i, d.n_circles, d.n_walls);
        if (!(d.rho > 0) || !(d.rho_radius > 0)) return pdm_set_error(PARADMM_EINVAL, "instance %d: penalties must be positive", i);
        maxN = std::max(maxN, d.n_circles);
    }
    paradmm_gpu *h = new paradmm_gpu();
    int rc = handle_init(h, opts);
    if (rc) { free_handle_memory(h); delete h; return rc; }
    DevGuard g(h->device);
    if (h->opts.engine != PARADMM_ENGINE_AUTO && h->opts.engine != PARADMM_ENGINE_PACKING) {
        free_handle_memory(h); delete h;
        return pdm_set_error(PARADMM_EUNSUPPORTED_GRAPH, "structured packing problems run on the packing engine only");
    }
    h->engine = PARADMM_ENGINE_PACKING;
    h->pk = new PkHost();
    PkHost &P = *h->pk;
    P.V = pick_V(h->opts, maxN);
    P.BW = 32 * P.V;
    P.stream_hint = true;
    P.dynamic = 1;
    for (int i = 0; i < count; ++i) pk_add_desc(P, descs[i], i);
    rc = pk_finalize_build(h);
    P.use_graphs = h->opts.reserved[1] ? 0 : 1;
    P.tail_yield = std::max(0, h->opts.reserved[2]);
    if (rc == PARADMM_OK) rc = pk_init_all(h, 0);
    if (rc) { free_handle_memory(h); delete h->pk; delete h; return rc; }
    h->num_dims = 2;
    *out = h;
    return PARADMM_OK;
}

// Packing handle from a host graph (single instance).
static int pk_build_from_graph(paradmm_gpu *h, const graph *G, const GraphInfo &gi)
{
    h->pk = new PkHost();
    PkHost &P = *h->pk;
    const int N = gi.N;
    P.V = pick_V(h->opts, N);
    P.BW = 32 * P.V;
    PkInst I{};
    I.N = N;
    I.nb = (N + P.BW - 1) / P.BW;
    I.circle_base = 0;
    I.tile_base = 0;
    P.n_tiles = (long long)I.nb * (I.nb + 1) / 2;
    I.inv_ncomp = 1.0 / ((double)G->num_edges * G->num_dims);
    // pair penalties/steps by position (uniform, checked by analyze_graph)
    double rho[4] = {1, 1, 1, 1}, al[4] = {1, 1, 1, 1};
    std::vector<int2> pmap;
    pmap.reserve((size_t)N * (N - 1) / 2);
    std::vector<std::vector<int>> walls_of(N), rads_of(N);
    for (int f = 0; f < G->num_opts; ++f) {
        const int e0 = G->operatorix_to_edgelistix[f][0];
        if (gi.kind[f] == PARADMM_OP_PAIR) {
            if (pmap.empty())
                for (int q = 0; q < 4; ++q) { rho[q] = G->RHOS[e0 + q]; al[q] = G->ALPHAS[e0 + q]; }
            const int Pc = gi.circle_of_var[G->edgeix_to_varlistix[e0]], Qc = gi.circle_of_var[G->edgeix_to_varlistix[e0 + 2]];
            pmap.push_back(make_int2(e0, (Pc << 16) | Qc));
        } else if (gi.kind[f] == PARADMM_OP_WALL) {
            walls_of[gi.circle_of_var[G->edgeix_to_varlistix[e0]]].push_back(f);
        } else {
            const int nv = G->operatorix_to_numedges[f];
            for (int q = 0; q < nv; ++q) rads_of[gi.circle_of_var[G->edgeix_to_varlistix[e0 + q]]].push_back(e0 + q);
        }
    }
    pair_coefficients(I, rho, al);
    std::vector<int> wmap, rmap;
    std::vector<int2> cmap(N);
    P.wall_base.push_back(0);
    P.rad_base.push_back(0);
    for (int c = 0; c < N; ++c) {
        PkCircle C{};
        const int cv = gi.centre_var[c], rv = gi.radius_var[c];
        cmap[c] = make_int2(cv, rv);
        double sc = 0, sr = 0;
        for (int q = 0; q < G->varix_to_numedges[cv]; ++q) sc += G->RHOS[G->varix_to_edgelistix[cv][q]];
        for (int q = 0; q < G->varix_to_numedges[rv]; ++q) sr += G->RHOS[G->varix_to_edgelistix[rv][q]];
        C.inv_rho_c = 1.0 / sc;
        C.inv_rho_r = 1.0 / sr;
        C.w_c = G->varix_to_numedges[cv];
        C.w_r = 2.0 * G->varix_to_numedges[rv];
        C.wall_start = (int)P.wall_vp.size();
        C.wall_count = (int)walls_of[c].size();
        for (int f : walls_of[c]) {
            const int e0 = G->operatorix_to_edgelistix[f][0];
            const double *W = (const double *)G->list_of_operators_param_pointers[f];
            P.wall_vp.push_back(make_float4((float)W[0], (float)W[1], (float)W[2], (float)W[3]));
            P.wall_coef.push_back(make_float4((float)G->RHOS[e0], (float)G->RHOS[e0 + 1], (float)G->ALPHAS[e0], (float)G->ALPHAS[e0 + 1]));
            P.wall_rho.push_back(make_double2(G->RHOS[e0], G->RHOS[e0 + 1]));
            P.wall_circle.push_back(c);
            wmap.push_back(e0);
        }
        C.rad_start = (int)P.rad_coef.size();
        C.rad_count = (int)rads_of[c].size();
        for (int e : rads_of[c]) {
            // exponent filled in below from the owning factor's params[0]
            P.rad_coef.push_back(make_float4(0.f, (float)G->RHOS[e], (float)G->ALPHAS[e], 0.f));
            P.rad_rho.push_back(G->RHOS[e]);
            P.rad_circle.push_back(c);
            rmap.push_back(e);
        }
        C.inst = 0;
        P.circ.push_back(C);
        P.init_Z.push_back(G->Z[2LL * cv]);
        P.init_Z.push_back(G->Z[2LL * cv + 1]);
        P.init_Z.push_back(G->Z[2LL * rv]);
    }
    // exponents of the radius factors, by edge
    {
        std::unordered_map<int, float> expo;
        for (int f = 0; f < G->num_opts; ++f)
            if (gi.kind[f] == PARADMM_OP_RADIUS) {
                const int e0 = G->operatorix_to_edgelistix[f][0], nv = G->operatorix_to_numedges[f];
                const float a = (float)((const double *)G->list_of_operators_param_pointers[f])[0];
                for (int q = 0; q < nv; ++q) expo[e0 + q] = a;
            }
        for (size_t q = 0; q < rmap.size(); ++q) P.rad_coef[q].x = expo[rmap[q]];
    }
    add_items(P, 0, N, I.nb);
    P.inst.push_back(I);
    int rc = pk_finalize_build(h);
    if (rc) return rc;
    P.n_pmap = (long long)pmap.size();
    if ((rc = dput(h, &P.d_pmap, pmap))) return rc;
    if ((rc = dput(h, &P.d_wmap, wmap))) return rc;
    if ((rc = dput(h, &P.d_rmap, rmap))) return rc;
    if ((rc = dput(h, &P.d_cmap, cmap))) return rc;
    if ((rc = dput(h, &P.d_wcirc, P.wall_circle))) return rc;
    if ((rc = dput(h, &P.d_rcirc, P.rad_circle))) return rc;
    return PARADMM_OK;
}

// Reference-layout staging buffers on the device (allocated on first use).
static int ensure_stage(paradmm_gpu *h)
{
    if (h->d_stage[0]) return PARADMM_OK;
    const size_t ne = (size_t)h->num_edges * h->num_dims, nz = (size_t)h->num_vars * h->num_dims;
    for (int q = 0; q < 4; ++q) {
        int rc = dalloc(h, (void **)&h->d_stage[q], sizeof(double) * ne);
        if (rc) return rc;
    }
    return dalloc(h, (void **)&h->d_stage[4], sizeof(double) * nz);
}

static int pk_upload_graph(paradmm_gpu *h, const graph *G)
{
    PkHost &P = *h->pk;
    int rc = ensure_stage(h);
    if (rc) return rc;
    if (!P.D.aux && (rc = dalloc(h, (void **)&P.D.aux, (size_t)(P.n_tiles * pk_tile_floats(P.BW) * 4LL)))) return rc;
    const size_t ne = (size_t)h->num_edges * 2, nz = (size_t)h->num_vars * 2;
    PDM_CUDA(cudaMemcpyAsync(h->d_stage[2], G->N, sizeof(double) * ne, cudaMemcpyHostToDevice, h->stream));
    PDM_CUDA(cudaMemcpyAsync(h->d_stage[3], G->U, sizeof(double) * ne, cudaMemcpyHostToDevice, h->stream));
    PDM_CUDA(cudaMemcpyAsync(h->d_stage[4], G->Z, sizeof(double) * nz, cudaMemcpyHostToDevice, h->stream));
    PDM_CUDA(cudaMemsetAsync(P.d_flag, 0, sizeof(int), h->stream));
    cudaError_t e = pk_launch_scatter(P.V, P.D, 0, P.d_pmap, P.n_pmap, P.d_wmap, 0, P.n_wall, P.d_rmap, 0, P.n_rad,
                                      P.d_cmap, h->d_stage[2], h->d_stage[3], h->d_stage[4], P.d_flag,
                                      h->num_sms * 8, h->stream);
    if (e != cudaSuccess) return pdm_cuda_fail(e, "pk_scatter", __FILE__, __LINE__);
    int flag = 0;
    PDM_CUDA(cudaMemcpyAsync(&flag, P.d_flag, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
    PDM_CUDA(cudaStreamSynchronize(h->stream));
    if (flag)
        return pdm_set_error(PARADMM_EUNSUPPORTED_GRAPH,
                             "the uploaded state has radius edges whose two components differ; "
                             "the packing engine keeps one (use PARADMM_ENGINE_GENERIC_F64)");
    P.nmode[0] = PK_MODE_N;
    P.upload_iter[0] = P.it_next;
    pk_state_set(P, 0);
    return PARADMM_OK;
}

static int pk_download_graph(paradmm_gpu *h, graph *G)
{
    PkHost &P = *h->pk;
    int rc = ensure_stage(h);
    if (rc) return rc;
    const int nm = P.nmode[0];
    // a rescale of the penalties due in the next pass belongs to the U of the
    // last sweep (the reference form applies it right after that sweep)
    const PkStatus &bs = P.status[0];
    const long long next_age = P.age[0] + 1;
    const float uf = (bs.bal_pass_age > 0 && bs.bal_pass_age == next_age && bs.bal_log2_new != bs.bal_log2_cur)
                         ? (bs.bal_log2_new > bs.bal_log2_cur ? 0.5f : 2.0f) : 1.0f;
    cudaError_t e = pk_launch_gather(P.V, P.D, 0, P.d_pmap, P.n_pmap, P.d_wmap, 0, P.n_wall, P.d_rmap, 0, P.n_rad,
                                     P.d_cmap, P.d_wcirc, P.d_rcirc, nm, uf, h->d_stage[0], h->d_stage[1],
                                     h->d_stage[2], h->d_stage[3], h->d_stage[4], h->num_sms * 8, h->stream);
    if (e != cudaSuccess) return pdm_cuda_fail(e, "pk_gather", __FILE__, __LINE__);
    const size_t ne = (size_t)h->num_edges * 2, nz = (size_t)h->num_vars * 2;
    double *dst[5] = {G->X, G->M, G->N, G->U, G->Z};
    for (int q = 0; q < 5; ++q) {
        if (nm == PK_MODE_N && q < 2) continue;  // no sweep since the upload: X and M are the caller's
        PDM_CUDA(cudaMemcpyAsync(dst[q], h->d_stage[q], sizeof(double) * (q == 4 ? nz : ne), cudaMemcpyDeviceToHost, h->stream));
    }
    PDM_CUDA(cudaStreamSynchronize(h->stream));
    return PARADMM_OK;
}

// The first-sweep mode an instance still owes its next sweep after a launch
// in which `last` was its last executed sweep (PK_MODE_RECOMPUTE: none).
static int pk_pending_mode(const PkStatus &s, long long last)
{
    if (last < s.mode_iter) return s.nmode;                         // the mode's sweep did not run
    if (last == s.mode_iter && s.nmode == PK_MODE_N) return PK_MODE_XN;  // X of that sweep came from N
    return PK_MODE_RECOMPUTE;
}

// Runs up to n sweeps of every instance (persistent launches of at most
// PK_SWEEPS_PER_LAUNCH sweeps).  Per-instance iteration counts land in
// P.iters_last_call, statuses in P.status.
#define PK_SWEEPS_PER_LAUNCH 8192
// The per-instance launch of one solve call: status in, control block reset,
// the kernel (with its timing events), status and control block out.  Sweep
// indices restart at 0 in every call, so the kernel parameters depend only
// on (n, tol, check_every, fallback, profiling, schedule) and the sequence is
// captured once into a CUDA graph and replayed by later calls with the same
// parameters; the status goes through pinned host buffers.
static int pk_enqueue_instances(paradmm_gpu *h, const PkRun &R, bool capturing)
{
    PkHost &P = *h->pk;
    // in a capture, the timing events must become event-record nodes
    const unsigned evflags = capturing ? cudaEventRecordExternal : cudaEventRecordDefault;
    PDM_CUDA(cudaMemcpyAsync(P.D.status, P.h_status, sizeof(PkStatus) * P.n_inst, cudaMemcpyHostToDevice, h->stream));
    PDM_CUDA(cudaMemsetAsync(h->ctl, 0, sizeof(DevCtl), h->stream));
    PDM_CUDA(cudaEventRecordWithFlags(h->ev0, h->stream, evflags));
    cudaError_t e;
    if (P.schedule == PARADMM_SCHEDULE_ONCHIP) {
        PDM_CUDA(cudaMemsetAsync(P.d_oc_ctr, 0, sizeof(unsigned) * OC_CLASSES, h->stream));
        e = pk_launch_onchip(P.V, P.D, R, P.oc_args, P.oc_clusters, P.oc_csize, P.oc_smem, h->stream);
    } else {
        e = pk_launch_instances(P.V, P.stream_hint, P.D, R, P.d_order, P.n_coop, P.n_early, &h->ctl->item_ctr[0],
                                P.inst_grid, P.cluster, h->stream);
    }
    if (e != cudaSuccess) return pdm_cuda_fail(e, "per-instance packing launch", __FILE__, __LINE__);
    PDM_CUDA(cudaEventRecordWithFlags(h->ev1, h->stream, evflags));
    PDM_CUDA(cudaMemcpyAsync(P.h_status, P.D.status, sizeof(PkStatus) * P.n_inst, cudaMemcpyDeviceToHost, h->stream));
    PDM_CUDA(cudaMemcpyAsync(P.h_ctl, h->ctl, sizeof(DevCtl), cudaMemcpyDeviceToHost, h->stream));
    return PARADMM_OK;
}

static void pk_drop_graph(PkHost &P)
{
    if (P.graph_exec) cudaGraphExecDestroy(P.graph_exec);
    P.graph_exec = nullptr;
}

static int pk_run_grid(paradmm_gpu *h, long long n, double tol, int check_every, double *ms,
                       const std::vector<char> *skip, const std::vector<long long> *budget, const PkDev *Dv);

static int pk_run_instances(paradmm_gpu *h, long long n, double tol, int check_every, double *ms)
{
    PkHost &P = *h->pk;
    if (!P.h_status) {
        PDM_CUDA(cudaMallocHost((void **)&P.h_status, sizeof(PkStatus) * (size_t)P.n_inst));
        PDM_CUDA(cudaMallocHost((void **)&P.h_ctl, sizeof(DevCtl)));
    }
    for (int i = 0; i < P.n_inst; ++i) {
        PkStatus &s = P.h_status[i];
        s = P.status[i];
        s.last_iter = LLONG_MAX;
        s.check_from = 1;
        s.converged = 0;
        s.nonfinite = 0;
        s.nmode = P.nmode[i];
        s.mode_iter = 0;
        s.pad = 0;
        s.t_begin_ns = s.t_end_ns = 0;
        s.bal_base = -P.age[i];  // sweep 0 of this call produces the iterate of age age[i] + 1
        s.yield_at = 0;
    }
    PkRun R{};
    R.it0 = 0;
    R.n_iter = (int)std::min<long long>(n, INT_MAX);
    R.dynamic = 0;
    R.tol = tol;
    R.check_every = check_every < 1 ? 1 : check_every;
    R.fallback_after = P.fallback_after < n ? P.fallback_after : 0;
    R.prof = P.prof;
    R.bal_period = P.bal_period;
    R.bal_mu = P.bal_mu;
    R.bal_lmin = P.bal_lmin;
    R.bal_lmax = P.bal_lmax;
    R.bal_any = pk_bal_any(P);
    // the tail hand-off needs the grid-wide schedule to take over; a fallback
    // budget (restart inside the launch) exists on the per-instance schedule only
    R.yield_below = (P.schedule == PARADMM_SCHEDULE_INSTANCE && R.fallback_after == 0) ? P.tail_yield : 0;
    PkGraphKey key;
    memset(&key, 0, sizeof key);
    key.yield_below = R.yield_below;
    key.bal_period = R.bal_period;
    key.bal_mu = R.bal_mu;
    key.bal_lmin = R.bal_lmin;
    key.bal_lmax = R.bal_lmax;
    key.schedule = P.schedule;
    key.bal_any = R.bal_any;
    key.n_iter = R.n_iter;
    key.tol = tol;
    key.check_every = R.check_every;
    key.fallback_after = R.fallback_after;
    key.prof = R.prof;
    key.cluster = P.cluster;
    key.n_coop = P.n_coop;
    key.n_early = P.n_early;
    key.inst_grid = P.inst_grid;
    if (P.use_graphs && (!P.graph_exec || memcmp(&key, &P.graph_key, sizeof key) != 0)) {
        pk_drop_graph(P);
        cudaGraph_t g = nullptr;
        int rc = PARADMM_OK;
        cudaError_t e = cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal);
        if (e == cudaSuccess) {
            rc = pk_enqueue_instances(h, R, true);
            e = cudaStreamEndCapture(h->stream, &g);
        }
        if (e == cudaSuccess && rc == PARADMM_OK) e = cudaGraphInstantiate(&P.graph_exec, g, 0);
        if (g) cudaGraphDestroy(g);
        if (e != cudaSuccess || rc != PARADMM_OK) {  // not capturable here: launch directly from now on
            cudaGetLastError();
            ok_status();
            P.graph_exec = nullptr;
            P.use_graphs = 0;
        } else {
            P.graph_key = key;
        }
    }
    if (P.graph_exec) {
        PDM_CUDA(cudaGraphLaunch(P.graph_exec, h->stream));
    } else {
        int rc = pk_enqueue_instances(h, R, false);
        if (rc) return rc;
    }
    ++h->launches;
    PDM_CUDA(cudaStreamSynchronize(h->stream));
    const DevCtl &c = *P.h_ctl;
    if (c.err != DEV_OK)
        return pdm_set_error(PARADMM_ETIMEOUT, "packing kernel: a device-side wait ran out (%s)", pdm_dev_err_name(c.err));
    float t = 0;
    PDM_CUDA(cudaEventElapsedTime(&t, h->ev0, h->ev1));
    if (ms) *ms = t;
    if (P.prof && c.pad[1] > 0)  // mean CTA time per sweep: pass, sync, consensus, sync + stop test
        for (int q = 0; q < 4; ++q) P.phase_us[q] = (double)c.prof[q] / 1e3 / (double)c.pad[1];
    int rc = PARADMM_OK;
    for (int i = 0; i < P.n_inst; ++i) {
        const PkStatus &st = P.h_status[i];
        const long long ran = st.last_iter + 1;
        P.iters_last_call[i] = ran > 0 ? ran : 0;
        P.nmode[i] = pk_pending_mode(st, st.last_iter);
        P.status[i] = st;
        P.age[i] = (ran > 0 ? ran : 0) - st.bal_base;  // a fallback restart moved bal_base
        if (st.nonfinite) rc = pdm_set_error(PARADMM_ENONFINITE, "instance %d: residual became NaN/Inf", i);
    }
    P.it_next += n;
    if (rc != PARADMM_OK || R.yield_below <= 0) return rc;
    // tail hand-off: the instances that stopped for it continue on the
    // grid-wide schedule for the rest of their budget of n sweeps
    std::vector<char> skip(P.n_inst, 1);
    std::vector<long long> budget(P.n_inst, 0);
    int nyield = 0;
    for (int i = 0; i < P.n_inst; ++i) {
        const PkStatus &st = P.status[i];
        if (st.yield_at > 0 && st.last_iter == st.yield_at && !st.converged && !st.nonfinite &&
            P.iters_last_call[i] < n) {
            skip[i] = 0;
            budget[i] = n - P.iters_last_call[i];
            ++nyield;
        }
    }
    P.yielded_last_call = nyield;
    if (nyield == 0) return rc;
    // the grid-wide launches claim only these instances' work items and run
    // only their consensus items
    std::vector<int> claim, fin;
    for (int q : P.claim_order)
        if (!skip[P.items[q].x]) claim.push_back(q);
    for (const int2 &f : P.fin_list)
        if (!skip[f.x]) fin.push_back(f.x), fin.push_back(f.y);
    if (!P.d_claim_tail) {
        if ((rc = dalloc(h, (void **)&P.d_claim_tail, sizeof(int) * (size_t)P.n_items))) return rc;
        if ((rc = dalloc(h, (void **)&P.d_fin_tail, sizeof(int2) * P.fin_list.size()))) return rc;
    }
    PDM_CUDA(cudaMemcpyAsync(P.d_claim_tail, claim.data(), sizeof(int) * claim.size(), cudaMemcpyHostToDevice, h->stream));
    PDM_CUDA(cudaMemcpyAsync(P.d_fin_tail, fin.data(), sizeof(int) * fin.size(), cudaMemcpyHostToDevice, h->stream));
    PkDev Dv = P.D;
    Dv.claim = P.d_claim_tail;
    Dv.n_claim = (int)claim.size();
    Dv.fin_items = P.d_fin_tail;
    Dv.n_finl = (int)(fin.size() / 2);
    double ms2 = 0;
    rc = pk_run_grid(h, n, tol, check_every, &ms2, &skip, &budget, &Dv);
    if (ms) *ms += ms2;
    return rc;
}

// Grid-wide schedule: up to n sweeps of every instance not in `skip`, and
// at most budget[i] sweeps of instance i when `budget` is given (a finite
// last_iter per launch); iteration counts add to P.iters_last_call.
static int pk_run_grid(paradmm_gpu *h, long long n, double tol, int check_every, double *ms,
                       const std::vector<char> *skip, const std::vector<long long> *budget, const PkDev *Dv)
{
    PkHost &P = *h->pk;
    std::vector<char> done(P.n_inst, 0);
    std::vector<long long> ran_here(P.n_inst, 0);
    if (skip) done = *skip;
    double total_ms = 0;
    long long left = n;
    if (budget) {
        left = 0;
        for (int i = 0; i < P.n_inst; ++i)
            if (!done[i]) left = std::max(left, std::min(n, (*budget)[i]));
    }
    int rc = PARADMM_OK;
    while (left > 0) {
        const int chunk = (int)std::min<long long>(left, PK_SWEEPS_PER_LAUNCH);
        const long long it0 = P.it_next;
        int active = 0;
        std::vector<PkStatus> st(P.n_inst);
        for (int i = 0; i < P.n_inst; ++i) {
            PkStatus &s = st[i];
            s = P.status[i];
            if (!done[i] && budget && (*budget)[i] - ran_here[i] <= 0) done[i] = 1;
            s.last_iter = done[i] ? it0 - 1 : LLONG_MAX;
            if (!done[i] && budget) s.last_iter = it0 + (*budget)[i] - ran_here[i] - 1;
            s.check_from = it0 + 2;
            s.converged = 0;
            s.nonfinite = 0;
            s.nmode = P.nmode[i];
            s.mode_iter = it0;
            s.bal_base = it0 - P.age[i];
            // the first two finalisations of a launch read residual sums of the two
            // sweeps before it: valid only if this instance ran them
            s.bal_eval_from = std::max(s.bal_base + 2, P.last_swept[i] == it0 - 1 ? it0 : it0 + 2);
            if (!done[i]) ++active;
        }
        if (active == 0) break;
        PDM_CUDA(cudaMemcpyAsync(P.D.status, st.data(), sizeof(PkStatus) * P.n_inst, cudaMemcpyHostToDevice, h->stream));
        DevCtl c{};
        c.n_active = active;
        PDM_CUDA(cudaMemcpyAsync(h->ctl, &c, sizeof c, cudaMemcpyHostToDevice, h->stream));
        PkRun R{};
        R.it0 = it0;
        R.n_iter = chunk;
        R.dynamic = P.dynamic;
        R.tol = tol;
        R.check_every = check_every < 1 ? 1 : check_every;
        R.prof = P.prof;
        R.bal_period = P.bal_period;
        R.bal_mu = P.bal_mu;
        R.bal_lmin = P.bal_lmin;
        R.bal_lmax = P.bal_lmax;
        R.bal_any = pk_bal_any(P);
        PDM_CUDA(cudaEventRecord(h->ev0, h->stream));
        cudaError_t e = pk_launch_persistent(P.V, P.stream_hint, Dv ? *Dv : P.D, R, P.grid, h->stream);
        if (e != cudaSuccess) return pdm_cuda_fail(e, "packing persistent launch", __FILE__, __LINE__);
        ++h->launches;
        PDM_CUDA(cudaEventRecord(h->ev1, h->stream));
        PDM_CUDA(cudaMemcpyAsync(&c, h->ctl, sizeof c, cudaMemcpyDeviceToHost, h->stream));
        PDM_CUDA(cudaMemcpyAsync(st.data(), P.D.status, sizeof(PkStatus) * P.n_inst, cudaMemcpyDeviceToHost, h->stream));
        PDM_CUDA(cudaStreamSynchronize(h->stream));
        float t = 0;
        cudaEventElapsedTime(&t, h->ev0, h->ev1);
        total_ms += t;
        if (c.err != DEV_OK)
            return pdm_set_error(PARADMM_ETIMEOUT, "packing kernel: a device-side wait ran out (%s)", pdm_dev_err_name(c.err));
        const long long sweeps = (long long)c.pad[0];
        if (P.prof && sweeps > 0)
            for (int q = 0; q < 4; ++q) P.phase_us[q] = (double)c.prof[q] / 1e3 / P.grid / (double)sweeps;
        for (int i = 0; i < P.n_inst; ++i) {
            if (done[i]) continue;
            const long long last = std::min(st[i].last_iter, it0 + sweeps - 1);
            const long long ran = last - it0 + 1;
            if (ran > 0) { P.iters_last_call[i] += ran; ran_here[i] += ran; }
            if (ran > 0) { P.age[i] += ran; P.last_swept[i] = last; }
            P.nmode[i] = pk_pending_mode(st[i], last);
            P.status[i] = st[i];
            if (st[i].converged || st[i].nonfinite) done[i] = 1;
            if (st[i].nonfinite) rc = pdm_set_error(PARADMM_ENONFINITE, "instance %d: residual became NaN/Inf", i);
        }
        P.it_next = it0 + sweeps;
        left -= sweeps;
        if (sweeps < chunk) break;  // every instance stopped
    }
    if (ms) *ms = total_ms;
    return rc;
}

static int pk_run(paradmm_gpu *h, long long n, double tol, int check_every, double *ms)
{
    PkHost &P = *h->pk;
    std::fill(P.iters_last_call.begin(), P.iters_last_call.end(), 0LL);
    P.yielded_last_call = 0;
    if (P.schedule == PARADMM_SCHEDULE_INSTANCE || P.schedule == PARADMM_SCHEDULE_ONCHIP)
        return pk_run_instances(h, n, tol, check_every, ms);
    return pk_run_grid(h, n, tol, check_every, ms, nullptr, nullptr, nullptr);
}

// ===========================================================================
// Generic engine
// ===========================================================================
static int gen_build(paradmm_gpu *h, const graph *G, const GraphInfo &gi, bool fp64)
{
    h->gen = new GenHost();
    GenHost &Gh = *h->gen;
    GenDev &D = Gh.D;
    const int d = G->num_dims;
    D.num_dims = d;
    D.num_vars = G->num_vars;
    D.num_edges = G->num_edges;
    D.num_opts = G->num_opts;
    D.fp64 = fp64 ? 1 : 0;
    std::vector<int> kind(gi.kind), nv(G->num_opts);
    std::vector<long long> e0(G->num_opts), prm_off(G->num_opts, -1);
    std::vector<double> params;
    for (int f = 0; f < G->num_opts; ++f) {
        e0[f] = G->operatorix_to_edgelistix[f][0];
        nv[f] = G->operatorix_to_numedges[f];
        const double *p = G->list_of_operators_param_pointers ? (const double *)G->list_of_operators_param_pointers[f] : nullptr;
        if (kind[f] == PARADMM_OP_WALL) { prm_off[f] = (long long)params.size(); params.insert(params.end(), p, p + 2 * d); }
        if (kind[f] == PARADMM_OP_RADIUS) { prm_off[f] = (long long)params.size(); params.push_back(p[0]); }
    }
    std::vector<int> e2v(G->edgeix_to_varlistix, G->edgeix_to_varlistix + G->num_edges);
    std::vector<long long> voff(G->num_vars + 1, 0);
    for (int v = 0; v < G->num_vars; ++v) voff[v + 1] = voff[v] + G->varix_to_numedges[v];
    std::vector<int> vedges((size_t)voff[G->num_vars]);
    for (int v = 0; v < G->num_vars; ++v)
        std::copy(G->varix_to_edgelistix[v], G->varix_to_edgelistix[v] + G->varix_to_numedges[v], vedges.begin() + voff[v]);
    int rc;
    if ((rc = dput(h, (int **)&D.f_kind, kind))) return rc;
    if ((rc = dput(h, (long long **)&D.f_e0, e0))) return rc;
    if ((rc = dput(h, (int **)&D.f_nv, nv))) return rc;
    if ((rc = dput(h, (long long **)&D.f_param, prm_off))) return rc;
    if ((rc = dput(h, (double **)&D.params, params))) return rc;
    if ((rc = dput(h, (int **)&D.e2v, e2v))) return rc;
    if ((rc = dput(h, (long long **)&D.v_off, voff))) return rc;
    if ((rc = dput(h, (int **)&D.v_edges, vedges))) return rc;
    const size_t ne = (size_t)G->num_edges * d, nz = (size_t)G->num_vars * d;
    const size_t ts = fp64 ? sizeof(double) : sizeof(float);
    if ((rc = dalloc(h, &D.X, ts * ne)) || (rc = dalloc(h, &D.M, ts * ne)) || (rc = dalloc(h, &D.N, ts * ne)) ||
        (rc = dalloc(h, &D.U, ts * ne)))
        return rc;
    if ((rc = dalloc(h, (void **)&D.Z, sizeof(double) * nz))) return rc;
    if ((rc = dalloc(h, (void **)&Gh.d_Zprev, sizeof(double) * nz))) return rc;
    if ((rc = dalloc(h, (void **)&D.RHOS, sizeof(double) * G->num_edges))) return rc;
    if ((rc = dalloc(h, (void **)&D.ALPHAS, sizeof(double) * G->num_edges))) return rc;
    if ((rc = dalloc(h, (void **)&Gh.d_acc, sizeof(double) * 2))) return rc;
    if ((rc = dalloc(h, (void **)&Gh.d_viol, sizeof(unsigned long long)))) return rc;
    if (gi.packing_ok)
        for (int c = 0; c < gi.N; ++c) Gh.radius_vars.push_back(gi.radius_var[c]);

    // factors with run-time compiled operators: their ids, compact operator
    // ids, parameter bytes (16-byte aligned copies), and the compiled X phase
    std::vector<int> ufac, uid(G->num_opts, -1);
    std::vector<long long> upoff(G->num_opts, -1);
    std::vector<unsigned char> ubytes;
    std::vector<std::pair<std::string, std::string>> ops;
    std::vector<int> reg_to_compact;
    for (int f = 0; f < G->num_opts; ++f) {
        if (kind[f] != PARADMM_OP_USER) continue;
        const int r = user_op_index(G->list_of_operators_functions_pointers[f]);
        if (r < 0) return pdm_set_error(PARADMM_EUNSUPPORTED_OP, "factor %d: operator was unregistered", f);
        if ((int)reg_to_compact.size() <= r) reg_to_compact.resize(r + 1, -1);
        if (reg_to_compact[r] < 0) {
            std::lock_guard<std::mutex> lk(g_reg_mu);
            for (const auto &o : ops)
                if (o.second == g_user_ops[r].name)
                    return pdm_set_error(PARADMM_EINVAL, "two operators of the graph use the device name '%s'", o.second.c_str());
            reg_to_compact[r] = (int)ops.size();
            ops.emplace_back(g_user_ops[r].src, g_user_ops[r].name);
        }
        uid[f] = reg_to_compact[r];
        ufac.push_back(f);
        const void *prm = G->list_of_operators_param_pointers ? G->list_of_operators_param_pointers[f] : nullptr;
        if (prm) {
            const int bytes = G->list_of_operators_param_sizes ? G->list_of_operators_param_sizes[f] : 0;
            if (bytes <= 0)
                return pdm_set_error(PARADMM_EINVAL, "factor %d: a run-time compiled operator's params need their byte size "
                                     "(addNodeWithParamSize)", f);
            upoff[f] = (long long)ubytes.size();
            ubytes.insert(ubytes.end(), (const unsigned char *)prm, (const unsigned char *)prm + bytes);
            ubytes.resize((ubytes.size() + 15) & ~(size_t)15, 0);
        }
    }
    if (!ufac.empty()) {
        if (!fp64) return pdm_set_error(PARADMM_EUNSUPPORTED_GRAPH, "run-time compiled operators need the FP64 generic engine");
        Gh.n_user = (int)ufac.size();
        if ((rc = dput(h, &Gh.d_user_f, ufac))) return rc;
        if ((rc = dput(h, &Gh.d_user_id, uid))) return rc;
        if ((rc = dput(h, &Gh.d_user_poff, upoff))) return rc;
        if (ubytes.empty()) ubytes.resize(16, 0);
        if ((rc = dput(h, &Gh.d_user_params, ubytes))) return rc;
        if ((rc = pdm_user_kernel(ops, h->device, &Gh.user_kernel))) return rc;
    }
    return PARADMM_OK;
}

static int gen_upload(paradmm_gpu *h, const graph *G)
{
    GenHost &Gh = *h->gen;
    GenDev &D = Gh.D;
    const size_t ne = (size_t)G->num_edges * G->num_dims, nz = (size_t)G->num_vars * G->num_dims;
    const double *src[4] = {G->X, G->M, G->N, G->U};
    void *dst[4] = {D.X, D.M, D.N, D.U};
    if (D.fp64) {
        for (int q = 0; q < 4; ++q) PDM_CUDA(cudaMemcpyAsync(dst[q], src[q], sizeof(double) * ne, cudaMemcpyHostToDevice, h->stream));
    } else {
        std::vector<float> tmp(ne);
        for (int q = 0; q < 4; ++q) {
            for (size_t i = 0; i < ne; ++i) tmp[i] = (float)src[q][i];
            PDM_CUDA(cudaMemcpyAsync(dst[q], tmp.data(), sizeof(float) * ne, cudaMemcpyHostToDevice, h->stream));
            PDM_CUDA(cudaStreamSynchronize(h->stream));
        }
    }
    PDM_CUDA(cudaMemcpyAsync(D.Z, G->Z, sizeof(double) * nz, cudaMemcpyHostToDevice, h->stream));
    PDM_CUDA(cudaMemcpyAsync((void *)D.RHOS, G->RHOS, sizeof(double) * G->num_edges, cudaMemcpyHostToDevice, h->stream));
    PDM_CUDA(cudaMemcpyAsync((void *)D.ALPHAS, G->ALPHAS, sizeof(double) * G->num_edges, cudaMemcpyHostToDevice, h->stream));
    PDM_CUDA(cudaStreamSynchronize(h->stream));
    Gh.zprev_valid = 0;
    // the uploaded state starts the balancing ages; its penalties are scale 1
    Gh.age = 0;
    Gh.bal_log2 = 0;
    Gh.bal_pending = 0;
    Gh.bal_apply_age = -1;
    return PARADMM_OK;
}

static int gen_download(paradmm_gpu *h, graph *G)
{
    GenDev &D = h->gen->D;
    const size_t ne = (size_t)G->num_edges * G->num_dims, nz = (size_t)G->num_vars * G->num_dims;
    double *dst[4] = {G->X, G->M, G->N, G->U};
    const void *src[4] = {D.X, D.M, D.N, D.U};
    if (D.fp64) {
        for (int q = 0; q < 4; ++q) PDM_CUDA(cudaMemcpyAsync(dst[q], src[q], sizeof(double) * ne, cudaMemcpyDeviceToHost, h->stream));
        PDM_CUDA(cudaMemcpyAsync(G->Z, D.Z, sizeof(double) * nz, cudaMemcpyDeviceToHost, h->stream));
        PDM_CUDA(cudaStreamSynchronize(h->stream));
    } else {
        std::vector<float> tmp(ne);
        for (int q = 0; q < 4; ++q) {
            PDM_CUDA(cudaMemcpyAsync(tmp.data(), src[q], sizeof(float) * ne, cudaMemcpyDeviceToHost, h->stream));
            PDM_CUDA(cudaStreamSynchronize(h->stream));
            for (size_t i = 0; i < ne; ++i) dst[q][i] = (double)tmp[i];
        }
        PDM_CUDA(cudaMemcpyAsync(G->Z, D.Z, sizeof(double) * nz, cudaMemcpyDeviceToHost, h->stream));
        PDM_CUDA(cudaStreamSynchronize(h->stream));
    }
    return PARADMM_OK;
}

static int gen_phase(paradmm_gpu *h, int phase)
{
    GenHost &Gh = *h->gen;
    cudaError_t e = gen_launch_phase(Gh.D, phase, h->stream);
    if (e != cudaSuccess) return pdm_cuda_fail(e, "generic phase kernel", __FILE__, __LINE__);
    ++h->launches;
    if (Gh.n_user > 0 && (phase == GEN_PHASE_X || phase == GEN_PHASE_XM)) {
        e = pdm_launch_user_x(Gh.user_kernel, Gh.D, Gh, phase == GEN_PHASE_XM, h->stream);
        if (e != cudaSuccess) return pdm_cuda_fail(e, "run-time compiled operator kernel", __FILE__, __LINE__);
        ++h->launches;
    }
    return PARADMM_OK;
}

static int gen_sweep(paradmm_gpu *h)
{
    int rc;
    if ((rc = gen_phase(h, GEN_PHASE_XM)) || (rc = gen_phase(h, GEN_PHASE_Z)) || (rc = gen_phase(h, GEN_PHASE_UN))) return rc;
    return PARADMM_OK;
}

static int gen_residuals(paradmm_gpu *h, double *primal, double *dual)
{
    GenHost &Gh = *h->gen;
    PDM_CUDA(cudaMemsetAsync(Gh.d_acc, 0, sizeof(double) * 2, h->stream));
    cudaError_t e = gen_launch_resid(Gh.D, Gh.zprev_valid ? Gh.d_Zprev : nullptr, Gh.d_acc, h->stream);
    if (e != cudaSuccess) return pdm_cuda_fail(e, "generic residual kernel", __FILE__, __LINE__);
    double acc[2];
    PDM_CUDA(cudaMemcpyAsync(acc, Gh.d_acc, sizeof acc, cudaMemcpyDeviceToHost, h->stream));
    PDM_CUDA(cudaStreamSynchronize(h->stream));
    const double n = (double)Gh.D.num_edges * Gh.D.num_dims;
    *primal = std::sqrt(acc[0] / n);
    *dual = Gh.zprev_valid ? std::sqrt(acc[1] / n) : NAN;
    return PARADMM_OK;
}

static int gen_run(paradmm_gpu *h, long long n, double tol, int check_every, paradmm_stats *stats)
{
    GenHost &Gh = *h->gen;
    const size_t nz = (size_t)Gh.D.num_vars * Gh.D.num_dims;
    if (check_every < 1) check_every = 1;
    PDM_CUDA(cudaEventRecord(h->ev0, h->stream));
    long long done = 0;
    int converged = 0, rc = PARADMM_OK;
    double rp = NAN, rd = NAN;
    while (done < n) {
        const long long age = Gh.age + 1;  // of the iterate this sweep produces
        const bool check = tol >= 0 && ((done + 1) % check_every == 0 || done + 1 == n);
        const bool decide = Gh.bal_period > 0 && age % Gh.bal_period == 0;
        if (check || decide || done + 1 == n) {
            PDM_CUDA(cudaMemcpyAsync(Gh.d_Zprev, Gh.D.Z, sizeof(double) * nz, cudaMemcpyDeviceToDevice, h->stream));
            Gh.zprev_valid = 1;
        }
        if ((rc = gen_sweep(h))) return rc;
        ++done;
        ++Gh.age;
        double r = NAN, sdual = NAN;
        if (check || decide) {
            if ((rc = gen_residuals(h, &r, &sdual))) return rc;
        }
        // the balancing rule of the packing engine (pk_bal_decide): a decision on
        // iterate age a applies right after the sweep of age a + 2
        if (Gh.bal_pending != 0 && age == Gh.bal_apply_age) {
            cudaError_t e = gen_launch_rescale(Gh.D, Gh.bal_pending > 0 ? 2.0 : 0.5, h->stream);
            if (e != cudaSuccess) return pdm_cuda_fail(e, "generic rescale kernel", __FILE__, __LINE__);
            ++h->launches;
            Gh.bal_log2 += Gh.bal_pending;
            Gh.bal_pending = 0;
        }
        if (decide) {
            Gh.bal_pending = 0;
            if (r > Gh.bal_mu * sdual && Gh.bal_log2 < Gh.bal_lmax) Gh.bal_pending = 1;
            else if (sdual > Gh.bal_mu * r && Gh.bal_log2 > Gh.bal_lmin) Gh.bal_pending = -1;
            Gh.bal_apply_age = age + 2;
        }
        if (check) {
            rp = r;
            rd = sdual;
            if (!std::isfinite(rp + rd)) { rc = pdm_set_error(PARADMM_ENONFINITE, "residual became NaN/Inf"); break; }
            if (rp + rd <= tol) { converged = 1; break; }
        }
    }
    PDM_CUDA(cudaEventRecord(h->ev1, h->stream));
    PDM_CUDA(cudaStreamSynchronize(h->stream));
    float ms = 0;
    cudaEventElapsedTime(&ms, h->ev0, h->ev1);
    Gh.last_primal = rp;
    Gh.last_dual = rd;
    if (stats) {
        stats->iterations = done;
        stats->converged = converged;
        stats->status = rc;
        stats->primal = rp;
        stats->dual = rd;
        stats->device_ms = ms;
    }
    return rc;
}

// ===========================================================================
// Public C-ABI
// ===========================================================================
extern "C" int paradmm_gpu_create(const graph *G, const paradmm_gpu_opts *opts, paradmm_gpu **out)
{
    ok_status();
    if (!out) return pdm_set_error(PARADMM_EINVAL, "out is NULL");
    *out = nullptr;
    GraphInfo gi;
    int rc = analyze_graph(G, gi, true);
    if (rc) return rc;
    paradmm_gpu *h = new paradmm_gpu();
    rc = handle_init(h, opts);
    if (rc) { free_handle_memory(h); delete h; return rc; }
    DevGuard guard(h->device);
    h->from_graph = 1;
    h->num_dims = G->num_dims;
    h->num_vars = G->num_vars;
    h->num_edges = G->num_edges;
    h->num_opts = G->num_opts;
    int eng = h->opts.engine;
    if (eng == PARADMM_ENGINE_PACKING && !gi.packing_ok) {
        free_handle_memory(h); delete h;
        return pdm_set_error(PARADMM_EUNSUPPORTED_GRAPH, "packing engine: %s", gi.packing_why.c_str());
    }
    if (eng == PARADMM_ENGINE_AUTO) eng = gi.packing_ok ? PARADMM_ENGINE_PACKING : PARADMM_ENGINE_GENERIC_F64;
    h->engine = eng;
    if (eng == PARADMM_ENGINE_PACKING) {
        rc = pk_build_from_graph(h, G, gi);
        if (!rc) rc = pk_upload_graph(h, G);
    } else {
        rc = gen_build(h, G, gi, eng == PARADMM_ENGINE_GENERIC_F64);
        if (!rc) rc = gen_upload(h, G);
    }
    if (rc) {
        free_handle_memory(h);
        delete h->pk;
        delete h->gen;
        delete h;
        return rc;
    }
    *out = h;
    return PARADMM_OK;
}

static bool same_topology(const paradmm_gpu *h, const graph *G)
{
    return G && h->from_graph && G->num_dims == h->num_dims && G->num_vars == h->num_vars && G->num_edges == h->num_edges &&
           G->num_opts == h->num_opts;
}

extern "C" int paradmm_gpu_upload(paradmm_gpu *h, const graph *G)
{
    ok_status();
    if (!h) return pdm_set_error(PARADMM_EINVAL, "handle is NULL");
    if (!same_topology(h, G)) return pdm_set_error(PARADMM_EINVAL, "graph does not match the handle's topology");
    if (!G->X || !G->M || !G->N || !G->U || !G->Z || !G->RHOS || !G->ALPHAS) return pdm_set_error(PARADMM_EINVAL, "graph state is not initialised");
    DevGuard guard(h->device);
    return h->engine == PARADMM_ENGINE_PACKING ? pk_upload_graph(h, G) : gen_upload(h, G);
}

extern "C" int paradmm_gpu_download(paradmm_gpu *h, graph *G)
{
    ok_status();
    if (!h) return pdm_set_error(PARADMM_EINVAL, "handle is NULL");
    if (!same_topology(h, G)) return pdm_set_error(PARADMM_EINVAL, "graph does not match the handle's topology");
    if (!G->X || !G->M || !G->N || !G->U || !G->Z) return pdm_set_error(PARADMM_EINVAL, "graph state arrays are not allocated");
    DevGuard guard(h->device);
    return h->engine == PARADMM_ENGINE_PACKING ? pk_download_graph(h, G) : gen_download(h, G);
}

extern "C" int paradmm_gpu_solve(paradmm_gpu *h, int maxiter, double tol, paradmm_stats *stats)
{
    ok_status();
    if (!h) return pdm_set_error(PARADMM_EINVAL, "handle is NULL");
    if (maxiter < 0) return pdm_set_error(PARADMM_EINVAL, "maxiter < 0");
    DevGuard guard(h->device);
    if (stats) memset(stats, 0, sizeof *stats);
    if (maxiter == 0) return PARADMM_OK;
    if (h->engine != PARADMM_ENGINE_PACKING) return gen_run(h, maxiter, tol, h->opts.check_every, stats);
    if (h->pk->shard_n > 0)
        return pdm_set_error(PARADMM_EINVAL, "a shard of an instance sweeps through paradmm_gpu_shard_begin/end only");
    double ms = 0;
    const int rc = pk_run(h, maxiter, tol, h->opts.check_every, &ms);
    if (stats) {
        PkHost &P = *h->pk;
        long long it = 0;
        int conv = 1;
        double rp = 0, rd = 0;
        for (int i = 0; i < P.n_inst; ++i) {
            it = std::max(it, P.iters_last_call[i]);
            conv &= P.status[i].converged;
            rp = std::max(rp, P.status[i].primal);
            rd = std::max(rd, P.status[i].dual);
        }
        stats->iterations = it;
        stats->converged = conv;
        stats->status = rc;
        stats->primal = rp;
        stats->dual = rd;
        stats->device_ms = ms;
        stats->max_violation = NAN;
        stats->total_radius = NAN;
    }
    return rc;
}

extern "C" int paradmm_gpu_iterate(paradmm_gpu *h, int n) { return paradmm_gpu_solve(h, n, -1.0, nullptr); }

// Max violation per instance (device) and total radius (host, from Z).
static int pk_metrics(paradmm_gpu *h, std::vector<double> &viol, std::vector<double> &total)
{
    PkHost &P = *h->pk;
    PDM_CUDA(cudaMemsetAsync(P.d_viol, 0, sizeof(unsigned long long) * P.n_inst, h->stream));
    cudaError_t e = pk_launch_violation(P.D, P.d_viol, h->num_sms * 8, h->stream);
    if (e != cudaSuccess) return pdm_cuda_fail(e, "pk_violation", __FILE__, __LINE__);
    std::vector<unsigned long long> vb(P.n_inst);
    std::vector<double4> z(P.n_circ);
    PDM_CUDA(cudaMemcpyAsync(vb.data(), P.d_viol, sizeof(unsigned long long) * P.n_inst, cudaMemcpyDeviceToHost, h->stream));
    PDM_CUDA(cudaMemcpyAsync(z.data(), P.D.Z, sizeof(double4) * P.n_circ, cudaMemcpyDeviceToHost, h->stream));
    PDM_CUDA(cudaStreamSynchronize(h->stream));
    viol.resize(P.n_inst);
    total.assign(P.n_inst, 0.0);
    for (int i = 0; i < P.n_inst; ++i) memcpy(&viol[i], &vb[i], sizeof(double));
    for (int g = 0; g < P.n_circ; ++g) total[P.circ[g].inst] += z[g].z;
    return PARADMM_OK;
}

extern "C" int paradmm_gpu_instance_stats(paradmm_gpu *h, paradmm_stats *stats)
{
    ok_status();
    if (!h || !stats) return pdm_set_error(PARADMM_EINVAL, "NULL argument");
    DevGuard guard(h->device);
    if (h->engine != PARADMM_ENGINE_PACKING) return paradmm_gpu_stats(h, stats);
    PkHost &P = *h->pk;
    std::vector<double> viol, total;
    int rc = pk_metrics(h, viol, total);
    if (rc) return rc;
    for (int i = 0; i < P.n_inst; ++i) {
        paradmm_stats &s = stats[i];
        memset(&s, 0, sizeof s);
        s.iterations = P.iters_last_call[i];
        s.converged = P.status[i].converged;
        s.status = P.status[i].nonfinite ? PARADMM_ENONFINITE : PARADMM_OK;
        s.primal = P.status[i].resid_iter >= 0 ? P.status[i].primal : NAN;
        s.dual = P.status[i].resid_iter >= 0 ? P.status[i].dual : NAN;
        s.max_violation = viol[i];
        s.total_radius = total[i];
    }
    return PARADMM_OK;
}

extern "C" int paradmm_gpu_stats(paradmm_gpu *h, paradmm_stats *out)
{
    ok_status();
    if (!h || !out) return pdm_set_error(PARADMM_EINVAL, "NULL argument");
    DevGuard guard(h->device);
    if (h->engine == PARADMM_ENGINE_PACKING) {
        if (h->pk->n_inst != 1) return pdm_set_error(PARADMM_EINVAL, "handle has %d instances: use paradmm_gpu_instance_stats", h->pk->n_inst);
        return paradmm_gpu_instance_stats(h, out);
    }
    GenHost &Gh = *h->gen;
    memset(out, 0, sizeof *out);
    int rc = gen_residuals(h, &out->primal, &out->dual);
    if (rc) return rc;
    PDM_CUDA(cudaMemsetAsync(Gh.d_viol, 0, sizeof(unsigned long long), h->stream));
    cudaError_t e = gen_launch_violation(Gh.D, Gh.d_viol, h->stream);
    if (e != cudaSuccess) return pdm_cuda_fail(e, "gen_violation", __FILE__, __LINE__);
    unsigned long long vb = 0;
    std::vector<double> z((size_t)Gh.D.num_vars * Gh.D.num_dims);
    PDM_CUDA(cudaMemcpyAsync(&vb, Gh.d_viol, sizeof vb, cudaMemcpyDeviceToHost, h->stream));
    PDM_CUDA(cudaMemcpyAsync(z.data(), Gh.D.Z, sizeof(double) * z.size(), cudaMemcpyDeviceToHost, h->stream));
    PDM_CUDA(cudaStreamSynchronize(h->stream));
    memcpy(&out->max_violation, &vb, sizeof(double));
    double tot = 0;
    for (int v : Gh.radius_vars) tot += z[(size_t)v * Gh.D.num_dims];
    out->total_radius = Gh.radius_vars.empty() ? NAN : tot;
    out->converged = 0;
    out->status = PARADMM_OK;
    return PARADMM_OK;
}

extern "C" int paradmm_gpu_engine(const paradmm_gpu *h) { return h ? h->engine : PARADMM_EINVAL; }
extern "C" int paradmm_gpu_instances(const paradmm_gpu *h) { return !h ? 0 : (h->pk ? h->pk->n_inst : 1); }
extern "C" int64_t paradmm_gpu_device_bytes(const paradmm_gpu *h) { return h ? h->device_bytes : 0; }
extern "C" int64_t paradmm_gpu_launches(const paradmm_gpu *h) { return h ? h->launches : 0; }

extern "C" int paradmm_gpu_instance_times(const paradmm_gpu *h, double *begin_ms, double *end_ms)
{
    ok_status();
    if (!h || !h->pk || !begin_ms || !end_ms) return pdm_set_error(PARADMM_EINVAL, "needs a packing handle");
    const PkHost &P = *h->pk;
    if (P.schedule != PARADMM_SCHEDULE_INSTANCE && P.schedule != PARADMM_SCHEDULE_ONCHIP)
        return pdm_set_error(PARADMM_EINVAL, "instance times need a per-instance schedule");
    unsigned long long t0 = ~0ull;
    for (const PkStatus &s : P.status) if (s.t_begin_ns && s.t_begin_ns < t0) t0 = s.t_begin_ns;
    for (int i = 0; i < P.n_inst; ++i) {
        begin_ms[i] = P.status[i].t_begin_ns ? (double)(P.status[i].t_begin_ns - t0) * 1e-6 : NAN;
        end_ms[i] = P.status[i].t_end_ns ? (double)(P.status[i].t_end_ns - t0) * 1e-6 : NAN;
    }
    return PARADMM_OK;
}

extern "C" int paradmm_gpu_set_tail_handoff(paradmm_gpu *h, int instances)
{
    ok_status();
    if (!h || !h->pk) return pdm_set_error(PARADMM_EINVAL, "the tail hand-off needs a packing handle");
    if (instances < 0) return pdm_set_error(PARADMM_EINVAL, "instances < 0");
    if (h->pk->shard_n > 0) return pdm_set_error(PARADMM_EINVAL, "a shard of an instance has no per-instance schedule");
    h->pk->tail_yield = instances;
    return PARADMM_OK;
}

extern "C" int paradmm_gpu_tail_handoffs(const paradmm_gpu *h)
{
    return h && h->pk ? h->pk->yielded_last_call : 0;
}

extern "C" int paradmm_gpu_set_profiling(paradmm_gpu *h, int on)
{
    ok_status();
    if (!h || !h->pk) return pdm_set_error(PARADMM_EINVAL, "profiling needs a packing handle");
    h->pk->prof = on ? 1 : 0;
    return PARADMM_OK;
}

extern "C" int paradmm_gpu_phase_times(const paradmm_gpu *h, double out[4])
{
    ok_status();
    if (!h || !h->pk || !out) return pdm_set_error(PARADMM_EINVAL, "profiling needs a packing handle");
    for (int q = 0; q < 4; ++q) out[q] = h->pk->phase_us[q];
    return PARADMM_OK;
}

// ---- pinned host state (large graphs move through pinned pages) ----
static std::mutex g_pin_mu;
static std::unordered_map<const graph *, std::vector<void *>> g_pinned;

extern "C" int paradmm_gpu_pin_graph(const graph *G)
{
    ok_status();
    if (!G || !G->X || !G->M || !G->N || !G->U || !G->Z) return pdm_set_error(PARADMM_EINVAL, "graph state is not allocated");
    std::lock_guard<std::mutex> lk(g_pin_mu);
    if (g_pinned.count(G)) return PARADMM_OK;
    const size_t ne = (size_t)G->num_edges * G->num_dims * sizeof(double), nz = (size_t)G->num_vars * G->num_dims * sizeof(double);
    void *arrs[5] = {G->X, G->M, G->N, G->U, G->Z};
    const size_t sz[5] = {ne, ne, ne, ne, nz};
    std::vector<void *> done;
    for (int q = 0; q < 5; ++q) {
        cudaError_t e = cudaHostRegister(arrs[q], sz[q], cudaHostRegisterPortable);
        if (e != cudaSuccess) {
            for (void *p : done) cudaHostUnregister(p);
            return pdm_cuda_fail(e, "cudaHostRegister", __FILE__, __LINE__);
        }
        done.push_back(arrs[q]);
    }
    g_pinned[G] = done;
    return PARADMM_OK;
}

extern "C" int paradmm_gpu_unpin_graph(const graph *G)
{
    ok_status();
    std::lock_guard<std::mutex> lk(g_pin_mu);
    auto it = g_pinned.find(G);
    if (it == g_pinned.end()) return PARADMM_OK;
    for (void *p : it->second) cudaHostUnregister(p);
    g_pinned.erase(it);
    return PARADMM_OK;
}

extern "C" int paradmm_gpu_get_circles(paradmm_gpu *h, int instance, double *out)
{
    ok_status();
    if (!h || !out) return pdm_set_error(PARADMM_EINVAL, "NULL argument");
    if (!h->pk) return pdm_set_error(PARADMM_EINVAL, "not a packing handle");
    PkHost &P = *h->pk;
    if (instance < 0 || instance >= P.n_inst) return pdm_set_error(PARADMM_EINVAL, "instance %d out of range", instance);
    DevGuard guard(h->device);
    const PkInst &I = P.inst[instance];
    std::vector<double4> z(I.N);
    PDM_CUDA(cudaMemcpyAsync(z.data(), P.D.Z + I.circle_base, sizeof(double4) * I.N, cudaMemcpyDeviceToHost, h->stream));
    PDM_CUDA(cudaStreamSynchronize(h->stream));
    for (int c = 0; c < I.N; ++c) { out[3 * c] = z[c].x; out[3 * c + 1] = z[c].y; out[3 * c + 2] = z[c].z; }
    return PARADMM_OK;
}

// Device copy of n floats narrowed from host doubles (NULL in, NULL out).
static int upload_narrowed(paradmm_gpu *h, const double *src, size_t n, float **dst)
{
    *dst = nullptr;
    if (!src || n == 0) return PARADMM_OK;
    std::vector<float> f(n);
    for (size_t i = 0; i < n; ++i) f[i] = (float)src[i];
    PDM_CUDA(cudaMalloc((void **)dst, sizeof(float) * n));
    cudaError_t e = cudaMemcpyAsync(*dst, f.data(), sizeof(float) * n, cudaMemcpyHostToDevice, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) { cudaFree(*dst); *dst = nullptr; return pdm_cuda_fail(e, "cudaMemcpyAsync", __FILE__, __LINE__); }
    return PARADMM_OK;
}

static int pk_set_instance_circles(paradmm_gpu *h, int instance, const double *circles)
{
    PkHost &P = *h->pk;
    const PkInst &I = P.inst[instance];
    std::vector<double4> z(I.N);
    for (int c = 0; c < I.N; ++c) z[c] = make_double4(circles[3 * c], circles[3 * c + 1], circles[3 * c + 2], 0.0);
    PDM_CUDA(cudaMemcpyAsync(P.D.Z + I.circle_base, z.data(), sizeof(double4) * I.N, cudaMemcpyHostToDevice, h->stream));
    PDM_CUDA(cudaStreamSynchronize(h->stream));
    return PARADMM_OK;
}

extern "C" int paradmm_gpu_warm_start(paradmm_gpu *h, int instance, const double *circles, const float *pair_duals)
{
    ok_status();
    if (!h || !circles) return pdm_set_error(PARADMM_EINVAL, "NULL argument");
    if (!h->pk) return pdm_set_error(PARADMM_EINVAL, "not a packing handle");
    PkHost &P = *h->pk;
    if (instance < 0 || instance >= P.n_inst) return pdm_set_error(PARADMM_EINVAL, "instance %d out of range", instance);
    DevGuard guard(h->device);
    const PkInst &I = P.inst[instance];
    int rc = pk_set_instance_circles(h, instance, circles);
    if (rc) return rc;
    float *d_du = nullptr;
    const size_t nd = (size_t)I.N * (I.N - 1) / 2 * 6;
    if (pair_duals) {
        PDM_CUDA(cudaMalloc(&d_du, sizeof(float) * nd));
        cudaError_t e = cudaMemcpyAsync(d_du, pair_duals, sizeof(float) * nd, cudaMemcpyHostToDevice, h->stream);
        if (e != cudaSuccess) { cudaFree(d_du); return pdm_cuda_fail(e, "cudaMemcpyAsync", __FILE__, __LINE__); }
    }
    PkInitArgs A{};
    A.pair_duals = d_du;
    rc = pk_init_instance_state(h, instance, A);
    if (d_du) cudaFree(d_du);
    return rc;
}

extern "C" int paradmm_gpu_warm_start_duals(paradmm_gpu *h, int instance, const double *circles, const double *pair_duals,
                                           const double *wall_duals, const double *radius_duals, int dual_iters)
{
    ok_status();
    if (!h || !circles) return pdm_set_error(PARADMM_EINVAL, "NULL argument");
    if (!h->pk) return pdm_set_error(PARADMM_EINVAL, "not a packing handle");
    PkHost &P = *h->pk;
    if (instance < 0 || instance >= P.n_inst) return pdm_set_error(PARADMM_EINVAL, "instance %d out of range", instance);
    if (dual_iters < 0 || dual_iters > 100000) return pdm_set_error(PARADMM_EINVAL, "dual_iters %d out of [0, 100000]", dual_iters);
    DevGuard guard(h->device);
    const PkInst &I = P.inst[instance];
    // wall factors of the instance: those of its circles, contiguous
    const int w0 = P.circ[I.circle_base].wall_start;
    const int w1 = P.circ[I.circle_base + I.N - 1].wall_start + P.circ[I.circle_base + I.N - 1].wall_count;
    int rc = pk_set_instance_circles(h, instance, circles);
    if (rc) return rc;
    float *dp = nullptr, *dw = nullptr, *dr = nullptr;
    if ((rc = upload_narrowed(h, pair_duals, (size_t)I.N * (I.N - 1) / 2 * 6, &dp)) ||
        (rc = upload_narrowed(h, wall_duals, (size_t)(w1 - w0) * 3, &dw)) ||
        (rc = upload_narrowed(h, radius_duals, (size_t)I.N, &dr))) {
        cudaFree(dp); cudaFree(dw); cudaFree(dr);
        return rc;
    }
    PkInitArgs A{};
    A.pair_duals = dp;
    A.wall_duals = dw;
    A.rad_duals = dr;
    A.dual_iters = dual_iters;
    rc = pk_init_instance_state(h, instance, A);
    cudaFree(dp); cudaFree(dw); cudaFree(dr);
    return rc;
}

extern "C" int paradmm_gpu_warm_start_all(paradmm_gpu *h, const double *circles, int radius_duals)
{
    return paradmm_gpu_warm_start_all_duals(h, circles, radius_duals, 0);
}

extern "C" int paradmm_gpu_warm_start_all_duals(paradmm_gpu *h, const double *circles, int radius_duals, int dual_iters)
{
    ok_status();
    if (!h || !circles) return pdm_set_error(PARADMM_EINVAL, "NULL argument");
    if (!h->pk) return pdm_set_error(PARADMM_EINVAL, "not a packing handle");
    if (dual_iters < 0 || dual_iters > 100000) return pdm_set_error(PARADMM_EINVAL, "dual_iters %d out of [0, 100000]", dual_iters);
    PkHost &P = *h->pk;
    DevGuard guard(h->device);
    std::vector<double4> z(P.n_circ);
    for (int g = 0; g < P.n_circ; ++g) z[g] = make_double4(circles[3 * g], circles[3 * g + 1], circles[3 * g + 2], 0.0);
    PDM_CUDA(cudaMemcpyAsync(P.D.Z, z.data(), sizeof(double4) * P.n_circ, cudaMemcpyHostToDevice, h->stream));
    return pk_init_all(h, radius_duals, dual_iters);
}

// ---- schedule autotuner ----
// Device copies of the state a probe run changes.
struct PkSnapshot {
    std::vector<std::pair<void *, size_t>> buf;  // (source, bytes); copies in the same order
    std::vector<void *> copy;
    std::vector<int> nmode;
    std::vector<PkStatus> status;
    std::vector<long long> iters, upload_iter, age;
    long long it_next = 0;
};

static int pk_snapshot_take(paradmm_gpu *h, PkSnapshot &S)
{
    PkHost &P = *h->pk;
    S.buf = {{P.D.tiles, (size_t)(P.n_tiles * pk_tile_floats(P.BW) * 4LL)},
             {P.D.Z, sizeof(double4) * (size_t)P.n_circ},
             {P.D.Zp, sizeof(float4) * (size_t)P.n_circ},
             {P.D.wall_X, sizeof(float4) * (size_t)std::max(P.n_wall, 1)},
             {P.D.wall_U, sizeof(float4) * (size_t)std::max(P.n_wall, 1)},
             {P.D.rad_XU, sizeof(float2) * (size_t)std::max(P.n_rad, 1)}};
    for (auto &b : S.buf) {
        void *c = nullptr;
        cudaError_t e = cudaMalloc(&c, b.second);
        if (e != cudaSuccess) return pdm_cuda_fail(e, "cudaMalloc (autotune snapshot)", __FILE__, __LINE__);
        S.copy.push_back(c);
        PDM_CUDA(cudaMemcpyAsync(c, b.first, b.second, cudaMemcpyDeviceToDevice, h->stream));
    }
    S.nmode = P.nmode;
    S.status = P.status;
    S.iters = P.iters_last_call;
    S.upload_iter = P.upload_iter;
    S.age = P.age;
    S.it_next = P.it_next;
    PDM_CUDA(cudaStreamSynchronize(h->stream));
    return PARADMM_OK;
}

static int pk_snapshot_restore(paradmm_gpu *h, const PkSnapshot &S)
{
    PkHost &P = *h->pk;
    for (size_t q = 0; q < S.buf.size(); ++q)
        PDM_CUDA(cudaMemcpyAsync(S.buf[q].first, S.copy[q], S.buf[q].second, cudaMemcpyDeviceToDevice, h->stream));
    PDM_CUDA(cudaStreamSynchronize(h->stream));
    P.nmode = S.nmode;
    P.status = S.status;
    P.iters_last_call = S.iters;
    P.upload_iter = S.upload_iter;
    P.age = S.age;
    P.it_next = S.it_next;
    // the residual slots were not saved: no balancing decision may read the
    // sums of the sweeps before the restore
    for (int i = 0; i < P.n_inst; ++i) { P.last_swept[i] = -1; P.status[i].sd_valid = 0; }
    return PARADMM_OK;
}

static void pk_snapshot_free(PkSnapshot &S)
{
    for (void *c : S.copy) cudaFree(c);
    S.copy.clear();
}

extern "C" int paradmm_gpu_autotune(paradmm_gpu *h, int sweeps, double tol, paradmm_gpu_tuning *out)
{
    ok_status();
    if (!h || !h->pk) return pdm_set_error(PARADMM_EINVAL, "autotune needs a packing handle");
    if (h->pk->shard_n > 0) return pdm_set_error(PARADMM_EINVAL, "a shard of an instance has no schedule to tune");
    if (sweeps < 1) return pdm_set_error(PARADMM_EINVAL, "sweeps < 1");
    DevGuard guard(h->device);
    PkHost &P = *h->pk;
    int maxN = 0;
    for (const PkInst &I : P.inst) maxN = std::max(maxN, I.N);
    // candidates: (schedule, cluster, coop_min_n)
    struct Cand { int schedule, cluster, coop; double ms; };
    std::vector<Cand> cand;
    cand.push_back({PARADMM_SCHEDULE_GRID, 0, 0, 0});
    if (maxN <= 1024 && P.n_inst > 1) {
        cand.push_back({PARADMM_SCHEDULE_INSTANCE, 1, 0, 0});
        for (int cl : {2, 4})
            for (int coop : {120, 200, 300})
                if (maxN >= coop) cand.push_back({PARADMM_SCHEDULE_INSTANCE, cl, coop, 0});
        // the cluster-resident schedule only when the handle asked for it: on
        // batches it runs fewer instances at once and loses to the tiled one
        if (P.schedule == PARADMM_SCHEDULE_ONCHIP) cand.push_back({PARADMM_SCHEDULE_ONCHIP, 0, 0, 0});
    }
    const int saved_schedule = P.schedule, saved_cluster = P.cluster, saved_coop = P.coop_min_n;
    const int saved_fallback = P.fallback_after;
    P.fallback_after = 0;
    PkSnapshot snap;
    int rc = pk_snapshot_take(h, snap);
    int best = -1;
    for (size_t q = 0; rc == PARADMM_OK && q < cand.size(); ++q) {
        Cand &c = cand[q];
        P.schedule = c.schedule;
        if (c.schedule == PARADMM_SCHEDULE_INSTANCE) pk_set_instance_schedule(h, c.cluster, c.coop);
        if ((rc = pk_snapshot_restore(h, snap))) break;
        double ms = 0;
        rc = pk_run(h, sweeps, tol, h->opts.check_every, &ms);
        if (rc == PARADMM_ENONFINITE) rc = PARADMM_OK;  // timing only
        c.ms = ms;
        if (rc == PARADMM_OK && (best < 0 || ms < cand[best].ms)) best = (int)q;
    }
    int rc2 = snap.copy.size() == snap.buf.size() ? pk_snapshot_restore(h, snap) : PARADMM_OK;
    pk_snapshot_free(snap);
    P.fallback_after = saved_fallback;
    if (rc == PARADMM_OK) rc = rc2;
    if (rc != PARADMM_OK || best < 0) {
        P.schedule = saved_schedule;
        if (saved_schedule == PARADMM_SCHEDULE_INSTANCE) pk_set_instance_schedule(h, saved_cluster, saved_coop);
        return rc != PARADMM_OK ? rc : pdm_set_error(PARADMM_ECUDA, "autotune: no configuration ran");
    }
    const Cand &b = cand[best];
    P.schedule = b.schedule;
    if (b.schedule == PARADMM_SCHEDULE_INSTANCE) pk_set_instance_schedule(h, b.cluster, b.coop);
    if (out) {
        memset(out, 0, sizeof *out);
        out->schedule = P.schedule;
        out->cluster_size = P.schedule == PARADMM_SCHEDULE_INSTANCE ? P.cluster : 0;
        out->coop_min_n = P.schedule == PARADMM_SCHEDULE_INSTANCE ? P.coop_min_n : 0;
        out->ms = b.ms;
        out->candidates = (int)cand.size();
        double worst = 0;
        for (const Cand &c : cand) worst = std::max(worst, c.ms);
        out->worst_ms = worst;
    }
    return PARADMM_OK;
}

extern "C" int paradmm_gpu_create_packing_tuned(const paradmm_packing_desc *descs, int count,
                                                const paradmm_gpu_opts *opts, int sweeps, double tol,
                                                paradmm_gpu **out, paradmm_gpu_tuning *tuning)
{
    ok_status();
    if (!out) return pdm_set_error(PARADMM_EINVAL, "out is NULL");
    *out = nullptr;
    paradmm_gpu_opts o;
    if (opts) o = *opts;
    else paradmm_gpu_default_opts(&o);
    const int widths[2] = {64, 128};
    paradmm_gpu *best = nullptr;
    paradmm_gpu_tuning bt{};
    int rc = PARADMM_OK;
    for (int w : widths) {
        if (opts && opts->block_width && opts->block_width != w) continue;  // a fixed width is kept
        o.block_width = w;
        paradmm_gpu *h = nullptr;
        rc = paradmm_gpu_create_packing(descs, count, &o, &h);
        if (rc) break;
        paradmm_gpu_tuning t{};
        rc = paradmm_gpu_autotune(h, sweeps, tol, &t);
        if (rc) { paradmm_gpu_destroy(h); break; }
        if (!best || t.ms < bt.ms) {
            if (best) paradmm_gpu_destroy(best);
            best = h;
            bt = t;
            bt.block_width = w;
        } else {
            paradmm_gpu_destroy(h);
        }
    }
    if (rc) {
        if (best) paradmm_gpu_destroy(best);
        return rc;
    }
    if (!best) return pdm_set_error(PARADMM_EINVAL, "no block width to try (block_width must be 0, 64 or 128)");
    if (tuning) *tuning = bt;
    *out = best;
    return PARADMM_OK;
}

extern "C" int paradmm_gpu_set_rho_balance(paradmm_gpu *h, int period, double mu, int log2_min, int log2_max)
{
    ok_status();
    if (!h) return pdm_set_error(PARADMM_EINVAL, "handle is NULL");
    if (period != 0 && period < 3) return pdm_set_error(PARADMM_EINVAL, "period %d: 0 (off) or >= 3", period);
    if (!(mu >= 1.0) || !std::isfinite(mu)) return pdm_set_error(PARADMM_EINVAL, "mu must be finite and >= 1");
    if (log2_min > 0 || log2_max < 0 || log2_min < -30 || log2_max > 30)
        return pdm_set_error(PARADMM_EINVAL, "scale bounds 2^%d .. 2^%d must bracket 1, within 2^-30 .. 2^30", log2_min, log2_max);
    if (h->pk) {
        PkHost &P = *h->pk;
        P.bal_period = period;
        P.bal_mu = mu;
        P.bal_lmin = log2_min;
        P.bal_lmax = log2_max;
    } else if (h->gen) {
        GenHost &Gh = *h->gen;
        Gh.bal_period = period;
        Gh.bal_mu = mu;
        Gh.bal_lmin = log2_min;
        Gh.bal_lmax = log2_max;
    } else {
        return pdm_set_error(PARADMM_EINVAL, "handle has no engine");
    }
    return PARADMM_OK;
}

extern "C" int paradmm_gpu_rho_scale(const paradmm_gpu *h, int instance, int *log2_scale)
{
    ok_status();
    if (!h || !log2_scale) return pdm_set_error(PARADMM_EINVAL, "NULL argument");
    if (h->pk) {
        const PkHost &P = *h->pk;
        if (instance < 0 || instance >= P.n_inst) return pdm_set_error(PARADMM_EINVAL, "instance %d out of range", instance);
        const PkStatus &s = P.status[instance];
        // the scale the next sweep's radius operator uses
        const bool after = s.bal_pass_age > 0 && P.age[instance] + 1 >= s.bal_pass_age;
        *log2_scale = after ? s.bal_log2_new : s.bal_log2_cur;
    } else if (h->gen) {
        if (instance != 0) return pdm_set_error(PARADMM_EINVAL, "instance %d out of range", instance);
        *log2_scale = h->gen->bal_log2;
    } else {
        return pdm_set_error(PARADMM_EINVAL, "handle has no engine");
    }
    return PARADMM_OK;
}

extern "C" int paradmm_gpu_set_fallback(paradmm_gpu *h, int64_t after_sweeps)
{
    ok_status();
    if (!h) return pdm_set_error(PARADMM_EINVAL, "handle is NULL");
    if (!h->pk) return pdm_set_error(PARADMM_EINVAL, "not a packing handle");
    if (after_sweeps < 0 || after_sweeps > INT_MAX) return pdm_set_error(PARADMM_EINVAL, "after_sweeps out of range");
    if (after_sweeps > 0 && h->pk->schedule != PARADMM_SCHEDULE_INSTANCE && h->pk->schedule != PARADMM_SCHEDULE_ONCHIP)
        return pdm_set_error(PARADMM_EINVAL, "the in-call fallback needs a per-instance schedule");
    h->pk->fallback_after = (int)after_sweeps;
    return PARADMM_OK;
}

extern "C" int paradmm_gpu_instance_fallbacks(const paradmm_gpu *h, int *restarted)
{
    ok_status();
    if (!h || !restarted) return pdm_set_error(PARADMM_EINVAL, "NULL argument");
    if (!h->pk) return pdm_set_error(PARADMM_EINVAL, "not a packing handle");
    for (int i = 0; i < h->pk->n_inst; ++i) restarted[i] = h->pk->status[i].pad != 0;
    return PARADMM_OK;
}

// ===========================================================================
// One instance sharded over ranks
// ===========================================================================
// Pair count of circle-block row I (its tiles (I, J >= I)) plus its circles'
// wall and radius factors.
static long long shard_row_cost(int N, int BW, int I)
{
    const long long nI = std::min(BW, N - I * BW);
    const long long right = std::max(0LL, (long long)N - (long long)(I + 1) * BW);
    return nI * (nI - 1) / 2 + nI * right + nI;
}

extern "C" int paradmm_gpu_shard_rows(int n_circles, int block_width, int nranks, int *bounds)
{
    ok_status();
    if (!bounds) return pdm_set_error(PARADMM_EINVAL, "bounds is NULL");
    const int BW = block_width == 128 ? 128 : 64;
    if (block_width != 0 && block_width != 32 && block_width != 64 && block_width != 128)
        return pdm_set_error(PARADMM_EINVAL, "block_width %d (0, 64 or 128)", block_width);
    if (n_circles < 2 || n_circles > 32767) return pdm_set_error(PARADMM_EINVAL, "n_circles %d", n_circles);
    const int nb = (n_circles + BW - 1) / BW;
    if (nranks < 1 || nranks > nb)
        return pdm_set_error(PARADMM_EINVAL, "%d ranks for %d circle-block rows (at most one rank per row)", nranks, nb);
    std::vector<long long> cum(nb + 1, 0);
    for (int I = 0; I < nb; ++I) cum[I + 1] = cum[I] + shard_row_cost(n_circles, BW, I);
    bounds[0] = 0;
    for (int r = 1; r < nranks; ++r) {
        // the boundary whose prefix cost is nearest to r / nranks of the total,
        // leaving at least one row to every rank
        const double target = (double)cum[nb] * r / nranks;
        int best = bounds[r - 1] + 1;
        for (int I = best + 1; I <= nb - (nranks - r); ++I)
            if (std::fabs((double)cum[I] - target) < std::fabs((double)cum[best] - target)) best = I;
        bounds[r] = best;
    }
    bounds[nranks] = nb;
    return PARADMM_OK;
}

extern "C" int paradmm_gpu_create_packing_shard(const paradmm_packing_desc *desc, int rank, int nranks,
                                                const paradmm_gpu_opts *opts, paradmm_gpu **out)
{
    ok_status();
    if (!out) return pdm_set_error(PARADMM_EINVAL, "out is NULL");
    *out = nullptr;
    if (!desc) return pdm_set_error(PARADMM_EINVAL, "desc is NULL");
    const paradmm_packing_desc &d = *desc;
    if (d.n_circles < 2 || d.n_circles > 32767 || d.n_walls < 0 || d.n_walls > 8 || (d.n_walls && !d.walls) || !d.init)
        return pdm_set_error(PARADMM_EINVAL, "bad description (n_circles %d, n_walls %d)", d.n_circles, d.n_walls);
    if (!(d.rho > 0) || !(d.rho_radius > 0)) return pdm_set_error(PARADMM_EINVAL, "penalties must be positive");
    if (nranks < 1 || rank < 0 || rank >= nranks) return pdm_set_error(PARADMM_EINVAL, "rank %d of %d", rank, nranks);
    paradmm_gpu *h = new paradmm_gpu();
    int rc = handle_init(h, opts);
    if (rc) { free_handle_memory(h); delete h; return rc; }
    DevGuard g(h->device);
    if (h->opts.engine != PARADMM_ENGINE_AUTO && h->opts.engine != PARADMM_ENGINE_PACKING) {
        free_handle_memory(h); delete h;
        return pdm_set_error(PARADMM_EUNSUPPORTED_GRAPH, "structured packing problems run on the packing engine only");
    }
    h->engine = PARADMM_ENGINE_PACKING;
    h->pk = new PkHost();
    PkHost &P = *h->pk;
    P.V = pick_V(h->opts, d.n_circles);
    P.BW = 32 * P.V;
    P.stream_hint = true;
    P.dynamic = 1;
    std::vector<int> bounds(nranks + 1);
    rc = paradmm_gpu_shard_rows(d.n_circles, P.BW, nranks, bounds.data());
    if (rc == PARADMM_OK) {
        P.shard_n = nranks;
        P.shard_rank = rank;
        P.row_lo = bounds[rank];
        P.row_hi = bounds[rank + 1];
        pk_add_desc(P, d, 0);
        rc = pk_finalize_build(h);
    }
    if (rc == PARADMM_OK) {
        // the shard's pass is a plain launch (no grid barrier): as many CTAs as fit
        int bps = 0;
        if (pk_shard_prepare(P.V, P.stream_hint, &bps) != cudaSuccess || bps < 1)
            rc = pdm_set_error(PARADMM_ECUDA, "shard pass kernel cannot run on this device");
        else {
            if (h->opts.ctas_per_sm > 0) bps = std::min(bps, h->opts.ctas_per_sm);
            P.grid = std::max(1, std::min(h->num_sms * bps, P.n_items));
        }
    }
    if (rc == PARADMM_OK) rc = dalloc(h, (void **)&P.d_done, sizeof(unsigned));
    if (rc == PARADMM_OK && cudaMemset(P.d_done, 0, sizeof(unsigned)) != cudaSuccess)
        rc = pdm_set_error(PARADMM_ECUDA, "cudaMemset failed");
    P.use_graphs = 0;
    if (rc == PARADMM_OK) rc = pk_init_all(h, 0);
    if (rc) { free_handle_memory(h); delete h->pk; delete h; return rc; }
    h->num_dims = 2;
    *out = h;
    return PARADMM_OK;
}

static int shard_handle(paradmm_gpu *h, PkHost **P)
{
    if (!h) return pdm_set_error(PARADMM_EINVAL, "handle is NULL");
    if (!h->pk || h->pk->shard_n < 1) return pdm_set_error(PARADMM_EINVAL, "not a shard (paradmm_gpu_create_packing_shard)");
    *P = h->pk;
    return PARADMM_OK;
}

extern "C" int paradmm_gpu_shard_info(const paradmm_gpu *h, int *row_lo, int *row_hi, int64_t *exchange_bytes)
{
    ok_status();
    if (!h || !h->pk || h->pk->shard_n < 1) return pdm_set_error(PARADMM_EINVAL, "not a shard");
    if (row_lo) *row_lo = h->pk->row_lo;
    if (row_hi) *row_hi = h->pk->row_hi;
    if (exchange_bytes) *exchange_bytes = (int64_t)sizeof(double4) * h->pk->inst[0].N;
    return PARADMM_OK;
}

extern "C" int paradmm_gpu_shard_start(paradmm_gpu *h, int maxiter, double tol, int check_every)
{
    ok_status();
    PkHost *Pp;
    int rc = shard_handle(h, &Pp);
    if (rc) return rc;
    PkHost &P = *Pp;
    if (maxiter < 1) return pdm_set_error(PARADMM_EINVAL, "maxiter < 1");
    if (P.shard_running) return pdm_set_error(PARADMM_EINVAL, "a run is armed: paradmm_gpu_shard_finish first");
    DevGuard guard(h->device);
    const long long it0 = P.it_next;
    PkStatus s = P.status[0];
    s.last_iter = LLONG_MAX;
    s.check_from = it0 + 2;
    s.converged = 0;
    s.nonfinite = 0;
    s.nmode = P.nmode[0];
    s.mode_iter = it0;
    s.bal_base = it0 - P.age[0];
    s.bal_eval_from = std::max(s.bal_base + 2, P.last_swept[0] == it0 - 1 ? it0 : it0 + 2);
    PDM_CUDA(cudaMemcpyAsync(P.D.status, &s, sizeof s, cudaMemcpyHostToDevice, h->stream));
    DevCtl c{};
    c.n_active = 1;
    PDM_CUDA(cudaMemcpyAsync(h->ctl, &c, sizeof c, cudaMemcpyHostToDevice, h->stream));
    PDM_CUDA(cudaMemsetAsync(P.d_done, 0, sizeof(unsigned), h->stream));
    PDM_CUDA(cudaStreamSynchronize(h->stream));
    P.shard_it0 = it0;
    P.shard_k = it0;
    P.shard_stop = it0 + maxiter;
    P.shard_tol = tol;
    P.shard_check_every = check_every < 1 ? 1 : check_every;
    P.shard_phase = 0;
    P.shard_running = 1;
    P.iters_last_call[0] = 0;
    return PARADMM_OK;
}

extern "C" int paradmm_gpu_shard_begin(paradmm_gpu *h, void *exchange, void *stream)
{
    ok_status();
    PkHost *Pp;
    int rc = shard_handle(h, &Pp);
    if (rc) return rc;
    PkHost &P = *Pp;
    if (!P.shard_running || P.shard_phase != 0 || P.shard_k >= P.shard_stop)
        return pdm_set_error(PARADMM_EINVAL, "no sweep to begin (paradmm_gpu_shard_start / shard_end first)");
    if (!exchange || ((uintptr_t)exchange & 15u)) return pdm_set_error(PARADMM_EINVAL, "exchange must be a 16-byte aligned device buffer");
    DevGuard guard(h->device);
    PkRun R{};
    R.it0 = P.shard_k;
    R.n_iter = 1;
    R.dynamic = 1;
    R.tol = P.shard_tol;
    R.check_every = P.shard_check_every;
    R.bal_period = P.bal_period;
    R.bal_mu = P.bal_mu;
    R.bal_lmin = P.bal_lmin;
    R.bal_lmax = P.bal_lmax;
    R.bal_any = pk_bal_any(P);
    cudaStream_t s = (cudaStream_t)stream;
    cudaError_t e = pk_launch_shard_begin(P.V, P.stream_hint, P.D, R, P.grid, P.inst[0].nb, P.row_lo, P.row_hi,
                                          (double4 *)exchange, s);
    if (e != cudaSuccess) return pdm_cuda_fail(e, "shard pass launch", __FILE__, __LINE__);
    h->launches += 2;
    P.shard_phase = 1;
    return PARADMM_OK;
}

extern "C" int paradmm_gpu_shard_end(paradmm_gpu *h, const void *exchange, void *stream)
{
    ok_status();
    PkHost *Pp;
    int rc = shard_handle(h, &Pp);
    if (rc) return rc;
    PkHost &P = *Pp;
    if (!P.shard_running || P.shard_phase != 1) return pdm_set_error(PARADMM_EINVAL, "no sweep begun");
    if (!exchange || ((uintptr_t)exchange & 15u)) return pdm_set_error(PARADMM_EINVAL, "exchange must be a 16-byte aligned device buffer");
    DevGuard guard(h->device);
    PkRun R{};
    R.it0 = P.shard_it0;
    R.n_iter = (int)std::min<long long>(P.shard_stop - P.shard_it0, INT_MAX);
    R.dynamic = 1;
    R.tol = P.shard_tol;
    R.check_every = P.shard_check_every;
    R.bal_period = P.bal_period;
    R.bal_mu = P.bal_mu;
    R.bal_lmin = P.bal_lmin;
    R.bal_lmax = P.bal_lmax;
    R.bal_any = pk_bal_any(P);
    cudaStream_t s = (cudaStream_t)stream;
    cudaError_t e = pk_launch_shard_end(P.V, P.D, R, P.shard_k, P.inst[0].nb, (const double4 *)exchange, P.d_done, s);
    if (e != cudaSuccess) return pdm_cuda_fail(e, "shard consensus launch", __FILE__, __LINE__);
    ++h->launches;
    ++P.shard_k;
    P.shard_phase = 0;
    return PARADMM_OK;
}

extern "C" int paradmm_gpu_shard_poll(paradmm_gpu *h, void *stream, int *active)
{
    ok_status();
    PkHost *Pp;
    int rc = shard_handle(h, &Pp);
    if (rc) return rc;
    if (!active) return pdm_set_error(PARADMM_EINVAL, "active is NULL");
    DevGuard guard(h->device);
    PDM_CUDA(cudaStreamSynchronize((cudaStream_t)stream));
    DevCtl c{};
    PDM_CUDA(cudaMemcpyAsync(&c, h->ctl, sizeof c, cudaMemcpyDeviceToHost, h->stream));
    PDM_CUDA(cudaStreamSynchronize(h->stream));
    if (c.err != DEV_OK)
        return pdm_set_error(PARADMM_ETIMEOUT, "shard kernels: a device-side wait ran out (%s)", pdm_dev_err_name(c.err));
    *active = c.n_active > 0 && Pp->shard_k < Pp->shard_stop ? 1 : 0;
    return PARADMM_OK;
}

extern "C" int paradmm_gpu_shard_finish(paradmm_gpu *h, void *stream, paradmm_stats *stats)
{
    ok_status();
    PkHost *Pp;
    int rc = shard_handle(h, &Pp);
    if (rc) return rc;
    PkHost &P = *Pp;
    if (!P.shard_running) return pdm_set_error(PARADMM_EINVAL, "no run armed");
    if (P.shard_phase != 0) return pdm_set_error(PARADMM_EINVAL, "a sweep waits for its paradmm_gpu_shard_end");
    DevGuard guard(h->device);
    PDM_CUDA(cudaStreamSynchronize((cudaStream_t)stream));
    PkStatus st{};
    PDM_CUDA(cudaMemcpyAsync(&st, P.D.status, sizeof st, cudaMemcpyDeviceToHost, h->stream));
    PDM_CUDA(cudaStreamSynchronize(h->stream));
    const long long last = std::min(st.last_iter, P.shard_k - 1);
    P.iters_last_call[0] = std::max(0LL, last - P.shard_it0 + 1);
    P.nmode[0] = pk_pending_mode(st, last);
    P.status[0] = st;
    if (P.iters_last_call[0] > 0) { P.age[0] += P.iters_last_call[0]; P.last_swept[0] = last; }
    P.it_next = P.shard_k;
    P.shard_running = 0;
    rc = st.nonfinite ? pdm_set_error(PARADMM_ENONFINITE, "residual became NaN/Inf") : PARADMM_OK;
    if (stats) {
        memset(stats, 0, sizeof *stats);
        stats->iterations = P.iters_last_call[0];
        stats->converged = st.converged;
        stats->status = rc;
        stats->primal = st.primal;
        stats->dual = st.dual;
        stats->device_ms = NAN;
        stats->max_violation = NAN;
        stats->total_radius = NAN;
    }
    return rc;
}

extern "C" int paradmm_gpu_shard_fused_buffers(paradmm_gpu *h, void **exchange, void **flags)
{
    ok_status();
    PkHost *Pp;
    int rc = shard_handle(h, &Pp);
    if (rc) return rc;
    PkHost &P = *Pp;
    if (P.shard_n > PK_XCH_MAX) return pdm_set_error(PARADMM_EINVAL, "the fused exchange takes at most %d ranks", PK_XCH_MAX);
    DevGuard guard(h->device);
    if (!P.d_fx_exch) {
        const size_t nx = 2ull * (size_t)P.shard_n * (size_t)P.inst[0].N * sizeof(double4);
        if ((rc = dalloc(h, (void **)&P.d_fx_exch, nx))) return rc;
        if ((rc = dalloc(h, (void **)&P.d_fx_flags, sizeof(unsigned long long) * P.shard_n))) return rc;
        PDM_CUDA(cudaMemset(P.d_fx_exch, 0, nx));
        PDM_CUDA(cudaMemset(P.d_fx_flags, 0, sizeof(unsigned long long) * P.shard_n));
    }
    if (exchange) *exchange = P.d_fx_exch;
    if (flags) *flags = P.d_fx_flags;
    return PARADMM_OK;
}

extern "C" int paradmm_gpu_shard_run_fused(paradmm_gpu *const *hs, int nlocal, void *const *exchanges,
                                           void *const *flags, int wait_ms, void *stream)
{
    ok_status();
    if (!hs || nlocal < 1 || nlocal > PK_XCH_MAX) return pdm_set_error(PARADMM_EINVAL, "nlocal must be 1 .. %d", PK_XCH_MAX);
    if (!exchanges || !flags) return pdm_set_error(PARADMM_EINVAL, "exchanges and flags are required");
    PkHost *L[PK_XCH_MAX];
    for (int i = 0; i < nlocal; ++i) {
        int rc = shard_handle(hs[i], &L[i]);
        if (rc) return rc;
    }
    PkHost &P0 = *L[0];
    const int R = P0.shard_n, rank0 = P0.shard_rank;
    if (R > PK_XCH_MAX) return pdm_set_error(PARADMM_EINVAL, "the fused exchange takes at most %d ranks", PK_XCH_MAX);
    if (rank0 + nlocal > R) return pdm_set_error(PARADMM_EINVAL, "more local ranks than ranks");
    for (int i = 0; i < nlocal; ++i) {
        const PkHost &P = *L[i];
        if (hs[i]->device != hs[0]->device) return pdm_set_error(PARADMM_EINVAL, "the local ranks must share one device");
        if (P.shard_n != R || P.shard_rank != rank0 + i)
            return pdm_set_error(PARADMM_EINVAL, "local ranks must be consecutive shards of one split");
        if (P.V != P0.V || P.stream_hint != P0.stream_hint || P.inst[0].N != P0.inst[0].N)
            return pdm_set_error(PARADMM_EINVAL, "local ranks differ in instance or tile side");
        if (!P.shard_running || P.shard_phase != 0 || P.shard_k != P.shard_it0)
            return pdm_set_error(PARADMM_EINVAL, "each rank needs a fresh run (paradmm_gpu_shard_start) to fuse");
        if (P.shard_it0 != P0.shard_it0 || P.shard_stop != P0.shard_stop || P.shard_tol != P0.shard_tol ||
            P.shard_check_every != P0.shard_check_every || P.fx_epoch != P0.fx_epoch)
            return pdm_set_error(PARADMM_EINVAL, "local ranks are not at the same point of the same run");
    }
    PkXch X{};
    X.nranks = R;
    X.rank0 = rank0;
    X.nlocal = nlocal;
    X.epoch = P0.fx_epoch + 1;
    for (int q = 0; q < R; ++q) {
        if (!exchanges[q] || ((uintptr_t)exchanges[q] & 15u) || !flags[q] || ((uintptr_t)flags[q] & 7u))
            return pdm_set_error(PARADMM_EINVAL, "rank %d: exchange (16-byte) or flag (8-byte) buffer missing or misaligned", q);
        X.exch[q] = (double4 *)exchanges[q];
        X.flag[q] = (unsigned long long *)flags[q];
    }
    DevGuard guard(hs[0]->device);
    int bps = 0;
    cudaError_t e = pk_shard_fused_blocks(P0.V, P0.stream_hint, &bps);
    if (e != cudaSuccess || bps < 1) return pdm_cuda_fail(e != cudaSuccess ? e : cudaErrorInvalidConfiguration, "fused shard occupancy", __FILE__, __LINE__);
    X.blocks = bps * hs[0]->num_sms / nlocal;
    if (X.blocks < 1) return pdm_set_error(PARADMM_EINVAL, "too many local ranks for one device");
    PkDev devs[PK_XCH_MAX];
    for (int i = 0; i < nlocal; ++i) {
        devs[i] = L[i]->D;
        X.row_lo[i] = L[i]->row_lo;
        X.row_hi[i] = L[i]->row_hi;
    }
    int rc;
    if (!P0.d_fx_devs && (rc = dalloc(hs[0], (void **)&P0.d_fx_devs, sizeof(PkDev) * PK_XCH_MAX))) return rc;
    cudaStream_t s = stream ? (cudaStream_t)stream : hs[0]->stream;
    PDM_CUDA(cudaMemcpyAsync(P0.d_fx_devs, devs, sizeof(PkDev) * nlocal, cudaMemcpyHostToDevice, s));
    const unsigned long long lim = wait_ms > 0 ? (unsigned long long)wait_ms * 1000000ull : 0ull;
    for (int i = 0; i < nlocal; ++i)
        PDM_CUDA(cudaMemcpyAsync((char *)hs[i]->ctl + offsetof(DevCtl, timeout_ns), &lim, sizeof lim, cudaMemcpyHostToDevice, s));
    PkRun Rr{};
    Rr.it0 = P0.shard_k;
    Rr.n_iter = (int)std::min<long long>(P0.shard_stop - P0.shard_k, INT_MAX);
    Rr.dynamic = 1;
    Rr.tol = P0.shard_tol;
    Rr.check_every = P0.shard_check_every;
    Rr.bal_period = P0.bal_period;
    Rr.bal_mu = P0.bal_mu;
    Rr.bal_lmin = P0.bal_lmin;
    Rr.bal_lmax = P0.bal_lmax;
    Rr.bal_any = pk_bal_any(P0);
    e = pk_launch_shard_fused(P0.V, P0.stream_hint, P0.d_fx_devs, Rr, X, s);
    if (e != cudaSuccess) return pdm_cuda_fail(e, "fused shard launch", __FILE__, __LINE__);
    PDM_CUDA(cudaStreamSynchronize(s));
    rc = PARADMM_OK;
    for (int i = 0; i < nlocal; ++i) {
        PkHost &P = *L[i];
        DevCtl c{};
        PDM_CUDA(cudaMemcpy(&c, hs[i]->ctl, sizeof c, cudaMemcpyDeviceToHost));
        ++hs[i]->launches;
        P.fx_epoch = X.epoch;
        P.shard_k = P.shard_it0 + (long long)c.pad[0];
        if (c.err != DEV_OK && rc == PARADMM_OK)
            rc = pdm_set_error(PARADMM_ETIMEOUT, "fused shard kernel, rank %d: a device-side wait ran out (%s)",
                               P.shard_rank, pdm_dev_err_name(c.err));
    }
    return rc;
}

extern "C" int paradmm_gpu_ipc_export(const void *dev_ptr, void *handle)
{
    ok_status();
    if (!dev_ptr || !handle) return pdm_set_error(PARADMM_EINVAL, "dev_ptr and handle are required");
    cudaIpcMemHandle_t hd;
    PDM_CUDA(cudaIpcGetMemHandle(&hd, const_cast<void *>(dev_ptr)));
    memcpy(handle, &hd, sizeof hd);
    return PARADMM_OK;
}

extern "C" int paradmm_gpu_ipc_import(int device, const void *handle, void **dev_ptr)
{
    ok_status();
    if (!handle || !dev_ptr) return pdm_set_error(PARADMM_EINVAL, "handle and dev_ptr are required");
    DevGuard guard(device);
    cudaIpcMemHandle_t hd;
    memcpy(&hd, handle, sizeof hd);
    PDM_CUDA(cudaIpcOpenMemHandle(dev_ptr, hd, cudaIpcMemLazyEnablePeerAccess));
    return PARADMM_OK;
}

extern "C" int paradmm_gpu_ipc_close(int device, void *dev_ptr)
{
    ok_status();
    DevGuard guard(device);
    PDM_CUDA(cudaIpcCloseMemHandle(dev_ptr));
    return PARADMM_OK;
}

extern "C" void paradmm_gpu_destroy(paradmm_gpu *h)
{
    if (!h) return;
    {
        DevGuard guard(h->device);
        free_handle_memory(h);
    }
    delete h->pk;
    delete h->gen;
    delete h;
}

// ===========================================================================
// paradmm.h sweep functions (GPU-backed drop-ins)
// ===========================================================================
static std::mutex g_sweep_mu;
static paradmm_gpu_opts g_sweep_opts = {0, PARADMM_ENGINE_AUTO, 0, 0, 1, PARADMM_SCHEDULE_AUTO, 0, {0}};

struct Cached {
    paradmm_gpu *h = nullptr;
    int engine_req = 0;
    int num_opts = 0, num_vars = 0, num_edges = 0, num_dims = 0;
    const void *ptrs[4] = {nullptr, nullptr, nullptr, nullptr};
    uint64_t coef_hash = 0;
};
static std::unordered_map<const graph *, std::vector<Cached>> g_cache;

extern "C" void paradmm_set_sweep_options(const paradmm_gpu_opts *opts)
{
    std::lock_guard<std::mutex> lk(g_sweep_mu);
    if (opts) g_sweep_opts = *opts;
    else paradmm_gpu_default_opts(&g_sweep_opts);
}

// Fingerprint of the penalties and steps: a handle is reused only while they
// are unchanged (the packing engine folds them into constants).  Hashed in
// parallel chunks, combined in chunk order.
static uint64_t fnv_chunk(const double *a, size_t n)
{
    uint64_t h = 1469598103934665603ULL;
    for (size_t i = 0; i < n; ++i) {
        uint64_t b;
        memcpy(&b, &a[i], 8);
        h = (h ^ b) * 1099511628211ULL;
    }
    return h;
}

static uint64_t coef_hash(const graph *G)
{
    const size_t n = (size_t)G->num_edges;
    unsigned nt = std::thread::hardware_concurrency();
    nt = std::max(1u, std::min(nt, 32u));
    if (n < ((size_t)1 << 20)) nt = 1;
    std::vector<uint64_t> part(2 * nt, 0);
    auto work = [&](unsigned t) {
        const size_t b = n * t / nt, e = n * (t + 1) / nt;
        part[t] = G->RHOS ? fnv_chunk(G->RHOS + b, e - b) : 0;
        part[nt + t] = G->ALPHAS ? fnv_chunk(G->ALPHAS + b, e - b) : 0;
    };
    std::vector<std::thread> th;
    for (unsigned t = 1; t < nt; ++t) th.emplace_back(work, t);
    work(0);
    for (auto &x : th) x.join();
    uint64_t h = 1469598103934665603ULL;
    for (uint64_t v : part) h = (h ^ v) * 1099511628211ULL;
    return h;
}

extern "C" int paradmm_gpu_unpin_graph(const graph *G);

extern "C" void paradmm_internal_forget_graph(const graph *G)
{
    const int st = t_status;
    {
        std::lock_guard<std::mutex> lk(g_sweep_mu);
        auto it = g_cache.find(G);
        if (it != g_cache.end()) {
            for (Cached &c : it->second) paradmm_gpu_destroy(c.h);
            g_cache.erase(it);
        }
    }
    paradmm_gpu_unpin_graph(G);
    t_status = st;
}

// Handle for G with the requested engine; uploads G's current state.
static paradmm_gpu *sweep_handle(graph *G, int engine_req)
{
    paradmm_gpu_opts o = g_sweep_opts;
    if (engine_req >= 0) o.engine = engine_req;
    const uint64_t hh = coef_hash(G);
    std::vector<Cached> &v = g_cache[G];
    for (auto it = v.begin(); it != v.end(); ++it) {
        if (it->engine_req != o.engine) continue;
        const bool same = it->num_opts == G->num_opts && it->num_vars == G->num_vars && it->num_edges == G->num_edges &&
                          it->num_dims == G->num_dims && it->ptrs[0] == (const void *)G->operatorix_to_edgelistix &&
                          it->ptrs[1] == (const void *)G->edgeix_to_varlistix &&
                          it->ptrs[2] == (const void *)G->list_of_operators_functions_pointers &&
                          it->ptrs[3] == (const void *)G->varix_to_edgelistix && it->coef_hash == hh;
        if (same) {
            if (paradmm_gpu_upload(it->h, G) == PARADMM_OK) return it->h;
            if (paradmm_last_status() != PARADMM_EUNSUPPORTED_GRAPH) return nullptr;
        }
        paradmm_gpu_destroy(it->h);
        v.erase(it);
        break;
    }
    paradmm_gpu *h = nullptr;
    if (paradmm_gpu_create(G, &o, &h) != PARADMM_OK) {
        // a packing-eligible topology whose state cannot be kept compact
        if (o.engine == PARADMM_ENGINE_AUTO && paradmm_last_status() == PARADMM_EUNSUPPORTED_GRAPH) {
            o.engine = PARADMM_ENGINE_GENERIC_F64;
            if (paradmm_gpu_create(G, &o, &h) != PARADMM_OK) return nullptr;
        } else {
            return nullptr;
        }
    }
    Cached c;
    c.h = h;
    c.engine_req = engine_req >= 0 ? engine_req : g_sweep_opts.engine;
    c.num_opts = G->num_opts; c.num_vars = G->num_vars; c.num_edges = G->num_edges; c.num_dims = G->num_dims;
    c.ptrs[0] = G->operatorix_to_edgelistix; c.ptrs[1] = G->edgeix_to_varlistix;
    c.ptrs[2] = G->list_of_operators_functions_pointers; c.ptrs[3] = G->varix_to_edgelistix;
    c.coef_hash = hh;
    v.push_back(c);
    return h;
}

// One reference phase (or a whole sweep) on the GPU: upload, run, download.
static void sweep_call(graph *G, int phase, int iters)
{
    std::lock_guard<std::mutex> lk(g_sweep_mu);
    ok_status();
    const int engine_req = phase < 0 ? -1 : PARADMM_ENGINE_GENERIC_F64;
    paradmm_gpu *h = sweep_handle(G, engine_req);
    if (!h) return;
    DevGuard guard(h->device);
    // Graphs with large state move it through pinned pages (registered once,
    // released by closeG).
    if ((size_t)G->num_edges * G->num_dims * sizeof(double) >= ((size_t)64 << 20)) {
        if (paradmm_gpu_pin_graph(G) != PARADMM_OK) ok_status();  // pageable copies still work
    }
    int rc;
    if (phase < 0) rc = paradmm_gpu_iterate(h, iters);
    else rc = gen_phase(h, phase);
    if (rc == PARADMM_OK) rc = paradmm_gpu_download(h, G);
    (void)rc;
}

extern "C" void updateXM(graph *G) { sweep_call(G, GEN_PHASE_XM, 1); }
extern "C" void updateX(graph *G) { sweep_call(G, GEN_PHASE_X, 1); }
extern "C" void updateM(graph *G) { sweep_call(G, GEN_PHASE_M, 1); }
extern "C" void updateZ(graph *G) { sweep_call(G, GEN_PHASE_Z, 1); }
extern "C" void updateUN(graph *G) { sweep_call(G, GEN_PHASE_UN, 1); }
extern "C" void updateU(graph *G) { sweep_call(G, GEN_PHASE_U, 1); }
extern "C" void updateN(graph *G) { sweep_call(G, GEN_PHASE_N, 1); }
extern "C" void updateG(graph *G) { sweep_call(G, -1, 1); }
extern "C" void update_outgoing_rhos(graph *G) { (void)G; }  // a no-op in the reference too (core/paradmm.c:564-566)
extern "C" void updateXOpenMP(graph *G) { updateX(G); }
extern "C" void updateMOpenMP(graph *G) { updateM(G); }
extern "C" void updateZOpenMP(graph *G) { updateZ(G); }
extern "C" void updateUOpenMP(graph *G) { updateU(G); }
extern "C" void updateNOpenMP(graph *G) { updateN(G); }
extern "C" void updateGOpenMP(graph *G, int maxiter, int numthreads)
{
    (void)numthreads;
    if (maxiter <= 0) return;
    sweep_call(G, -1, maxiter);
}

// ===========================================================================
// Failure detection self-test: a grid barrier one block never reaches.
// ===========================================================================
__global__ void pdm_barrier_probe(DevCtl *ctl)
{
    if (blockIdx.x == gridDim.x - 1) return;  // this block never arrives
    grid_barrier(ctl);
}

extern "C" int paradmm_gpu_selftest_barrier_timeout(int device, int timeout_ms)
{
    ok_status();
    if (timeout_ms < 1 || timeout_ms > 10000) return pdm_set_error(PARADMM_EINVAL, "timeout_ms must be in [1, 10000]");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev)
        return pdm_set_error(PARADMM_ENODEVICE, "no CUDA device %d", device);
    DevGuard guard(device);
    DevCtl *d = nullptr;
    PDM_CUDA(cudaMalloc(&d, sizeof(DevCtl)));
    DevCtl c{};
    c.timeout_ns = (unsigned long long)timeout_ms * 1000000ull;
    cudaError_t e = cudaMemcpy(d, &c, sizeof c, cudaMemcpyHostToDevice);
    void *args[] = {(void *)&d};
    if (e == cudaSuccess) e = cudaLaunchCooperativeKernel((const void *)pdm_barrier_probe, dim3(2), dim3(32), args, 0, 0);
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e == cudaSuccess) e = cudaMemcpy(&c, d, sizeof c, cudaMemcpyDeviceToHost);
    cudaFree(d);
    if (e != cudaSuccess) return pdm_cuda_fail(e, "barrier self-test", __FILE__, __LINE__);
    if (c.err == DEV_BARRIER_TIMEOUT)
        return pdm_set_error(PARADMM_ETIMEOUT, "grid barrier wait ran out after %d ms (self-test: one block never arrives)",
                             timeout_ms);
    return pdm_set_error(PARADMM_ECUDA, "barrier self-test: the missing block was not detected (device error %d)", c.err);
}
