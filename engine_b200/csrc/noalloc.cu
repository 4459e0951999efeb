// Allocation-free entry point: fused packing sweeps whose scratch lives in a
// fixed device array of this library, for callers that cannot allocate
// device memory (see paradmm_gpu.h, paradmm_gpu_packing_iterate_noalloc).
//
// It runs the same persistent sweep kernel (pk_persistent) as the handle
// API; only where its scratch lives differs.  Scratch = per-instance tables,
// work items, the tile row/column partial sums of the consensus, residual
// partials, run status and the grid-barrier control block.  The caller owns
// the inputs/outputs: the consensus circles and the edge-state buffer.
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <chrono>
#include <climits>
#include <cmath>
#include <mutex>

#include "engine_internal.h"
#include "packing_launch.h"
#include "paradmm_gpu.h"

// Fixed limits of the allocation-free path (block width 64, one instance).
#define NA_V 2
#define NA_BW 64
#define NA_MAX_CIRCLES PARADMM_NOALLOC_MAX_CIRCLES
#define NA_MAX_WALLS PARADMM_NOALLOC_MAX_WALLS
#define NA_NB ((NA_MAX_CIRCLES + NA_BW - 1) / NA_BW)
#define NA_TILES (NA_NB * (NA_NB + 1) / 2)
#define NA_ITEMS (NA_TILES + (NA_MAX_CIRCLES + PK_THREADS - 1) / PK_THREADS)
#define NA_WALLS (NA_MAX_CIRCLES * NA_MAX_WALLS)
// Tag in the state header of a buffer this entry point has initialised.
#define NA_STATE_TAG 0x5044414e

static constexpr size_t na_al(size_t x) { return (x + 255) & ~(size_t)255; }

// Byte offsets of each table inside the scratch array.
struct NaLayout {
    static constexpr size_t inst = 0;
    static constexpr size_t items = inst + na_al(sizeof(PkInst));
    static constexpr size_t claim = items + na_al(sizeof(int4) * NA_ITEMS);
    static constexpr size_t circ = claim + na_al(sizeof(int) * NA_ITEMS);
    static constexpr size_t row_part = circ + na_al(sizeof(PkCircle) * NA_MAX_CIRCLES);
    static constexpr size_t col_part = row_part + na_al(sizeof(double4) * NA_TILES * NA_BW);
    static constexpr size_t Z = col_part + na_al(sizeof(double4) * NA_TILES * NA_BW);
    static constexpr size_t local_part = Z + na_al(sizeof(double4) * NA_MAX_CIRCLES);
    static constexpr size_t fin_items = local_part + na_al(sizeof(double4) * NA_MAX_CIRCLES);
    static constexpr size_t blk_primal = fin_items + na_al(sizeof(int2) * NA_NB);
    static constexpr size_t blk_dual = blk_primal + na_al(sizeof(double) * 4 * NA_NB);
    static constexpr size_t status = blk_dual + na_al(sizeof(double) * 4 * NA_NB);
    static constexpr size_t wall_vp = status + na_al(sizeof(PkStatus));
    static constexpr size_t wall_coef = wall_vp + na_al(sizeof(float4) * NA_WALLS);
    static constexpr size_t wall_rho = wall_coef + na_al(sizeof(float4) * NA_WALLS);
    static constexpr size_t rad_coef = wall_rho + na_al(sizeof(double2) * NA_WALLS);
    static constexpr size_t rad_rho = rad_coef + na_al(sizeof(float4) * NA_MAX_CIRCLES);
    static constexpr size_t ctl = rad_rho + na_al(sizeof(double) * NA_MAX_CIRCLES);
    static constexpr size_t total = ctl + na_al(sizeof(DevCtl));
};
static_assert(NaLayout::total <= PARADMM_NOALLOC_SCRATCH_BYTES, "scratch array too small for its limits");

// The scratch itself: one copy per device that loads this library, held
// until the process exits.  Host code must not use this name as a pointer
// (it is a host-side stand-in); it asks cudaGetSymbolAddress for the device
// address once per device.
static __device__ __align__(256) unsigned char g_noalloc_scratch[PARADMM_NOALLOC_SCRATCH_BYTES];

#define NA_MAX_DEVICES 64
static std::mutex g_na_mu;
static unsigned char *g_na_ptr[NA_MAX_DEVICES];  // device address of the scratch, per device
static int g_na_grid[NA_MAX_DEVICES];

// Host staging of the tables (fixed size: no host allocation either).
static PkInst s_inst;
static int4 s_items[NA_ITEMS];
static int s_claim[NA_ITEMS];
static int2 s_fin[NA_NB];
static PkCircle s_circ[NA_MAX_CIRCLES];
static float4 s_wall_vp[NA_WALLS], s_wall_coef[NA_WALLS];
static double2 s_wall_rho[NA_WALLS];
static float4 s_rad_coef[NA_MAX_CIRCLES];
static double s_rad_rho[NA_MAX_CIRCLES];
static PkStatus s_status;
static DevCtl s_ctl;

static int64_t na_tiles_of(int n)
{
    const int nb = (n + NA_BW - 1) / NA_BW;
    return (int64_t)nb * (nb + 1) / 2;
}

// Radius (X, U) pairs of n circles, padded so the FP32 circles after them
// start on a 16-byte boundary.
static int64_t na_rad_bytes(int n) { return ((int64_t)n * (int64_t)sizeof(float2) + 15) & ~(int64_t)15; }

extern "C" int64_t paradmm_noalloc_state_bytes(int n_circles, int n_walls)
{
    if (n_circles < 2 || n_circles > NA_MAX_CIRCLES || n_walls < 0 || n_walls > NA_MAX_WALLS) return -1;
    return na_tiles_of(n_circles) * pk_tile_floats(NA_BW) * 4 + (int64_t)n_circles * n_walls * 2 * sizeof(float4) +
           na_rad_bytes(n_circles) + (int64_t)n_circles * sizeof(float4) + 16;
}

// Per-device set-up: the scratch's device address (cudaGetSymbolAddress with
// the device current) and the cooperative grid size.
static int na_setup(int device)
{
    if (g_na_ptr[device]) return PARADMM_OK;
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return pdm_cuda_fail(e, "cudaGetSymbolAddress(noalloc scratch)", __FILE__, __LINE__);
    int sms = 0, bps = 0;
    PDM_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    e = pk_max_blocks_per_sm(NA_V, true, &bps);
    if (e != cudaSuccess || bps < 1) return pdm_set_error(PARADMM_ECUDA, "packing kernel cannot be resident on device %d", device);
    g_na_grid[device] = sms * bps;
    g_na_ptr[device] = (unsigned char *)p;
    return PARADMM_OK;
}

// Host tables of one instance (same content as the handle path builds).
static void na_tables(const paradmm_packing_desc &d, int *n_items_out)
{
    const int N = d.n_circles;
    PkInst &I = s_inst;
    memset(&I, 0, sizeof I);
    I.N = N;
    I.nb = (N + NA_BW - 1) / NA_BW;
    const double rho[4] = {d.rho, d.rho, d.rho, d.rho}, al[4] = {d.alpha, d.alpha, d.alpha, d.alpha};
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
        for (int q = 0; q < 4; ++q) { I.rho[q] = rho[q]; I.alpha[q] = (float)al[q]; }
    }
    const long long E = (long long)N + 2LL * d.n_walls * N + 4LL * N * (N - 1) / 2;
    I.inv_ncomp = 1.0 / (2.0 * (double)E);
    int nw = 0;
    for (int c = 0; c < N; ++c) {
        PkCircle &C = s_circ[c];
        memset(&C, 0, sizeof C);
        C.inv_rho_c = 1.0 / (d.rho * (N - 1) + d.rho * d.n_walls);
        C.inv_rho_r = 1.0 / (d.rho * (N - 1) + d.rho * d.n_walls + d.rho_radius);
        C.w_c = (N - 1) + d.n_walls;
        C.w_r = 2.0 * ((N - 1) + d.n_walls + 1);
        C.wall_start = nw;
        C.wall_count = d.n_walls;
        for (int w = 0; w < d.n_walls; ++w, ++nw) {
            const double *W = d.walls + 4 * w;
            s_wall_vp[nw] = make_float4((float)W[0], (float)W[1], (float)W[2], (float)W[3]);
            s_wall_coef[nw] = make_float4((float)d.rho, (float)d.rho, (float)d.alpha, (float)d.alpha);
            s_wall_rho[nw] = make_double2(d.rho, d.rho);
        }
        C.rad_start = c;
        C.rad_count = 1;
        s_rad_coef[c] = make_float4((float)d.exponent, (float)d.rho_radius, (float)d.alpha, 0.f);
        s_rad_rho[c] = d.rho_radius;
        C.inst = 0;
    }
    int n = 0;
    for (int a = 0; a < I.nb; ++a)
        for (int b = a; b < I.nb; ++b) s_items[n++] = make_int4(0, 0, a, b);
    for (int c0 = 0; c0 < N; c0 += PK_THREADS) s_items[n++] = make_int4(0, 1, c0, std::min(PK_THREADS, N - c0));
    I.item_base = 0;
    I.n_items = n;
    I.fin_base = 0;
    for (int b = 0; b < I.nb; ++b) s_fin[b] = make_int2(0, b);
    for (int q = 0; q < n; ++q) s_claim[q] = q;  // tiles come first: largest first already
    *n_items_out = n;
}

extern "C" int paradmm_gpu_packing_iterate_noalloc(const paradmm_packing_desc *desc, double *d_circles, void *d_state,
                                                   int init_state, int sweeps, double tol, paradmm_stats *stats,
                                                   int device, void *stream)
{
    pdm_clear_status();
    if (stats) memset(stats, 0, sizeof *stats);
    if (!desc || !d_circles || !d_state) return pdm_set_error(PARADMM_EINVAL, "noalloc: NULL argument");
    const paradmm_packing_desc &d = *desc;
    if (d.n_circles < 2 || d.n_circles > NA_MAX_CIRCLES)
        return pdm_set_error(PARADMM_EINVAL, "noalloc: %d circles is outside [2, %d], the limit of the fixed scratch",
                             d.n_circles, NA_MAX_CIRCLES);
    if (d.n_walls < 0 || d.n_walls > NA_MAX_WALLS || (d.n_walls && !d.walls))
        return pdm_set_error(PARADMM_EINVAL, "noalloc: %d walls is outside [0, %d]", d.n_walls, NA_MAX_WALLS);
    if (!(d.rho > 0) || !(d.rho_radius > 0)) return pdm_set_error(PARADMM_EINVAL, "noalloc: penalties must be positive");
    if (sweeps < 0) return pdm_set_error(PARADMM_EINVAL, "noalloc: sweeps < 0");
    if (((uintptr_t)d_state & 15u) || ((uintptr_t)d_circles & 7u))
        return pdm_set_error(PARADMM_EINVAL, "noalloc: d_state must be 16-byte and d_circles 8-byte aligned");
    if (device < 0 || device >= NA_MAX_DEVICES) return pdm_set_error(PARADMM_ENODEVICE, "noalloc: bad device %d", device);
    std::lock_guard<std::mutex> lk(g_na_mu);
    int prev = -1;
    cudaGetDevice(&prev);
    if (prev != device) PDM_CUDA(cudaSetDevice(device));
    struct Restore {
        int prev, dev;
        ~Restore() { if (prev >= 0 && prev != dev) cudaSetDevice(prev); }
    } restore{prev, device};
    int rc = na_setup(device);
    if (rc) return rc;
    cudaStream_t s = (cudaStream_t)stream;
    unsigned char *base = g_na_ptr[device];
    const int N = d.n_circles;

    int n_items = 0;
    na_tables(d, &n_items);
    PkDev D{};
    D.inst = (const PkInst *)(base + NaLayout::inst);
    D.items = (const int4 *)(base + NaLayout::items);
    D.claim = (const int *)(base + NaLayout::claim);
    D.circ = (const PkCircle *)(base + NaLayout::circ);
    D.n_inst = 1;
    D.n_items = n_items;
    D.n_claim = n_items;
    D.n_circ = N;
    D.row_part = (double4 *)(base + NaLayout::row_part);
    D.col_part = (double4 *)(base + NaLayout::col_part);
    D.Z = (double4 *)(base + NaLayout::Z);
    D.local_part = (double4 *)(base + NaLayout::local_part);
    D.fin_items = (const int2 *)(base + NaLayout::fin_items);
    D.n_fin = s_inst.nb;
    D.n_finl = s_inst.nb;
    D.blk_primal = (double *)(base + NaLayout::blk_primal);
    D.blk_dual = (double *)(base + NaLayout::blk_dual);
    D.status = (PkStatus *)(base + NaLayout::status);
    D.wall_vp = (const float4 *)(base + NaLayout::wall_vp);
    D.wall_coef = (const float4 *)(base + NaLayout::wall_coef);
    D.wall_rho = (const double2 *)(base + NaLayout::wall_rho);
    D.rad_coef = (const float4 *)(base + NaLayout::rad_coef);
    D.rad_rho = (const double *)(base + NaLayout::rad_rho);
    D.ctl = (DevCtl *)(base + NaLayout::ctl);
    // caller-owned edge state: pair tiles (U), wall X, wall U, radius (X, U),
    // the previous sweep's circles (FP32) and a 16-byte header holding the
    // first-sweep mode the state owes its next sweep
    const int64_t tile_bytes = na_tiles_of(N) * pk_tile_floats(NA_BW) * 4;
    const int nwall = N * d.n_walls;
    D.tiles = (float *)d_state;
    D.wall_X = (float4 *)((char *)d_state + tile_bytes);
    D.wall_U = D.wall_X + nwall;
    D.rad_XU = (float2 *)(D.wall_U + nwall);
    D.Zp = (float4 *)((char *)D.rad_XU + na_rad_bytes(N));
    int *d_mode = (int *)(D.Zp + N);

    // Tables into the scratch; residual partials start at zero (the array
    // keeps whatever the previous call left).
    PDM_CUDA(cudaMemcpyAsync((void *)D.inst, &s_inst, sizeof s_inst, cudaMemcpyHostToDevice, s));
    PDM_CUDA(cudaMemcpyAsync((void *)D.items, s_items, sizeof(int4) * n_items, cudaMemcpyHostToDevice, s));
    PDM_CUDA(cudaMemcpyAsync((void *)D.claim, s_claim, sizeof(int) * n_items, cudaMemcpyHostToDevice, s));
    PDM_CUDA(cudaMemcpyAsync((void *)D.circ, s_circ, sizeof(PkCircle) * N, cudaMemcpyHostToDevice, s));
    if (nwall) {
        PDM_CUDA(cudaMemcpyAsync((void *)D.wall_vp, s_wall_vp, sizeof(float4) * nwall, cudaMemcpyHostToDevice, s));
        PDM_CUDA(cudaMemcpyAsync((void *)D.wall_coef, s_wall_coef, sizeof(float4) * nwall, cudaMemcpyHostToDevice, s));
        PDM_CUDA(cudaMemcpyAsync((void *)D.wall_rho, s_wall_rho, sizeof(double2) * nwall, cudaMemcpyHostToDevice, s));
    }
    PDM_CUDA(cudaMemcpyAsync((void *)D.rad_coef, s_rad_coef, sizeof(float4) * N, cudaMemcpyHostToDevice, s));
    PDM_CUDA(cudaMemcpyAsync((void *)D.rad_rho, s_rad_rho, sizeof(double) * N, cudaMemcpyHostToDevice, s));
    PDM_CUDA(cudaMemcpyAsync((void *)D.fin_items, s_fin, sizeof(int2) * s_inst.nb, cudaMemcpyHostToDevice, s));
    PDM_CUDA(cudaMemsetAsync(D.blk_primal, 0, sizeof(double) * 4 * s_inst.nb, s));
    PDM_CUDA(cudaMemsetAsync(D.blk_dual, 0, sizeof(double) * 4 * s_inst.nb, s));
    // consensus: caller's [cx, cy, r] rows -> the kernel's (cx, cy, r, -) rows
    PDM_CUDA(cudaMemcpy2DAsync(D.Z, sizeof(double4), d_circles, 3 * sizeof(double), 3 * sizeof(double), N,
                               cudaMemcpyDeviceToDevice, s));
    // State header (16 bytes after the FP32 circles): {mode, tag, 0, 0}.  The
    // tag marks a buffer this entry point initialised; a zero-filled or
    // foreign buffer has none and is refused when init_state = 0.  Any error
    // after the state may have changed clears the tag, so a later call must
    // start again with init_state = 1 rather than resume from a state whose
    // circles and mode no longer agree.
    static int s_hdr[4];
    auto invalidate = [&]() {
        static int zero[4] = {0, 0, 0, 0};
        cudaGetLastError();
        if (cudaMemcpyAsync(d_mode, zero, sizeof zero, cudaMemcpyHostToDevice, s) == cudaSuccess) cudaStreamSynchronize(s);
    };
    int s_mode;
    if (init_state) {
        cudaError_t e = pk_launch_init(NA_V, D, 0, PkInitArgs{}, g_na_grid[device], s);
        if (e != cudaSuccess) { invalidate(); return pdm_cuda_fail(e, "noalloc init", __FILE__, __LINE__); }
        s_mode = PK_MODE_Z;
    } else {
        PDM_CUDA(cudaMemcpyAsync(s_hdr, d_mode, sizeof s_hdr, cudaMemcpyDeviceToHost, s));
        PDM_CUDA(cudaStreamSynchronize(s));
        s_mode = s_hdr[0];
        if (s_hdr[1] != NA_STATE_TAG || s_mode < PK_MODE_RECOMPUTE || s_mode > PK_MODE_XN)
            return pdm_set_error(PARADMM_EINVAL, "noalloc: the state buffer was never initialised (call with init_state = 1)");
    }

    const auto t0 = std::chrono::steady_clock::now();
    long long done = 0;
    int status_rc = PARADMM_OK;
    long long left = sweeps;
    long long it0 = 0;
    while (left > 0) {
        const int chunk = (int)std::min<long long>(left, 8192);
        memset(&s_status, 0, sizeof s_status);
        s_status.last_iter = LLONG_MAX;
        s_status.check_from = it0 + 2;
        s_status.resid_iter = -1;
        s_status.primal = s_status.dual = NAN;
        s_status.nmode = s_mode;
        s_status.mode_iter = it0;
        memset(&s_ctl, 0, sizeof s_ctl);
        s_ctl.n_active = 1;
        cudaError_t e = cudaMemcpyAsync(D.status, &s_status, sizeof s_status, cudaMemcpyHostToDevice, s);
        if (e == cudaSuccess) e = cudaMemcpyAsync(D.ctl, &s_ctl, sizeof s_ctl, cudaMemcpyHostToDevice, s);
        PkRun R{};
        R.it0 = it0;
        R.n_iter = chunk;
        R.dynamic = 1;
        R.tol = tol;
        R.check_every = 1;
        R.prof = 0;
        if (e == cudaSuccess) e = pk_launch_persistent(NA_V, true, D, R, g_na_grid[device], s);
        if (e == cudaSuccess) e = cudaMemcpyAsync(&s_ctl, D.ctl, sizeof s_ctl, cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaMemcpyAsync(&s_status, D.status, sizeof s_status, cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) { invalidate(); return pdm_cuda_fail(e, "noalloc persistent launch", __FILE__, __LINE__); }
        if (s_ctl.err != DEV_OK) {
            invalidate();
            return pdm_set_error(PARADMM_ETIMEOUT, "noalloc: a device-side wait ran out (%s)", pdm_dev_err_name(s_ctl.err));
        }
        const long long last = std::min<long long>(s_status.last_iter, it0 + s_ctl.pad[0] - 1);
        const long long ran = last - it0 + 1;
        done += ran;
        if (last < s_status.mode_iter) s_mode = s_status.nmode;
        else if (last == s_status.mode_iter && s_status.nmode == PK_MODE_N) s_mode = PK_MODE_XN;
        else s_mode = PK_MODE_RECOMPUTE;
        it0 += s_ctl.pad[0];
        left -= s_ctl.pad[0];
        if (s_status.nonfinite) { status_rc = pdm_set_error(PARADMM_ENONFINITE, "noalloc: residual became NaN/Inf"); break; }
        if (s_status.converged || (long long)s_ctl.pad[0] < chunk) break;
    }
    // consensus back to the caller's rows; the mode and the tag into the
    // state header (a NaN/Inf stop leaves a consistent state: the circles and
    // the mode of the sweeps that ran)
    s_hdr[0] = s_mode;
    s_hdr[1] = NA_STATE_TAG;
    s_hdr[2] = s_hdr[3] = 0;
    cudaError_t e = cudaMemcpy2DAsync(d_circles, 3 * sizeof(double), D.Z, sizeof(double4), 3 * sizeof(double), N,
                                      cudaMemcpyDeviceToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_mode, s_hdr, sizeof s_hdr, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) { invalidate(); return pdm_cuda_fail(e, "noalloc write-back", __FILE__, __LINE__); }
    const double ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    if (stats) {
        stats->iterations = done;
        stats->converged = s_status.converged;
        stats->status = status_rc;
        stats->primal = s_status.resid_iter >= 0 ? s_status.primal : NAN;
        stats->dual = s_status.resid_iter >= 0 ? s_status.dual : NAN;
        stats->max_violation = NAN;
        stats->total_radius = NAN;
        stats->device_ms = ms;
    }
    return status_rc;
}
