// Cluster-resident solver for batches of packing instances (the
// per-instance schedule's PARADMM_SCHEDULE_ONCHIP form).
//
// A batch of instances of uneven size (N up to a few hundred circles) is
// latency-bound when each sweep streams an instance's few tiles from L2/HBM:
// every tile carries block barriers, Z loads and a row pipeline that fills
// and drains.  Here an instance's whole U-only pair state stays in the shared
// memory of a group of k CTAs of one thread-block cluster (k = 1 .. 16, one
// CTA per SM, up to ~220 KB each) for all of its sweeps, so a sweep touches
// no global memory at all; the group meets at two barriers per sweep and
// reads the other CTAs' partial sums through distributed shared memory.
//
// Layout (per instance).  Circles are cut into blocks of 32; the pairs of
// block I against block J >= I form tile (I, J), cut into OC_S strips of
// OC_SR rows x 32 columns (lane = column).  Strips are numbered tile-major
// (tile index pk_tri(I, J, nb)) and dealt to the group's CTAs in contiguous
// ranges; circles are dealt the same way (the CTA that "owns" a circle runs
// its wall and radius factors and its consensus).  Every CTA holds, as FP32,
// the current and previous consensus of all the instance's circles.  A strip
// keeps U of its pairs ([row][component][lane]), the row sums of M and of the
// primal residual of its rows over its 32 columns, and the column sums of M
// over its rows.
//
// Sweep k of an instance (the same arithmetic as the tiled engine's fused
// pass, packing_kernels.cu): pass over the CTA's strips and owned circles;
// group barrier; consensus of the owned circles (row partials from the
// strips of block row b, column partials from the strips of block column b,
// in a fixed order, in FP64), new Z written into every group CTA's copy;
// per-CTA residual sums to the group leader; group barrier; the stop test,
// computed identically by every CTA of the group.  Which CTA holds a strip
// does not enter the arithmetic, so an instance gives the same result bit
// for bit whatever its group size.  State goes from and back to the
// handle's tiled global layout at the start and end of an instance's solve.
#include <climits>

#include <cooperative_groups.h>

#include "common.cuh"
#include "packing.cuh"
#include "packing_launch.h"
#include "packing_ops.cuh"

namespace cg = cooperative_groups;

#define OC_THREADS 512
#define OC_WARPS (OC_THREADS / 32)
#define OC_T 32                           // strip width (columns) = lanes
#define OC_SR 4                           // rows per strip
#define OC_S (OC_T / OC_SR)               // strips per tile
#define OC_SU (OC_SR * PK_COMPS * OC_T)   // floats of U per strip
#define OC_SP (OC_SR * 4)                 // row partial floats per strip
#define OC_SC (OC_T * 3)                  // column partial floats per strip

// Bytes of dynamic shared memory an instance of N circles needs on each of k
// CTAs (same carve for every CTA of the group: the largest share).
PDM_HD long long oc_bytes(int N, int k)
{
    const int nb = (N + OC_T - 1) / OC_T;
    const long long ns = ((long long)nb * (nb + 1) / 2 * OC_S + k - 1) / k;
    const long long no = (N + k - 1) / k;
    long long b = 2LL * 16 * N;                              // zf, zpf (float4)
    b += no * (32 + 32 + 2 * 16 * OC_MAX_WALLS + 8);         // zd, lp, wX, wU, rXU
    b = (b + 15) & ~15LL;
    b += ns * (OC_SU + OC_SP + OC_SC) * 4;                   // strips
    return b;
}

struct OcCarve {
    float4 *zf, *zpf;    // [N] consensus of the current / previous sweep, FP32 (every CTA)
    double4 *zd;         // [no] owned circles' consensus, FP64
    double4 *lp;         // [no] owned circles' wall + radius contributions (x, y, r, primal)
    float4 *wX, *wU;     // [no][OC_MAX_WALLS]
    float2 *rXU;         // [no]
    float *su, *sp, *sc; // strips: U, row partials, column partials
};

PDM_D OcCarve oc_carve(unsigned char *base, int N, int k)
{
    const int nb = (N + OC_T - 1) / OC_T;
    const int ns = (nb * (nb + 1) / 2 * OC_S + k - 1) / k;
    const int no = (N + k - 1) / k;
    OcCarve c;
    c.zf = reinterpret_cast<float4 *>(base);
    c.zpf = c.zf + N;
    c.zd = reinterpret_cast<double4 *>(c.zpf + N);
    c.lp = c.zd + no;
    c.wX = reinterpret_cast<float4 *>(c.lp + no);
    c.wU = c.wX + no * OC_MAX_WALLS;
    c.rXU = reinterpret_cast<float2 *>(c.wU + no * OC_MAX_WALLS);
    uintptr_t p = reinterpret_cast<uintptr_t>(c.rXU + no);
    p = (p + 15) & ~(uintptr_t)15;
    c.su = reinterpret_cast<float *>(p);
    c.sp = c.su + (long long)ns * OC_SU;
    c.sc = c.sp + (long long)ns * OC_SP;
    return c;
}

// First strip (or circle) of group rank r when n are dealt over k CTAs.
PDM_HD int oc_first(int r, int n, int k) { return (int)((long long)r * n / k); }
PDM_D int oc_owner(int x, int n, int k)
{
    int r = (int)((long long)x * k / n);
    while (r + 1 < k && oc_first(r + 1, n, k) <= x) ++r;
    while (r > 0 && oc_first(r, n, k) > x) --r;
    return r;
}

// Synchronisation of a group of k CTAs inside the cluster: the whole
// cluster's hardware barrier when the group is the cluster, a counter in the
// group leader's shared memory otherwise (arrival with cluster-scope
// release, bounded polling with acquire).  Every CTA of the group calls it
// the same number of times.
struct OcSync {
    unsigned bar_addr;   // cluster shared-memory address of the leader's counter
    unsigned target;     // arrivals that end the next barrier (thread 0 only)
    int k;
    bool whole;
};

PDM_D void oc_group_sync(OcSync &g, DevCtl *ctl)
{
    if (g.whole) {
        cg::this_cluster().sync();
        return;
    }
    __syncthreads();
    if (g.k > 1 && threadIdx.x == 0) {
        g.target += (unsigned)g.k;
        asm volatile("red.release.cluster.shared::cluster.add.u32 [%0], 1;" ::"r"(g.bar_addr) : "memory");
        unsigned v = 0;
        for (unsigned long long n = 0;; ++n) {
            asm volatile("ld.acquire.cluster.shared::cluster.u32 %0, [%1];" : "=r"(v) : "r"(g.bar_addr) : "memory");
            if ((int)(v - g.target) >= 0) break;
            if (n > PDM_BARRIER_MAX_POLLS) {
                atomicCAS(&ctl->err, DEV_OK, DEV_BARRIER_TIMEOUT);
                break;
            }
        }
    }
    __syncthreads();
}

// Four values summed over the 32 lanes in six shuffles (a reduce-scatter
// butterfly): afterwards lane l holds the sum of value 2 (l >> 4 & 1) +
// (l >> 3 & 1); lanes 0, 8, 16, 24 hold values 0, 1, 2, 3.  Fixed order.
PDM_D float oc_sum4(float a0, float a1, float a2, float a3, int lane)
{
    const bool hi = (lane & 16) != 0;
    const float r0 = __shfl_xor_sync(0xffffffffu, hi ? a0 : a2, 16);
    const float r1 = __shfl_xor_sync(0xffffffffu, hi ? a1 : a3, 16);
    const float b0 = (hi ? a2 : a0) + r0, b1 = (hi ? a3 : a1) + r1;
    const bool mid = (lane & 8) != 0;
    float c = (mid ? b1 : b0) + __shfl_xor_sync(0xffffffffu, mid ? b0 : b1, 8);
    c += __shfl_xor_sync(0xffffffffu, c, 4);
    c += __shfl_xor_sync(0xffffffffu, c, 2);
    c += __shfl_xor_sync(0xffffffffu, c, 1);
    return c;
}

// Global (tiled engine layout, block width 32 V) float offset of component q
// of pair (i, j), i < j, of instance P.
template <int V>
PDM_D long long oc_goff(const PkInst &P, int i, int j, int q)
{
    constexpr int BW = 32 * V;
    const int I = i / BW, J = j / BW;
    int row, slot;
    pk_pair_row_slot(I == J, min(BW, P.N - I * BW), i - I * BW, j - J * BW, row, slot);
    return (P.tile_base + pk_tri(I, J, P.nb)) * pk_tile_floats(BW) + (long long)row * (PK_COMPS * BW) +
           pk_uoff<V>(q, slot);
}

// Tile (I, J) of tile index t among nb blocks.
PDM_D void oc_tile_ij(int t, int nb, int &I, int &J)
{
    I = 0;
    while (pk_tri(I + 1, I + 1, nb) <= t) ++I;
    J = I + (int)(t - pk_tri(I, I, nb));
}

struct OcGroup {
    int k, grank, gbase;   // group size, rank in the group, cluster rank of the leader
};

// Solves instance i with this CTA's share of the group's work.  The same
// stop, fallback and balancing rules as pk_solve_instance (packing_kernels.cu).
template <int V>
PDM_D void oc_solve(const PkDev &D, const PkRun &R, int i, const OcGroup &G, OcSync &gs, unsigned char *smem,
                    double2 *s_res, int *s_stop, PkBalState *s_bal)
{
    cg::cluster_group cl = cg::this_cluster();
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    const PkInst &P = D.inst[i];
    PkStatus *st = &D.status[i];
    const int N = P.N, k = G.k, gr = G.grank;
    const int nb = (N + OC_T - 1) / OC_T;
    const int NS = nb * (nb + 1) / 2 * OC_S;
    const int s0 = oc_first(gr, NS, k), ns = oc_first(gr + 1, NS, k) - s0;
    const int o0 = oc_first(gr, N, k), no = oc_first(gr + 1, N, k) - o0;
    const OcCarve C = oc_carve(smem, N, k);
    const int g0 = P.circle_base;
    const float aCi = P.alpha[0], aRi = P.alpha[1], aCj = P.alpha[2], aRj = P.alpha[3];
    const float al[6] = {aCi, aCi, aRi, aCj, aCj, aRj};

    // ---- load: consensus of all circles, owned circles' factors, strips
    for (int c = tid; c < N; c += OC_THREADS) {
        const double4 z = ldcg_d4(&D.Z[g0 + c]);
        C.zf[c] = make_float4((float)z.x, (float)z.y, (float)z.z, 0.f);
        C.zpf[c] = __ldcg(&D.Zp[g0 + c]);
    }
    for (int o = tid; o < no; o += OC_THREADS) {
        const int g = g0 + o0 + o;
        const PkCircle Cc = D.circ[g];
        C.zd[o] = ldcg_d4(&D.Z[g]);
        for (int q = 0; q < Cc.wall_count; ++q) {
            C.wX[o * OC_MAX_WALLS + q] = __ldcg(&D.wall_X[Cc.wall_start + q]);
            C.wU[o * OC_MAX_WALLS + q] = __ldcg(&D.wall_U[Cc.wall_start + q]);
        }
        C.rXU[o] = __ldcg(&D.rad_XU[Cc.rad_start]);
    }
    for (int e = tid; e < ns * OC_SR * OC_T; e += OC_THREADS) {
        const int ls = e / (OC_SR * OC_T), rr = (e / OC_T) % OC_SR, l = e % OC_T;
        const int x = s0 + ls, t = x / OC_S, s = x % OC_S;
        int I, J;
        oc_tile_ij(t, nb, I, J);
        const int ri = I * OC_T + s * OC_SR + rr, cj = J * OC_T + l;
        const bool ok = ri < N && cj < N && cj > ri;
        float *u = C.su + (long long)ls * OC_SU + rr * PK_COMPS * OC_T + l;
#pragma unroll
        for (int q = 0; q < PK_COMPS; ++q) u[q * OC_T] = ok ? __ldcg(D.tiles + oc_goff<V>(P, ri, cj, q)) : 0.f;
    }
    const int m0 = pk_mode_at(__ldcg(&st->nmode), __ldcg(&st->mode_iter), R.it0);
    long long zmode_at = m0 == PK_MODE_Z ? R.it0 : -1;  // sweep whose X^k is Z^k (state just set)
    long long check_from = __ldcg(&st->check_from);
    long long restart_at = R.fallback_after > 0 ? R.it0 + R.fallback_after : -1;
    const bool sd_valid = __ldcg(&st->sd_valid) != 0;
    double sd_prev = sd_valid ? __ldcg(&st->sd_last) : 0.0;
    long long bal_from = R.it0 + (sd_valid ? 0 : 1);
    if (gr == 0 && tid == 0) st->t_begin_ns = globaltimer_ns();
    // this CTA's copy of the balancing state (every CTA of the group takes
    // the same decisions; the leader records them in the status)
    if (tid == 0) *s_bal = pk_bal_load(st);
    __syncthreads();

    long long k_sw = R.it0;
    for (; k_sw < R.it0 + R.n_iter; ++k_sw) {
        const bool zmode = k_sw == zmode_at;
        const PkBal bal = R.bal_any ? pk_bal_eval(*s_bal, k_sw) : pk_bal_none();
        // ---- pass: strips (warps)
        for (int ls = w; ls < ns; ls += OC_WARPS) {
            const int x = s0 + ls, t = x / OC_S, s = x % OC_S;
            int I, J;
            oc_tile_ij(t, nb, I, J);
            const int cj = J * OC_T + lane;
            const bool col_ok = cj < N;
            float4 zc = make_float4(0.f, 0.f, 0.f, 0.f), zpc = zc;
            if (col_ok) { zc = C.zf[cj]; zpc = C.zpf[cj]; }
            float cx = 0.f, cy = 0.f, cr = 0.f;
            float *su = C.su + (long long)ls * OC_SU;
#pragma unroll
            for (int rr = 0; rr < OC_SR; ++rr) {
                const int ri = I * OC_T + s * OC_SR + rr;
                const bool ok = col_ok && ri < N && cj > ri;
                float m0v = 0.f, m1v = 0.f, m2v = 0.f, sq = 0.f;
                if (ok) {
                    const float4 zi = C.zf[ri], zpi = C.zpf[ri];
                    const float z[6] = {zi.x, zi.y, zi.z, zc.x, zc.y, zc.z};
                    float u[6], xv[6], n[6];
#pragma unroll
                    for (int q = 0; q < 6; ++q) u[q] = su[(rr * PK_COMPS + q) * OC_T + lane];
                    if (zmode) {
#pragma unroll
                        for (int q = 0; q < 6; ++q) xv[q] = z[q];
                    } else {
                        const float zp[6] = {zpi.x, zpi.y, zpi.z, zpc.x, zpc.y, zpc.z};
#pragma unroll
                        for (int q = 0; q < 6; ++q) n[q] = zp[q] - u[q];
                        pair_prox(P, n, xv);  // X^k = prox(Z^(k-1) - U^(k-1)), as the last pass had it
                    }
#pragma unroll
                    for (int q = 0; q < 6; ++q) {
                        const float dk = xv[q] - z[q];
                        u[q] = fmaf(al[q], dk, u[q]);
                        sq += ((q == 2 || q == 5) ? 2.0f : 1.0f) * dk * dk;
                    }
                    if (bal.uf != 1.0f) {
#pragma unroll
                        for (int q = 0; q < 6; ++q) u[q] *= bal.uf;
                    }
#pragma unroll
                    for (int q = 0; q < 6; ++q) n[q] = z[q] - u[q];
                    pair_prox(P, n, xv);
                    m0v = xv[0] + u[0]; m1v = xv[1] + u[1]; m2v = xv[2] + u[2];
                    cx += xv[3] + u[3]; cy += xv[4] + u[4]; cr += xv[5] + u[5];
#pragma unroll
                    for (int q = 0; q < 6; ++q) su[(rr * PK_COMPS + q) * OC_T + lane] = u[q];
                }
                const float r4 = oc_sum4(m0v, m1v, m2v, sq, lane);
                if ((lane & 7) == 0) C.sp[(long long)ls * OC_SP + rr * 4 + (lane >> 3)] = r4;
            }
            float *scp = C.sc + (long long)ls * OC_SC + lane * 3;
            scp[0] = cx; scp[1] = cy; scp[2] = cr;
        }
        // ---- pass: owned circles' wall and radius factors (as pk_circle_block)
        for (int o = tid; o < no; o += OC_THREADS) {
            const int c = o0 + o, g = g0 + c;
            const PkCircle Cc = D.circ[g];
            const float4 z4 = C.zf[c];
            const float zx = z4.x, zy = z4.y, zr = z4.z;
            double ax = 0.0, ay = 0.0, ar = 0.0;
            float sq = 0.f;
            for (int q = 0; q < Cc.wall_count; ++q) {
                float4 X = C.wX[o * OC_MAX_WALLS + q], U = C.wU[o * OC_MAX_WALLS + q];
                const float4 vp = __ldg(&D.wall_vp[Cc.wall_start + q]), cf = __ldg(&D.wall_coef[Cc.wall_start + q]);
                const double2 rd = __ldg(&D.wall_rho[Cc.wall_start + q]);
                const float dx = X.x - zx, dy = X.y - zy, dr = X.z - zr;
                U.x = fmaf(cf.z, dx, U.x) * bal.uf; U.y = fmaf(cf.z, dy, U.y) * bal.uf;
                U.z = fmaf(cf.w, dr, U.z) * bal.uf;
                sq += dx * dx + dy * dy + 2.0f * dr * dr;
                wall_prox(zx - U.x, zy - U.y, zr - U.z, vp, cf.x, cf.y, X);
                ax += rd.x * (double)(X.x + U.x);
                ay += rd.x * (double)(X.y + U.y);
                ar += rd.y * (double)(X.z + U.z);
                C.wX[o * OC_MAX_WALLS + q] = X;
                C.wU[o * OC_MAX_WALLS + q] = U;
            }
            {
                float2 xu = C.rXU[o];
                const float4 cf = __ldg(&D.rad_coef[Cc.rad_start]);
                const float dr = xu.x - zr;
                xu.y = fmaf(cf.z, dr, xu.y) * bal.uf;
                sq += 2.0f * dr * dr;
                xu.x = radius_prox(zr - xu.y, cf.y * bal.rs, cf.x);
                ar += __ldg(&D.rad_rho[Cc.rad_start]) * (double)(xu.x + xu.y);
                C.rXU[o] = xu;
            }
            C.lp[o] = make_double4(ax, ay, ar, (double)sq);
        }
        oc_group_sync(gs, D.ctl);
        // ---- consensus of the owned circles: one warp per circle, its terms
        // (the row partials of the strips of block row b holding the circle's
        // row, then the column partials of the strips of block column b) dealt
        // over the lanes by position, summed in FP64 and reduced over the warp
        // in a fixed order -- the same whatever the group size.
        double dual = 0.0, prim = 0.0;
        for (int o = w; o < no; o += OC_WARPS) {
            const int c = o0 + o, b = c / OC_T, q = c % OC_T;
            const int n_row = nb - b, n_term = n_row + (b + 1) * OC_S;
            double rx = 0.0, ry = 0.0, rr = 0.0, rp = 0.0, cx = 0.0, cy = 0.0, cr = 0.0;
            for (int t = lane; t < n_term; t += 32) {
                if (t < n_row) {
                    const int x = (int)pk_tri(b, b + t, nb) * OC_S + q / OC_SR;
                    const int r = oc_owner(x, NS, k);
                    const float4 v = *reinterpret_cast<const float4 *>(
                        cl.map_shared_rank(C.sp, G.gbase + r) + (long long)(x - oc_first(r, NS, k)) * OC_SP + (q % OC_SR) * 4);
                    rx += (double)v.x; ry += (double)v.y; rr += (double)v.z; rp += (double)v.w;
                } else {
                    const int u = t - n_row, I = u / OC_S;
                    const int x = (int)pk_tri(I, b, nb) * OC_S + u % OC_S;
                    const int r = oc_owner(x, NS, k);
                    const float *p = cl.map_shared_rank(C.sc, G.gbase + r) + (long long)(x - oc_first(r, NS, k)) * OC_SC + q * 3;
                    cx += (double)p[0]; cy += (double)p[1]; cr += (double)p[2];
                }
            }
            rx = warp_sum(rx); ry = warp_sum(ry); rr = warp_sum(rr); rp = warp_sum(rp);
            cx = warp_sum(cx); cy = warp_sum(cy); cr = warp_sum(cr);
            const double4 zo = C.zd[o];
            const int g = g0 + c;
            const PkCircle Cc = D.circ[g];
            const double4 l4 = C.lp[o];
            const double sx = P.rho[0] * rx + P.rho[2] * cx + l4.x;
            const double sy = P.rho[0] * ry + P.rho[2] * cy + l4.y;
            const double sr = P.rho[1] * rr + P.rho[3] * cr + l4.z;
            const double4 zn = make_double4(sx * Cc.inv_rho_c, sy * Cc.inv_rho_c, sr * Cc.inv_rho_r, 0.0);
            const double dx = zn.x - zo.x, dy = zn.y - zo.y, dr = zn.z - zo.z;
            if (lane == 0) {
                C.zd[o] = zn;
                dual += Cc.w_c * (dx * dx + dy * dy) + Cc.w_r * dr * dr;
                prim += rp + l4.w;
            }
            if (lane < k) {  // the new consensus into every group CTA's copy
                *cl.map_shared_rank(C.zf + c, G.gbase + lane) =
                    make_float4((float)zn.x, (float)zn.y, (float)zn.z, 0.f);
                *cl.map_shared_rank(C.zpf + c, G.gbase + lane) =
                    make_float4((float)zo.x, (float)zo.y, (float)zo.z, 0.f);
            }
        }
        const double2 pd = block_sum2(prim, dual);
        if (tid == 0) *cl.map_shared_rank(s_res + gr, G.gbase) = pd;
        oc_group_sync(gs, D.ctl);
        // ---- stop test (every CTA of the group takes the same decision)
        if (tid == 0) {
            double sp = 0.0, sd = 0.0;
            for (int m = 0; m < k; ++m) {
                const double2 v = *cl.map_shared_rank(s_res + m, G.gbase);
                sp += v.x;
                sd += v.y;
            }
            int stop = 0;
            const bool bal_due = R.bal_period > 0 && k_sw >= bal_from && (k_sw - s_bal->base) % R.bal_period == 0;
            if (k_sw >= check_from || bal_due) {
                const double rp = sqrt(sp * P.inv_ncomp), rd = sqrt(sd_prev * P.inv_ncomp);
                if (bal_due && pk_bal_step(*s_bal, R, k_sw - 1, rp, rd) && gr == 0) pk_bal_store(st, *s_bal);
                if (k_sw >= check_from) {
                    const bool finite = isfinite(rp) && isfinite(rd);
                    const bool due = R.check_every <= 1 || ((k_sw - R.it0) % R.check_every) == 0;
                    if (!finite) stop = 2;
                    else if (R.tol >= 0.0 && due && rp + rd <= R.tol) stop = 1;
                    if (stop == 2 && restart_at > k_sw + 1) stop = 3;  // a diverging warm start falls back at once
                    if (gr == 0) {
                        st->primal = rp;
                        st->dual = rd;
                        st->resid_iter = k_sw - 1;
                        if (stop == 2) st->nonfinite = 1;
                        if (stop == 1) st->converged = 1;
                    }
                }
            }
            if (stop == 0 && k_sw + 1 == restart_at) stop = 3;  // budget of the warm start spent
            if (ld_volatile_i32(&D.ctl->err) != DEV_OK) stop = 4;
            sd_prev = sd;
            *s_stop = stop;
        }
        __syncthreads();
        const int stop = *s_stop;
        __syncthreads();
        if (stop == 3) {
            // fall back to the plain start for the rest of the call
            for (int c = tid; c < N; c += OC_THREADS) {
                const double4 z = D.Z0[g0 + c];
                C.zf[c] = C.zpf[c] = make_float4((float)z.x, (float)z.y, (float)z.z, 0.f);
            }
            for (int o = tid; o < no; o += OC_THREADS) {
                const int g = g0 + o0 + o;
                const double4 z = D.Z0[g];
                const float4 zf = make_float4((float)z.x, (float)z.y, (float)z.z, 0.f);
                C.zd[o] = z;
                for (int q = 0; q < OC_MAX_WALLS; ++q) {
                    C.wX[o * OC_MAX_WALLS + q] = zf;
                    C.wU[o * OC_MAX_WALLS + q] = make_float4(0.f, 0.f, 0.f, 0.f);
                }
                C.rXU[o] = make_float2(zf.z, 0.f);
            }
            for (long long e = tid; e < (long long)ns * OC_SU; e += OC_THREADS) C.su[e] = 0.f;
            if (gr == 0 && tid == 0) {
                st->nmode = PK_MODE_Z;
                st->mode_iter = k_sw + 1;
                st->pad = 1;
                pk_bal_reset(*st, k_sw + 1);
            }
            if (tid == 0) {
                sd_prev = 0.0;
                *s_bal = pk_bal_fresh(k_sw + 1);
            }
            zmode_at = k_sw + 1;
            check_from = k_sw + 2;
            bal_from = k_sw + 2;
            restart_at = -1;
            // the leader's reset of the status (penalty scale included) reaches
            // every CTA of the group before the next pass reads it
            oc_group_sync(gs, D.ctl);
            continue;
        }
        if (stop) break;
    }
    // ---- state back to the handle's global layout
    for (int e = tid; e < ns * OC_SR * OC_T; e += OC_THREADS) {
        const int ls = e / (OC_SR * OC_T), rr = (e / OC_T) % OC_SR, l = e % OC_T;
        const int x = s0 + ls, t = x / OC_S, s = x % OC_S;
        int I, J;
        oc_tile_ij(t, nb, I, J);
        const int ri = I * OC_T + s * OC_SR + rr, cj = J * OC_T + l;
        if (!(ri < N && cj < N && cj > ri)) continue;
        const float *u = C.su + (long long)ls * OC_SU + rr * PK_COMPS * OC_T + l;
#pragma unroll
        for (int q = 0; q < PK_COMPS; ++q) __stcg(D.tiles + oc_goff<V>(P, ri, cj, q), u[q * OC_T]);
    }
    for (int o = tid; o < no; o += OC_THREADS) {
        const int c = o0 + o, g = g0 + c;
        const PkCircle Cc = D.circ[g];
        stcg_d4(&D.Z[g], C.zd[o]);
        __stcg(&D.Zp[g], C.zpf[c]);
        for (int q = 0; q < Cc.wall_count; ++q) {
            __stcg(&D.wall_X[Cc.wall_start + q], C.wX[o * OC_MAX_WALLS + q]);
            __stcg(&D.wall_U[Cc.wall_start + q], C.wU[o * OC_MAX_WALLS + q]);
        }
        __stcg(&D.rad_XU[Cc.rad_start], C.rXU[o]);
    }
    if (gr == 0 && tid == 0) {
        st->last_iter = k_sw < R.it0 + R.n_iter ? k_sw : R.it0 + R.n_iter - 1;
        st->t_end_ns = globaltimer_ns();
        st->sd_last = sd_prev;  // the consensus of the last sweep run
        st->sd_valid = 1;
    }
}

// One launch, clusters of A.csize CTAs (one CTA per SM).  Cluster c is cut
// into groups of 2^A.glog2[c] CTAs; a group takes instances from the queue
// of its own size class (instances that need exactly that many CTAs), then
// from the smaller classes, largest first, until both are empty.
template <int V>
__global__ void __launch_bounds__(OC_THREADS, 1) pk_onchip(PkDev D, PkRun R, OcArgs A)
{
    extern __shared__ __align__(16) unsigned char oc_smem[];
    __shared__ unsigned s_bar;
    __shared__ int s_inst;
    __shared__ int s_stop;
    __shared__ double2 s_res[OC_MAX_GROUP];
    __shared__ PkBalState s_bal;
    cg::cluster_group cl = cg::this_cluster();
    const int crank = (int)cl.block_rank(), csize = (int)cl.num_blocks();
    const int cid = (int)(blockIdx.x / (unsigned)csize);
    const int lg = A.glog2[cid];
    OcGroup G;
    G.k = 1 << lg;
    G.grank = crank % G.k;
    G.gbase = crank - G.grank;
    OcSync gs;
    gs.k = G.k;
    gs.whole = G.k == csize && G.k > 1;
    gs.target = 0;
    gs.bar_addr = 0;
    if (threadIdx.x == 0) {
        s_bar = 0u;
        unsigned a = smem_u32(&s_bar), m;
        asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(m) : "r"(a), "r"(G.gbase));
        gs.bar_addr = m;
    }
    cl.sync();  // every counter is zero before anyone arrives
    for (;;) {
        if (G.grank == 0 && threadIdx.x == 0) {
            int inst = -1;
            if (ld_volatile_i32(&D.ctl->err) == DEV_OK) {
                for (int c = lg; c >= 0 && inst < 0; --c) {
                    const int n = A.qoff[c + 1] - A.qoff[c];
                    if (n <= 0) continue;
                    const unsigned q = atomicAdd(&A.ctr[c], 1u);
                    if (q < (unsigned)n) inst = A.queue[A.qoff[c] + (int)q];
                }
            }
            for (int m = 0; m < G.k; ++m) *cl.map_shared_rank(&s_inst, G.gbase + m) = inst;
        }
        oc_group_sync(gs, D.ctl);
        const int i = s_inst;
        if (i < 0) break;  // group-uniform
        if (__ldcg(&D.status[i].last_iter) >= R.it0) oc_solve<V>(D, R, i, G, gs, oc_smem, s_res, &s_stop, &s_bal);
        oc_group_sync(gs, D.ctl);  // the group is done with this instance's shared memory
    }
    cl.sync();  // no CTA leaves while a group member may still read its shared memory
}

// ---------------------------------------------------------------------------
// Launchers.
// ---------------------------------------------------------------------------
template <int V>
static cudaError_t oc_prepare(int smem)
{
    cudaError_t e = cudaFuncSetAttribute(pk_onchip<V>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(pk_onchip<V>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
    return e;
}

template <int V>
static cudaError_t oc_clusters_t(int csize, int smem, int *clusters)
{
    cudaError_t e = oc_prepare<V>(smem);
    if (e != cudaSuccess) return e;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(csize);
    cfg.blockDim = dim3(OC_THREADS);
    cfg.dynamicSmemBytes = smem;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = csize;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaOccupancyMaxActiveClusters(clusters, pk_onchip<V>, &cfg);
}

template <int V>
static cudaError_t oc_launch_t(const PkDev &D, const PkRun &R, const OcArgs &A, int n_clusters, int csize, int smem,
                               cudaStream_t s)
{
    cudaError_t e = oc_prepare<V>(smem);
    if (e != cudaSuccess) return e;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(n_clusters * csize);
    cfg.blockDim = dim3(OC_THREADS);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = csize;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, pk_onchip<V>, D, R, A);
}

long long pk_onchip_bytes(int n_circles, int group) { return oc_bytes(n_circles, group); }

cudaError_t pk_onchip_max_clusters(int V, int csize, int smem, int *clusters)
{
    if (V == 2) return oc_clusters_t<2>(csize, smem, clusters);
    if (V == 4) return oc_clusters_t<4>(csize, smem, clusters);
    return cudaErrorInvalidValue;
}

cudaError_t pk_launch_onchip(int V, const PkDev &D, const PkRun &R, const OcArgs &A, int n_clusters, int csize,
                             int smem, cudaStream_t s)
{
    if (V == 2) return oc_launch_t<2>(D, R, A, n_clusters, csize, smem, s);
    if (V == 4) return oc_launch_t<4>(D, R, A, n_clusters, csize, smem, s);
    return cudaErrorInvalidValue;
}
