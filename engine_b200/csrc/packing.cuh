// Fused circle-packing ADMM engine: data layout shared by kernels and host.
//
// Problem (per instance): N circles; circle i owns the centre variable c_i
// (2 components) and the radius variable r_i (2 components in the reference,
// both always equal here, so one is stored).  Factors:
//   pair   (i < j): edges [c_i, r_i, c_j, r_j]  disk_collision_variable_radius
//                   (packing/host.c:83-132)
//   wall   (i, w):  edges [c_i, r_i]            disk_plane_collision_variable_radius
//                   (packing/host.c:31-65)
//   radius (i):     edge  [r_i]                 maximize_sum_of_squared_disk_radii_alpha
//                   (packing/host.c:10-29, 67-81)
//
// One ADMM sweep (reference core/paradmm.c:736-741: updateXM, updateZ,
// updateUN) is restated as ONE pass over the edge state plus a consensus
// finalisation.  The only state kept per live pair-edge component is
// U^(k-1) (FP32), plus, per circle, Z^k (FP64) and Zp = Z^(k-1) (FP32).
// X^k is not stored: it is prox(Zp - U^(k-1)), recomputed with the same
// FP32 operations that produced it in the previous pass.  Sweep k+1 then
// does, per component,
//     X^k = prox(Z^(k-1) - U^(k-1))          (recomputed)
//     U^k = U^(k-1) + alpha (X^k - Z^k)      (updateU of sweep k)
//     N^k = Z^k - U^k                        (updateN of sweep k)
//     X^(k+1) = prox(N^k)                    (updateX of sweep k+1)
//     M = X^(k+1) + U^k                      (updateM of sweep k+1)
// and accumulates rho*M into per-circle FP64 partial sums, which the
// finalisation turns into Z^(k+1) (updateZ of sweep k+1).  So each sweep
// reads and writes U once: 8 bytes per live component.  The prox of a pair
// is a few dozen FP32 operations, far cheaper than the 24 bytes of X it
// replaces.  The first sweep after a state change has no previous X to
// recompute; PkStatus::nmode says what stands in for it:
//     PK_MODE_Z  X^k = Z^k (plain or warm start: U^k = U^(k-1))
//     PK_MODE_N  N^k and U^k given (state uploaded from a reference graph;
//                N lives in the aux tiles); the sweep after it recomputes
//                X from that N (PK_MODE_XN), not from Z - U
// Wall and radius edges (a few per circle) keep X and U explicitly.
//
// Pair state layout.  Circles are cut into blocks of BW = 32*V; the pairs of
// block I against block J >= I form tile (I, J), numbered row-major over the
// upper triangle.  A tile is BW rows (circle i) x 6 components x BW columns
// (circle j) of U floats.  Lane l of a warp owns columns [V l, V l + V);
// its 6V values of a row, q = comp * V + (col - V l) with comp = cx_i, cy_i,
// r_i, cx_j, cy_j, r_j, sit in 16-byte chunks: chunk q/4 of lane l at float
// (q/4) * 128 + 4 l (pk_uoff).  So the warp moves a row as 3V/2 fully
// coalesced 512-byte segments and each lane touches only its own chunks.
// A diagonal tile (I, I) with n circles is stored folded (pk_pair_row_slot):
// storage row t holds circle t's pairs (t, c) at slot c - 1 and circle
// n - 1 - t's pairs at slot n - 1 - c, so its ceil(n / 2) storage rows are
// full.  Slots past N are never touched.
#pragma once

#include <stdint.h>

#include "common.cuh"

#define PK_THREADS 256
// The per-instance schedule's on-chip solver takes instances of at most
// PK_SMALL_N circles (one tile) with at most PK_SMALL_W walls per circle.
#define PK_SMALL_N 40
#define PK_SMALL_W 4
#define PK_WARPS (PK_THREADS / 32)
#define PK_COMPS 6

// First-sweep modes (PkStatus::nmode).
#define PK_MODE_RECOMPUTE 0
#define PK_MODE_Z 1
#define PK_MODE_N 2
#define PK_MODE_XN 3

// Per-instance constants.
struct PkInst {
    int N;                  // circles
    int nb;                 // circle blocks (ceil(N / BW))
    int circle_base;        // global index of the instance's circle 0
    int item_base;          // first work item
    int n_items;            // work items (pair tiles + circle blocks)
    int fin_base;           // first consensus item (one per circle block)
    long long tile_base;    // global index of tile (0, 0)
    float alpha[4];         // pair edge steps by position (c_i, r_i, c_j, r_j)
    float A1, A2, B2m1, C1; // pair prox coefficients (see pair_prox)
    float D1, C2, D2, pad1;
    double rho[4];          // pair edge penalties by position (FP64, consensus weights)
    double inv_ncomp;       // 1 / (num_edges * num_dims) of the reference graph
    double pad2;
};

// Per-circle constants (global circle index).
struct PkCircle {
    double inv_rho_c;   // 1 / sum of rho over the centre variable's edges
    double inv_rho_r;   // 1 / sum of rho over the radius variable's edges
    double w_c;         // edges of the centre variable (dual-residual weight per dim)
    double w_r;         // 2 x edges of the radius variable (both dims)
    int wall_start, wall_count;
    int rad_start, rad_count;
    int inst;
    int pad[3];
};

// Work item of the pass: x = instance, y = kind (0 pair tile, 1 circle
// block), kind 0: z = I, w = J (block indices); kind 1: z = first circle,
// w = count (int4).  Consensus item: x = instance, y = circle block (int2).

// Per-instance run status, written by the kernel.
struct PkStatus {
    long long last_iter;    // last sweep index this instance executes (LLONG_MAX: none yet)
    long long check_from;   // first sweep index whose finalisation may stop it
    long long resid_iter;   // iterate the residuals below belong to (-1: none)
    double primal, dual;
    int converged;
    int nonfinite;
    int nmode;              // PK_MODE_* of sweep mode_iter (every other sweep recomputes X)
    int pad;                // 1 once the instance fell back to its plain start (per-instance schedule)
    long long mode_iter;    // sweep index the mode applies to
    unsigned long long t_begin_ns, t_end_ns;  // per-instance schedule: device clock at start / stop
    // residual balancing of the penalties (PkRun::bal_period > 0; pk_bal_at)
    long long bal_base;      // sweep index whose iterate is the first since the state was set (age 1)
    long long bal_pass_age;  // age of the first iterate computed with scale 2^bal_log2_new (0: none yet)
    long long bal_eval_from; // grid schedule: first finalisation whose residual sums may feed a decision
    int bal_log2_cur;        // log2 of the penalty scale of the iterates before bal_pass_age
    int bal_log2_new;        // ... from bal_pass_age on
    double sd_last;          // per-instance schedule: dual-residual sum of the last consensus run
    int sd_valid;            // sd_last belongs to the state the next call continues
    int yield_at;            // per-instance schedule: sweep at which the instance stops for the grid-wide schedule (0: none)
};

// Device pointers of a packing handle (passed by value to kernels).
struct PkDev {
    const PkInst *inst;
    const int4 *items;
    const PkCircle *circ;
    const int *claim;        // [n_claim] order in which blocks claim items (largest first)
    int n_inst, n_items, n_circ, n_claim;  // n_claim: items in `claim` (n_items, or a subset's)
    float *tiles;            // pair state
    double4 *row_part;       // [tile][BW] sums of M over the row circle's pair edges; w: their primal-residual sum
    double4 *col_part;       // [tile][BW] same for the column circle
    double4 *Z;              // [circle] consensus (cx, cy, r, -)
    const double4 *Z0;       // [circle] the instance's plain start (fallback target)
    float4 *Zp;              // [circle] Z of the previous sweep (FP32: the values the pass used)
    float *aux;              // N of the pair edges for PK_MODE_N (tile layout; graph handles only)
    double4 *local_part;     // [circle] rho-weighted wall + radius contributions; w: their primal-residual sum
    const int2 *fin_items;   // [n_finl] consensus items (instance, circle block) the grid schedule runs
    int n_fin, n_finl;       // n_fin: all consensus items (the stride of blk_*); n_finl: items in fin_items
    double *blk_primal;      // [4][n_fin] per consensus item, by sweep index mod 4
    double *blk_dual;        // [4][n_fin]
    PkStatus *status;        // [n_inst]
    // walls (sorted by circle)
    const float4 *wall_vp;   // v_x, v_y, p_x, p_y
    const float4 *wall_coef; // rho_c, rho_r, alpha_c, alpha_r
    const double2 *wall_rho; // rho_c, rho_r (FP64)
    float4 *wall_X;          // cx, cy, r, -
    float4 *wall_U;
    // radius factors (sorted by circle)
    const float4 *rad_coef;  // exponent, rho, alpha, -
    const double *rad_rho;
    float2 *rad_XU;          // X, U of the radius edge
    struct DevCtl *ctl;
};

struct PkRun {
    long long it0;    // global sweep index of the launch's first sweep
    int n_iter;       // sweeps to run
    int dynamic;      // dynamic work-item scheduling
    double tol;       // stop when primal + dual <= tol (tol < 0: never)
    int check_every;  // sweeps between stopping checks
    int prof;         // accumulate per-phase block times into DevCtl::prof
    int fallback_after;  // per-instance schedule: restart an unconverged instance from Z0 after this many sweeps (0: never)
    int bal_period;   // residual balancing: decide every bal_period iterates (0: off; >= 3)
    double bal_mu;    // ... double the penalties when r > mu s, halve them when s > mu r
    int bal_lmin, bal_lmax;  // ... within scales 2^bal_lmin .. 2^bal_lmax
    int bal_any;      // balancing on, or some instance's penalties not at scale 1: passes read the scale
    int yield_below;  // per-instance schedule: once every instance has started and at most this many are
                      // unfinished, they stop (yielded) for the grid-wide schedule to finish (0: never)
};

// Residual balancing of the penalties (no reference counterpart: the
// reference's hook for it, update_outgoing_rhos, is empty,
// core/paradmm.c:564-566).  Every penalty of an instance is scaled by 2^l.
// Power-of-two scaling is exact, and the pair and wall operators and the
// consensus weights are homogeneous in the penalties, so only the radius
// operator (absolute penalty) and the scaled duals U = y / rho see it.  A
// decision taken on the residuals of the iterate of age a (a a multiple of
// the period) applies in the pass that produces the iterate of age a + 3:
// that pass divides U^(a+2) by t = 2^(l_new - l_cur) right after updating
// it (before N = Z - U), and its radius operator and every later one use
// 2^l_new.  Ages count iterates since the state was set (create, upload,
// warm start, fallback restart).
struct PkBal {
    float uf;  // factor on U right after its update in this pass (1, 1/2 or 2)
    float rs;  // penalty scale of this pass's radius operator
};

PDM_D PkBal pk_bal_none()
{
    PkBal b;
    b.uf = 1.0f;
    b.rs = 1.0f;
    return b;
}

// An instance's balancing state as a kernel carries it from sweep to sweep.
// CTAs that solve one instance together each keep their own copy and take
// the same decisions from the same residual sums, so none reads the status
// while another writes it.
struct PkBalState {
    long long base, pass_age;
    int cur, nw;
};

PDM_D PkBalState pk_bal_load(const PkStatus *st)
{
    PkBalState b;
    b.base = __ldcg(&st->bal_base);
    b.pass_age = __ldcg(&st->bal_pass_age);
    b.cur = __ldcg(&st->bal_log2_cur);
    b.nw = __ldcg(&st->bal_log2_new);
    return b;
}

PDM_D PkBal pk_bal_eval(const PkBalState &s, long long k)
{
    const long long age = k - s.base + 1;
    PkBal b;
    b.rs = ldexpf(1.0f, (s.pass_age > 0 && age >= s.pass_age) ? s.nw : s.cur);
    b.uf = (s.pass_age > 0 && age == s.pass_age && s.nw != s.cur) ? (s.nw > s.cur ? 0.5f : 2.0f) : 1.0f;
    return b;
}

PDM_D PkBal pk_bal_at(const PkStatus *st, long long k) { return pk_bal_eval(pk_bal_load(st), k); }

// The balancing decision on the residuals (rp, rd) of iterate j; returns
// whether the state changed.
PDM_D bool pk_bal_step(PkBalState &s, const PkRun &R, long long j, double rp, double rd)
{
    if (R.bal_period <= 0) return false;
    const long long age = j - s.base + 1;
    if (age < R.bal_period || age % R.bal_period != 0) return false;
    const int cur = s.nw;  // the previous decision applied at least period - 3 iterates ago
    int nw = cur;
    if (rp > R.bal_mu * rd && cur < R.bal_lmax) nw = cur + 1;
    else if (rd > R.bal_mu * rp && cur > R.bal_lmin) nw = cur - 1;
    s.cur = cur;
    s.nw = nw;
    s.pass_age = age + 3;
    return true;
}

PDM_D void pk_bal_store(PkStatus *st, const PkBalState &s)
{
    st->bal_log2_cur = s.cur;
    st->bal_log2_new = s.nw;
    st->bal_pass_age = s.pass_age;
}

// The same decision on the status itself (one thread, no other reader).
PDM_D void pk_bal_decide(PkStatus *st, const PkRun &R, long long j, double rp, double rd)
{
    PkBalState b;
    b.base = st->bal_base;
    b.pass_age = st->bal_pass_age;
    b.cur = st->bal_log2_cur;
    b.nw = st->bal_log2_new;
    if (pk_bal_step(b, R, j, rp, rd)) pk_bal_store(st, b);
}

// Balancing state of a freshly set state whose first sweep is k.
PDM_D PkBalState pk_bal_fresh(long long k)
{
    PkBalState b;
    b.base = k;
    b.pass_age = 0;
    b.cur = b.nw = 0;
    return b;
}

PDM_HD void pk_bal_reset(PkStatus &s, long long k)
{
    s.bal_base = k;
    s.bal_pass_age = 0;
    s.bal_eval_from = k + 2;
    s.bal_log2_cur = s.bal_log2_new = 0;
    s.sd_last = 0.0;
    s.sd_valid = 0;
}

// Initial-state arguments of pk_init_state (device arrays of one instance;
// NULL = none).
struct PkInitArgs {
    const float *pair_duals = nullptr;  // [pair, row-major i < j][6]
    const float *wall_duals = nullptr;  // [wall factor of the instance][3]
    const float *rad_duals = nullptr;   // [circle]
    int radius_duals = 0;     // rad_duals NULL: 1 = radius duals at the radius prox's fixed point, 0 = 0
    int dual_iters = 0;       // rounds of the reference's optimal-initialisation map after that
    int row_lo = 0, row_hi = -1;  // stored block rows (row_hi < 0: all)
};

PDM_HD long long pk_tri(int I, int J, int nb) { return (long long)I * nb - (long long)I * (I - 1) / 2 + (J - I); }
PDM_HD long long pk_tile_floats(int BW) { return (long long)BW * PK_COMPS * BW; }

// Mode of sweep k for an instance whose status is st.
PDM_HD int pk_mode_at(int nmode, long long mode_iter, long long k)
{
    if (k == mode_iter) return nmode;
    if (k == mode_iter + 1 && nmode == PK_MODE_N) return PK_MODE_XN;
    return PK_MODE_RECOMPUTE;
}

// Storage row and slot of pair (i, j), i < j, local to tile (I, J) with nI
// circles in block I: (i, j) for an off-diagonal tile, the folded position
// for a diagonal one.
PDM_HD void pk_pair_row_slot(bool diag, int nI, int i, int j, int &row, int &slot)
{
    if (!diag) { row = i; slot = j; }
    else if (i < (nI + 1) / 2) { row = i; slot = j - 1; }
    else { row = nI - 1 - i; slot = nI - 1 - j; }
}

// Float offset of (component, column) within a tile row (layout above).
template <int V>
PDM_HD int pk_uoff(int comp, int col)
{
    const int q = comp * V + col % V;
    return (q >> 2) * 128 + (col / V) * 4 + (q & 3);
}
