// FP32 proximal operators of the three circle-packing factors, shared by
// the tiled engine (packing_kernels.cu) and the cluster-resident solver
// (onchip_kernels.cu).
#pragma once

#include "packing.cuh"

// ---------------------------------------------------------------------------
// Proximal operators in FP32 (reference: packing/host.c:10-132).
// ---------------------------------------------------------------------------

// disk_collision_variable_radius (packing/host.c:83-132).  n/x hold
// [cx_i, cy_i, r_i, cx_j, cy_j, r_j].  With the edge penalties fixed per
// position, the reference's closed form is linear in (nx2, nr1, nr2) with
// coefficients precomputed on the host (PkInst::A1 ...):
//   x1lin = (nx2 - nr1 - nr2) A1
//   x2lin - nx2 = (nr1 + nr2) A2 + nx2 (B2 - 1)
//   r1lin = (nx2 - nr2) C1 + nr1 D1,   r2lin = (nx2 - nr1) C2 + nr2 D2
// and the centres move along (c_j - c_i) / |c_j - c_i|.
PDM_D void pair_prox(const PkInst &P, const float n[6], float x[6])
{
#pragma unroll
    for (int k = 0; k < 6; ++k) x[k] = n[k];
    const float dx = n[0] - n[3], dy = n[1] - n[4];
    const float d2 = dx * dx + dy * dy;
    const float s = n[2] + n[5];
    if (d2 < s * s) {
        const float d = sqrtf(d2);
        const float inv = 1.0f / d;
        const float ux = (n[3] - n[0]) * inv, uy = (n[4] - n[1]) * inv;
        const float x1 = (d - n[2] - n[5]) * P.A1;
        const float x2m = (n[2] + n[5]) * P.A2 + d * P.B2m1;
        x[0] = n[0] + ux * x1;
        x[1] = n[1] + uy * x1;
        x[3] = n[3] + ux * x2m;
        x[4] = n[4] + uy * x2m;
        x[2] = (d - n[5]) * P.C1 + n[2] * P.D1;
        x[5] = (d - n[2]) * P.C2 + n[5] * P.D2;
    }
}

// disk_plane_collision_variable_radius (packing/host.c:31-65), 2-D.
PDM_D void wall_prox(float nx, float ny, float nr, float4 vp, float rc, float rr, float4 &X)
{
    const float inner = vp.x * (nx - vp.z) + vp.y * (ny - vp.w);
    if (inner + nr > 0.0f) {
        float r = (-inner * rc + nr * rr) / (rc + rr);
        if (r < 0.0f) r = 0.0f;
        X.x = nx - inner * vp.x - vp.x * r;
        X.y = ny - inner * vp.y - vp.y * r;
        X.z = r;
    } else {
        X.x = nx; X.y = ny; X.z = nr;
    }
}

// max_alpha_radius (packing/host.c:10-29): ten Newton steps on the prox of
// -r^a; r^(a-1) and r^(a-2) are exact for a = 2 (r, 1) and a = 1 (1, 1/r).
// For a = 2 the Newton function -r + (rho/a)(r - n) is linear in r, so the
// first step lands on its root rho n / (rho - 2) and the other nine move r by
// rounding only: one step is taken (ten FP32 divisions were two thirds of a
// small instance's consensus).  a = 1 keeps the ten steps, which carry the
// reference's NaN at n = 0 (1/r at r = 0).
PDM_D float radius_prox(float n, float rho, float a)
{
    float r = fabsf(n * 0.5f);
    const float ra = rho / a;
    if (a == 2.0f) {
        r -= (-r + ra * (r - n)) / (-1.0f + ra);
        return r < 0.0f ? 0.0f : r;
    }
    for (int it = 0; it < 10; ++it) {
        float p1, p2;
        if (a == 2.0f) { p1 = r; p2 = 1.0f; }
        else if (a == 1.0f) { p1 = 1.0f; p2 = 1.0f / r; }
        else { p1 = powf(r, a - 1.0f); p2 = powf(r, a - 2.0f); }
        const float num = -p1 + ra * (r - n);
        const float den = -(a - 1.0f) * p2 + ra;
        r -= num / den;
        if (r < 0.0f) return 0.0f;
    }
    return r;
}

