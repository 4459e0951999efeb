"""The packing engine's FP32 proximal operators against the reference's FP64
ones on about a million random inputs each.

A random edge state (independent random N on every edge, U = 0) is uploaded
into a graph of 1415 circles (1,000,405 pair factors, 5,660 wall factors,
1,415 radius factors).  The engine's next sweep starts with X = prox(N) for
every factor (reference updateXM, core/paradmm.c:569-623), and the download
reports that X.  The reference's own updateX runs the reference operators
(packing/host.c:10-132) on the same N in FP64.  Inputs are rounded to FP32
first so both sides see the same numbers.

Checked: the branch each factor took (pair: d^2 < (r1 + r2)^2, host.c:104;
wall: inner + r > 0, host.c:43; radius: r < 0 clamps to 0, host.c:23-26)
agrees away from the branch boundaries, and there the outputs agree to
1e-5 (absolute, for inputs of order 1).  Factors within 1e-4 of a boundary,
and pairs whose centres nearly coincide (direction undefined), are counted
but not compared.
"""
import numpy as np
import pytest

import engine_b200 as eb
import oracle_lib

pytestmark = pytest.mark.gpu

RHO, RHO_R, ALPHA, EXP = 10.0, 5.0, 1.0, 2.0
TOL = 1e-5


def _factor_tables(G):
    o2n = np.ctypeslib.as_array(G.operatorix_to_numedges, shape=(G.num_opts,))
    first = np.concatenate([[0], np.cumsum(o2n)[:-1]]).astype(np.int64)
    return o2n, first


def test_operators_on_a_million_random_inputs():
    N = 1415
    walls = eb.box_walls(1.0, 1.0)
    rng = np.random.default_rng(2026)
    pg = eb.PackingGraph(N, walls, EXP)
    pg.init_seeded(eb.seeded_circles(N, 1.0, 1.0, 0.05, 5), RHO, RHO_R, ALPHA)
    orc = oracle_lib.OraclePacking(oracle_lib.best(), N, walls, EXP)
    orc.init(5, 1.0, 1.0, 0.05, RHO, RHO_R, ALPHA)
    G, R = pg.G, orc.G
    assert G.num_edges == R.num_edges and np.array_equal(G.arr("RHOS"), R.arr("RHOS"))

    # random N: centres uniform in [-0.1, 1.1]^2 (walls violated or not),
    # radii uniform in [-0.02, 0.12] with both components equal
    ev = np.ctypeslib.as_array(G.edgeix_to_varlistix, shape=(G.num_edges,))
    n = np.empty((G.num_edges, 2))
    cen = ev % 2 == 0
    n[cen] = rng.uniform(-0.1, 1.1, size=(cen.sum(), 2))
    rr = rng.uniform(-0.02, 0.12, size=(~cen).sum())
    n[~cen, 0] = rr
    n[~cen, 1] = rr
    n = n.astype(np.float32).astype(np.float64)
    G.arr("N")[:] = n
    G.arr("U")[:] = 0.0
    R.arr("N")[:] = n
    R.arr("U")[:] = 0.0

    with eb.Handle.from_graph(G, engine=eb.ENGINE_PACKING) as h:
        h.iterate(1)
        h.download(G)
    xg = G.arr("X").copy()
    orc.lib.updateX(orc.graph_ptr())
    xr = R.arr("X").copy()

    o2n, first = _factor_tables(G)
    pairs = first[o2n == 4]
    wall_f = first[o2n == 2]
    rad_e = first[o2n == 1]
    assert len(pairs) == N * (N - 1) // 2 and len(wall_f) == 4 * N and len(rad_e) == N

    # pairs: inputs (ci, ri, cj, rj) at edges e0 .. e0 + 3
    ci, cj = n[pairs], n[pairs + 2]
    ri, rj = n[pairs + 1, 0], n[pairs + 3, 0]
    d2 = ((ci - cj) ** 2).sum(1)
    s2 = (ri + rj) ** 2
    ref_branch = d2 < s2
    eidx = (pairs[:, None] + np.arange(4)[None, :]).ravel()
    gx = xg[eidx].reshape(-1, 4, 2)
    rx = xr[eidx].reshape(-1, 4, 2)
    nx = n[eidx].reshape(-1, 4, 2)
    gpu_branch = (gx != nx).any(axis=(1, 2))
    near = (np.abs(np.sqrt(d2) - np.abs(ri + rj)) < 1e-4) | (d2 < 1e-6)
    away = ~near
    err = np.abs(gx - rx).max(axis=(1, 2))
    print(f"pairs: {len(pairs)}, overlapping {int(ref_branch.sum())}, near a boundary {int(near.sum())}, "
          f"branch disagreements away from it {int((gpu_branch != ref_branch)[away].sum())}, "
          f"max |diff| away {err[away].max():.2e}")
    assert ref_branch[away].sum() > 10000 and (~ref_branch[away]).sum() > 10000  # both branches exercised
    assert np.array_equal(gpu_branch[away], ref_branch[away])
    assert err[away].max() <= TOL

    # walls: inputs (c, r) at edges e0, e0 + 1, parameters (v, p) in factor order
    wpar = np.repeat(walls, N, axis=0)  # walls are added wall-major (all circles of wall 0, then wall 1, ...)
    c, r = n[wall_f], n[wall_f + 1, 0]
    inner = (wpar[:, :2] * (c - wpar[:, 2:])).sum(1)
    ref_w = inner + r > 0
    eidx = (wall_f[:, None] + np.arange(2)[None, :]).ravel()
    gx, rx, nx = (a[eidx].reshape(-1, 2, 2) for a in (xg, xr, n))
    gpu_w = (gx != nx).any(axis=(1, 2))
    away = np.abs(inner + r) >= 1e-4
    err = np.abs(gx - rx).max(axis=(1, 2))
    assert ref_w[away].sum() > 100 and (~ref_w[away]).sum() > 100
    assert np.array_equal(gpu_w[away], ref_w[away])
    assert err[away].max() <= TOL

    # radius factors: prox of -r^2, rho n / (rho - 2) clamped at 0
    nr = n[rad_e, 0]
    away = np.abs(nr) >= 1e-4
    err = np.abs(xg[rad_e] - xr[rad_e]).max(1)
    assert (nr[away] < 0).sum() > 50 and (nr[away] > 0).sum() > 50
    assert np.array_equal(xg[rad_e][away, 0] == 0.0, xr[rad_e][away, 0] == 0.0)
    assert err[away].max() <= TOL
