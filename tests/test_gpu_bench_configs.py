"""GPU parity at the benchmark's own configurations, against the reference's
CPU path (oracle/_ref: core/paradmm.c + packing/host.c compiled from their
sources; updateGOpenMP advances it, bit-identical to updateG because every
variable's consensus sum runs in one thread in insertion order,
core/paradmm.c:949-1092).

  * the bench workload: N = 8000 circles in a 2 x 1 box, radii in
    [0, 0.01], rho 10 / 5, alpha 1, exponent 2, the bench's seed --
    teacher-forced (one engine sweep from reference iterate k against
    iterate k + 1) at k = 0 .. 4 and 50, overlapping pairs present; and five
    free-running sweeps from the seeded start, checked on the consensus Z;
  * configuration 1: N = 2000 in the unit box, radii in [0, 0.05] --
    teacher-forced at k = 0 .. 7, 50 and 500, and eight free-running sweeps
    checked on Z;
  * the batched workload: instances of the 512-instance time-to-residual
    batch (N uniform in [20, 400]), each set inside the batch handle to a
    reference iterate (Z^k and U^k through paradmm_gpu_warm_start_duals) and
    swept together with the rest of the batch on the per-instance schedule;
    its next two consensus iterates are compared with the reference's.

Tolerance: the packing engine's per-iterate max |difference| 1e-4 (FP32
edge state).  Free-running, only Z is held to it: at these sizes the
random start has pairs with nearly coincident centres, whose projection
direction amplifies FP32 rounding of the edge state, and FP32 arithmetic on
its own -- a numpy restatement with none of the engine's code -- leaves the
reference's per-edge X and U by 1.2e-4 at the second sweep of
configuration 1 while Z stays within 2e-7
(test_fp32_horizon.py::test_fp32_per_edge_horizon_at_configuration1).  The
N = 8000 case holds two FP64 host graphs (about 13 GB each) and runs about
50 reference sweeps on up to 8 host threads.
"""
import ctypes as C
import os

import numpy as np
import pytest

import engine_b200 as eb
import oracle_lib

pytestmark = pytest.mark.gpu

TOL_F32 = 1e-4
# From reference iterates 2 .. 4 of the N = 8000 workload one FP32 sweep of
# the per-edge arrays is limited by FP32 arithmetic itself: the numpy FP32
# restatement (test_fp32_horizon.Twin), teacher-forced from iterate 2, lands
# 1.66e-4 from the reference's X, M, U and N (Z 1.2e-7) -- the same figure
# the engine reaches.  Z stays held to TOL_F32 there.
TOL_EDGE_N8000 = {2: 4e-4, 3: 4e-4, 4: 4e-4}
RHO, RHO_R, ALPHA, EXP = 10.0, 5.0, 1.0, 2.0
THREADS = os.cpu_count() or 1


def _maxdiff(G, H) -> float:
    """max |difference| over X, M, N, U, Z of two graphs (no full copies)."""
    worst = 0.0
    for k in ("X", "M", "N", "U", "Z"):
        a, b = G.arr(k), H.arr(k)
        step = 1 << 24
        flat_a, flat_b = a.reshape(-1), b.reshape(-1)
        for i in range(0, flat_a.size, step):
            worst = max(worst, float(np.max(np.abs(flat_a[i:i + step] - flat_b[i:i + step]))))
    return worst


def _overlapping_pairs(c: np.ndarray) -> int:
    n = 0
    for i in range(0, len(c), 512):
        d = np.hypot(c[i:i + 512, None, 0] - c[None, :, 0], c[i:i + 512, None, 1] - c[None, :, 1])
        s = c[i:i + 512, None, 2] + c[None, :, 2]
        ii = np.arange(i, min(i + 512, len(c)))[:, None]
        n += int(np.sum((d < s) & (np.arange(len(c))[None, :] > ii)))
    return n


def _pair(N, W, H, rmax, seed):
    walls = eb.box_walls(W, H)
    circles = eb.seeded_circles(N, W, H, rmax, seed)
    pg = eb.PackingGraph(N, walls, EXP)
    pg.init_seeded(circles, RHO, RHO_R, ALPHA)
    orc = oracle_lib.OraclePacking(oracle_lib.best(), N, walls, EXP)
    orc.init(seed, W, H, rmax, RHO, RHO_R, ALPHA)
    assert np.array_equal(orc.circles(), circles)
    return pg, orc, circles


def _copy_state(dst, src):
    for k in ("X", "M", "N", "U", "Z"):
        dst.arr(k)[:] = src.arr(k)


def _zdiff(G, H) -> float:
    return float(np.max(np.abs(G.arr("Z") - H.arr("Z"))))


def _teacher_forced(pg, orc, ks, N, tol_edge=None):
    """One engine sweep from each reference iterate k in ks (ascending)
    against reference iterate k + 1; Z is held to TOL_F32, the per-edge
    arrays to tol_edge.get(k, TOL_F32).  Returns the worst max |difference|."""
    tol_edge = tol_edge or {}
    worst, done = 0.0, 0
    with eb.Handle.from_graph(pg.G, engine=eb.ENGINE_PACKING) as h:
        assert h.engine() == eb.ENGINE_PACKING
        for k in ks:
            orc.run(k - done, THREADS, trace=False)
            _copy_state(pg.G, orc.G)
            h.upload(pg.G)
            h.iterate(1)
            h.download(pg.G)
            orc.run(1, THREADS, trace=False)
            done = k + 1
            d, z = _maxdiff(pg.G, orc.G), _zdiff(pg.G, orc.G)
            print(f"N={N}: teacher-forced from iterate {k}: max |diff| {d:.2e} (Z {z:.2e})")
            assert z <= TOL_F32, f"N={N}, teacher-forced from iterate {k}: max |diff| of Z {z}"
            assert d <= tol_edge.get(k, TOL_F32), f"N={N}, teacher-forced from iterate {k}: max |diff| {d}"
            worst = max(worst, d)
    return worst


def _free_running_z(pg, orc, sweeps, N):
    with eb.Handle.from_graph(pg.G, engine=eb.ENGINE_PACKING) as h:
        for k in range(sweeps):
            h.iterate(1)
            h.download(pg.G)
            orc.run(1, THREADS, trace=False)
            d = _zdiff(pg.G, orc.G)
            assert d <= TOL_F32, f"N={N}, free-running sweep {k + 1}: max |diff| of Z {d}"


def test_bench_workload_n8000():
    import bench
    N = bench.N_CIRCLES
    pg, orc, circles = _pair(N, bench.BOX_W, bench.BOX_H, bench.RMAX, bench.SEED)
    assert _overlapping_pairs(circles) > 1000  # the overlap branch of the pair operator is exercised
    _free_running_z(pg, orc, 5, N)
    orc.init(bench.SEED, bench.BOX_W, bench.BOX_H, bench.RMAX, RHO, RHO_R, ALPHA)
    worst = _teacher_forced(pg, orc, [0, 1, 2, 3, 4, 50], N, TOL_EDGE_N8000)
    print(f"N={N}: teacher-forced worst max|diff| {worst:.2e}")
    pg.close()
    orc.close()


def test_configuration1_n2000():
    N = 2000
    pg, orc, circles = _pair(N, 1.0, 1.0, 0.05, 7)
    assert _overlapping_pairs(circles) > 1000
    _free_running_z(pg, orc, 8, N)
    orc.init(7, 1.0, 1.0, 0.05, RHO, RHO_R, ALPHA)
    worst = _teacher_forced(pg, orc, [0, 1, 2, 3, 4, 5, 6, 7, 50, 500], N)
    print(f"N={N}: teacher-forced worst max|diff| {worst:.2e}")


@pytest.mark.parametrize("schedule,cluster,coop_min_n", [(eb.SCHEDULE_INSTANCE, 2, 200), (eb.SCHEDULE_INSTANCE, 1, 0),
                                                       (eb.SCHEDULE_ONCHIP, 0, 0)])
def test_batched_instances_teacher_forced_inside_the_batch(schedule, cluster, coop_min_n):
    """Instances of the time-to-residual batch (seed 900000), picked to cover
    the small-instance solver (N <= 40), single CTAs and whole clusters of the
    tiled per-instance schedule, and every group size of the cluster-resident
    one, set to reference iterates k in {0, 40, 300} inside the 512-instance
    handle."""
    from engine_b200 import learned
    inst = learned.make_instances(512, 900000)
    sizes = np.array([d["n_circles"] for d in inst])
    picks = [int(np.argmin(sizes)), int(np.argmin(np.abs(sizes - 37))), int(np.argmin(np.abs(sizes - 120))),
             int(np.argmin(np.abs(sizes - 150))), int(np.argmin(np.abs(sizes - 199))),
             int(np.argmin(np.abs(sizes - 260))), int(np.argmin(np.abs(sizes - 330))), int(np.argmax(sizes))]
    picks = list(dict.fromkeys(picks))
    b = learned.Batch(inst, device=0, schedule=schedule, cluster=cluster, coop_min_n=coop_min_n)
    h = eb.Handle(b.h.value, b.lib)
    try:
        orcs = {}
        for i in picks:
            d = inst[i]
            o = oracle_lib.OraclePacking(oracle_lib.best(), d["n_circles"], eb.box_walls(d["aspect"], 1.0), EXP)
            o.init(1, d["aspect"], 1.0, 0.05, RHO, RHO_R, ALPHA)
            o.set_circles_plain(d["init"])
            orcs[i] = o
        done = 0
        for k in (0, 40, 300):
            for i in picks:
                orcs[i].run(k - done, THREADS, trace=False)
                pair, wall, rad = orcs[i].duals()
                h.warm_start_duals(i, orcs[i].circles(), pair, wall, rad, 0)
            done = k
            for step in (1, 2):
                b.solve(1, -1.0)
                for i in picks:
                    orcs[i].run(1, THREADS, trace=False)
                    got = h.circles(i, inst[i]["n_circles"])
                    diff = float(np.max(np.abs(got - orcs[i].circles())))
                    assert diff <= TOL_F32, f"instance {i} (N={sizes[i]}), iterate {k} + {step}: max |diff| {diff}"
            done += 2
    finally:
        h.ptr = C.c_void_p()  # the batch owns the handle
        b.close()
