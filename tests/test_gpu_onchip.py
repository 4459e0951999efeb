"""GPU: the cluster-resident per-instance schedule (PARADMM_SCHEDULE_ONCHIP,
onchip_kernels.cu), where every instance's pair state stays in the shared
memory of a group of 1-16 CTAs of a thread-block cluster for its solve.

Parity against the reference is in test_gpu_bench_configs.py (instances of
the time-to-residual batch teacher-forced inside the batch, every size
class).  Here: batches equal their instances solved alone, bit for bit
(stop decisions included); the schedule agrees with the tiled per-instance
schedule to FP32 rounding over a free-running horizon and reaches the same
tolerance; the in-call fallback and the penalty balancing behave as on the
tiled schedule; sizes beyond one cluster are refused."""
import numpy as np
import pytest

import engine_b200 as eb

pytestmark = pytest.mark.gpu

RHO, RHO_R, ALPHA, EXP = 10.0, 5.0, 1.0, 2.0


def _descs(n, seed, nmin=20, nmax=400):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        N = int(rng.integers(nmin, nmax + 1))
        asp = float(rng.uniform(1, 2))
        out.append(dict(n_circles=N, walls=eb.box_walls(asp, 1.0), exponent=EXP, rho=RHO, rho_radius=RHO_R,
                        alpha=ALPHA, init=eb.seeded_circles(N, asp, 1.0, 0.05, seed * 1000 + i)))
    return out


def test_onchip_batch_equals_single_instances():
    descs = _descs(40, 3)
    with eb.Handle.packing(descs, schedule=eb.SCHEDULE_ONCHIP) as hb:
        s = hb.solve(3000, 1e-5)
        assert s["status"] == eb.OK
        st = hb.instance_stats()
        circ = [hb.circles(i, d["n_circles"]) for i, d in enumerate(descs)]
    assert sum(x["converged"] for x in st) >= 10
    for i in (0, 7, 13, 21, 33):
        with eb.Handle.packing([descs[i]], schedule=eb.SCHEDULE_ONCHIP) as h1:
            h1.solve(3000, 1e-5)
            one = h1.instance_stats()[0]
            assert one["iterations"] == st[i]["iterations"], i
            assert np.array_equal(h1.circles(0, descs[i]["n_circles"]), circ[i]), i


def test_onchip_follows_the_tiled_schedule():
    """Same instances on both per-instance schedules: the arithmetic is the
    same up to the grouping of the FP32 partial sums, so the free-running
    trajectories agree to FP32 rounding early and both reach the tolerance."""
    descs = _descs(24, 5, 20, 400)
    res = {}
    for sched in (eb.SCHEDULE_INSTANCE, eb.SCHEDULE_ONCHIP):
        with eb.Handle.packing(descs, schedule=sched) as h:
            h.iterate(3)
            early = [h.circles(i, d["n_circles"]) for i, d in enumerate(descs)]
            s = h.solve(20000, 1e-5)
            res[sched] = (early, h.instance_stats())
    e1, st1 = res[eb.SCHEDULE_INSTANCE]
    e2, st2 = res[eb.SCHEDULE_ONCHIP]
    d = max(float(np.max(np.abs(a - b))) for a, b in zip(e1, e2))
    assert d <= 1e-4, f"3 sweeps: max |diff| {d}"
    c1 = sum(x["converged"] for x in st1)
    c2 = sum(x["converged"] for x in st2)
    assert abs(c1 - c2) <= 2 and c2 >= len(descs) - 3
    for a in st2:
        if a["converged"]:
            assert a["primal"] + a["dual"] <= 1e-5


def test_onchip_fallback_and_balancing():
    descs = _descs(16, 9, 20, 300)
    rng = np.random.default_rng(1)
    warm = np.concatenate([d["init"] + rng.normal(0, 0.3, d["init"].shape) * np.array([1, 1, 0]) for d in descs])
    for sched in (eb.SCHEDULE_ONCHIP,):
        with eb.Handle.packing(descs, schedule=sched) as h:
            lib = h.lib
            import ctypes as C
            lib.paradmm_gpu_warm_start_all.argtypes = [C.c_void_p, C.POINTER(C.c_double), C.c_int]
            w = np.ascontiguousarray(warm)
            eb.check(lib.paradmm_gpu_warm_start_all(h.ptr, w.ctypes.data_as(C.POINTER(C.c_double)), 1))
            h.set_fallback(50)
            h.set_rho_balance(20, 10.0, -1, 2)
            h.solve(400, -1.0)
            fb = h.instance_fallbacks()
            assert fb.all()  # every instance restarted from its plain start after 50 sweeps
            circ = [h.circles(i, d["n_circles"]) for i, d in enumerate(descs)]
        # from the restart on, each instance is the plain solve of 350 sweeps
        with eb.Handle.packing(descs, schedule=sched) as hp:
            hp.set_rho_balance(20, 10.0, -1, 2)
            hp.solve(350, -1.0)
            for i, d in enumerate(descs):
                assert np.array_equal(circ[i], hp.circles(i, d["n_circles"])), i


def test_onchip_refuses_instances_beyond_one_cluster():
    d = _descs(1, 2, 2000, 2000)
    with pytest.raises(eb.ParadmmError) as e:
        eb.Handle.packing(d, schedule=eb.SCHEDULE_ONCHIP)
    assert "cluster-resident" in str(e.value)
