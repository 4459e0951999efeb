"""GPU: the warm start with duals (paradmm_gpu_warm_start_duals) against the
reference's own initialize_X_N_Z_M_U_optimal (core/paradmm.c:266-375), run
by the oracle on the same graph, and a teacher-forced sweep after it.

The engine keeps its edge state in FP32, so the comparison tolerance is the
packing engine's per-iterate 1e-4 (max |difference| of X, M, N, U, Z).
"""
import ctypes as C

import numpy as np
import pytest

import engine_b200 as eb
import oracle_lib

pytestmark = pytest.mark.gpu

TOL_F32 = 1e-4
RHO, RHO_R, ALPHA, EXP = 10.0, 5.0, 1.0, 2.0


def _problem(N, seed, W=1.0, H=1.0):
    walls = eb.box_walls(W, H)
    pg = eb.PackingGraph(N, walls, EXP)
    pg.init_seeded(eb.seeded_circles(N, W, H, 0.05, seed), RHO, RHO_R, ALPHA)
    orc = oracle_lib.OraclePacking(oracle_lib.best(), N, walls, EXP)
    orc.init(seed, W, H, 0.05, RHO, RHO_R, ALPHA)
    return pg, orc


def _maxdiff(a, b):
    return max(float(np.max(np.abs(a[k] - b[k]))) for k in ("X", "M", "N", "U", "Z"))


@pytest.mark.parametrize("iters,with_uinit", [(0, True), (1, False), (6, False), (6, True)])
def test_warm_start_duals_match_reference_optimal_init(iters, with_uinit):
    """Zinit (and Uinit) from a reference iterate mid-solve: the engine's
    device-side initialisation equals the reference's initialize_X_N_Z_M_U_optimal
    with the same maxiter, then one sweep of each agrees too."""
    N = 60
    pg, orc = _problem(N, 31)
    orc.run(250, trace=False)
    zinit = orc.G.arr("Z").copy()
    uinit = orc.G.arr("U").copy() if with_uinit else np.zeros_like(orc.G.arr("U"))
    # the reference radius edges carry equal dims; the engine keeps one
    assert np.array_equal(uinit[:N, 0], uinit[:N, 1])
    circles = orc.circles()
    pair, wall, rad = orc.duals() if with_uinit else (None, None, None)

    orc.lib.initialize_X_N_Z_M_U_optimal(orc.graph_ptr(), zinit.ctypes.data_as(C.POINTER(C.c_double)),
                                         uinit.ctypes.data_as(C.POINTER(C.c_double)), iters)
    if iters == 0:  # the reference leaves U unset then (core/paradmm.c:278); the contract is U = Uinit
        G = orc.G
        G.arr("U")[:] = uinit
        G.arr("N")[:] = G.arr("X") - uinit
        G.arr("M")[:] = G.arr("X") + uinit
    with eb.Handle.from_graph(pg.G, engine=eb.ENGINE_PACKING) as h:
        h.warm_start_duals(0, circles, pair, wall, rad, iters)
        h.download(pg.G)
        d0 = _maxdiff(pg.G.state(), orc.state())
        assert d0 <= TOL_F32, f"after the initialisation: max |diff| {d0}"
        h.iterate(1)
        h.download(pg.G)
    orc.sweep()
    d1 = _maxdiff(pg.G.state(), orc.state())
    assert d1 <= TOL_F32, f"one sweep after it: max |diff| {d1}"
    # the refined duals are not trivially zero here: some pairs overlap at Zinit
    if iters > 0:
        assert float(np.max(np.abs(orc.G.arr("U")))) > 1e-4


def test_warm_start_all_duals_batch_matches_single_instances():
    """paradmm_gpu_warm_start_all_duals on a batch gives every instance the
    state paradmm_gpu_warm_start_duals gives it alone (same FP32 map)."""
    from engine_b200 import learned
    inst = learned.make_instances(6, 77, nmin=20, nmax=150)
    rng = np.random.default_rng(2)
    circ = [d["init"] + rng.normal(0, 0.01, d["init"].shape) * np.array([1, 1, 0]) for d in inst]
    b = learned.Batch(inst, device=0, schedule=eb.SCHEDULE_INSTANCE)
    b.warm_start(np.concatenate(circ), radius_duals=0, dual_iters=8)
    b.solve(30, -1.0)
    got = b.circles()
    b.close()
    for d, c, g in zip(inst, circ, got):
        one = learned.Batch([d], device=0, schedule=eb.SCHEDULE_INSTANCE)
        h = eb.Handle(one.h.value, one.lib)
        h.warm_start_duals(0, c, dual_iters=8)
        h.ptr = C.c_void_p()  # the batch owns the handle
        one.solve(30, -1.0)
        want = one.circles()[0]
        one.close()
        assert np.array_equal(g, want)
