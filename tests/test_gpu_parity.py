"""GPU parity: the engine against the reference's own CPU path.

The oracle is the reference C (core/paradmm.c + packing/host.c) compiled
from its own sources into oracle/_ref (or, without it, the C restatement
oracle/paradmm_port.c, which tests/test_oracle.py pins bit-for-bit to it).

Tolerances:
  generic engine, FP64   bit-identical (reference summation order, no FMA)
  packing engine, FP32   max |difference| <= 1e-4 per iterate (north star:
                         FP32 edge state, per-iterate max abs diff 1e-4)
"""
import ctypes as C

import numpy as np
import pytest

import engine_b200 as eb
import oracle_lib

pytestmark = pytest.mark.gpu

TOL_F32 = 1e-4
RHO, RHO_R, ALPHA, EXP = 10.0, 5.0, 1.0, 2.0


def problem(N, seed, W=1.0, H=1.0, rmax=0.05, order=0, lib=None):
    walls = eb.box_walls(W, H)
    circles = eb.seeded_circles(N, W, H, rmax, seed)
    pg = eb.PackingGraph(N, walls, EXP, order=order)
    pg.init_seeded(circles, RHO, RHO_R, ALPHA)
    orc = oracle_lib.OraclePacking(lib or oracle_lib.best(), N, walls, EXP, order=order)
    orc.init(seed, W, H, rmax, RHO, RHO_R, ALPHA)
    return pg, orc, circles


def maxdiff(a: dict, b: dict) -> float:
    return max(float(np.max(np.abs(a[k] - b[k]))) for k in ("X", "M", "N", "U", "Z"))


def assert_same(a: dict, b: dict):
    for k in ("X", "M", "N", "U", "Z"):
        assert np.array_equal(a[k], b[k]), f"{k} differs (max {np.max(np.abs(a[k] - b[k]))})"


# ------------------------------------------------------------ generic FP64
@pytest.mark.parametrize("order", [0, 1])
def test_generic_f64_bit_identical_to_reference(order):
    """The FP64 engine follows the reference bit for bit through 2500 sweeps
    (checked at 300 and at 2500), past the chaotic early phase."""
    pg, orc, _ = problem(24, 11, order=order)
    assert_same(pg.G.state(), orc.state())
    with eb.Handle.from_graph(pg.G, engine=eb.ENGINE_GENERIC_F64) as h:
        assert h.engine() == eb.ENGINE_GENERIC_F64
        for n in (300, 2200):
            h.iterate(n)
            h.download(pg.G)
            orc.run(n, trace=False)
            assert_same(pg.G.state(), orc.state())


def test_generic_f64_random_full_state():
    """Reference-style random state (both radius dims differ): all dims evolve."""
    pg, orc, _ = problem(16, 5)
    rng = np.random.default_rng(3)
    st = {k: rng.uniform(-1, 2, size=v.shape) for k, v in orc.state().items()}
    orc.set_state(st)
    for k, v in st.items():
        pg.G.arr(k)[:] = v
    with eb.Handle.from_graph(pg.G) as h:  # AUTO must fall back to the generic engine
        assert h.engine() == eb.ENGINE_GENERIC_F64
        h.iterate(40)
        h.download(pg.G)
    orc.run(40, trace=False)
    assert_same(pg.G.state(), orc.state())


@pytest.mark.parametrize("phase", ["updateX", "updateM", "updateXM", "updateZ", "updateU", "updateN", "updateUN",
                                   "updateG"])
def test_dropin_phase_functions_bit_identical(phase):
    pg, orc, _ = problem(12, 7)
    rng = np.random.default_rng(9)
    st = {k: rng.uniform(0, 1, size=v.shape) for k, v in orc.state().items()}
    orc.set_state(st)
    for k, v in st.items():
        pg.G.arr(k)[:] = v
    lib = eb.load()
    o = eb.opts(engine=eb.ENGINE_GENERIC_F64)
    lib.paradmm_set_sweep_options(C.byref(o))
    try:
        getattr(lib, phase)(C.byref(pg.G))
        assert eb.last_status() == eb.OK, eb.last_error()
    finally:
        lib.paradmm_set_sweep_options(None)
    getattr(orc.lib, phase)(orc.graph_ptr())
    assert_same(pg.G.state(), orc.state())


def test_dropin_updateGOpenMP_generic():
    pg, orc, _ = problem(20, 8)
    lib = eb.load()
    o = eb.opts(engine=eb.ENGINE_GENERIC_F64)
    lib.paradmm_set_sweep_options(C.byref(o))
    try:
        lib.updateGOpenMP(C.byref(pg.G), 25, 8)
        assert eb.last_status() == eb.OK, eb.last_error()
    finally:
        lib.paradmm_set_sweep_options(None)
    orc.run(25, trace=False)
    assert_same(pg.G.state(), orc.state())


# ---------------------------------------------------------- packing FP32
@pytest.mark.parametrize("bw", [32, 64, 128])
def test_packing_teacher_forced_one_sweep(bw):
    """From oracle iterate k, one engine sweep vs oracle iterate k+1."""
    N = 150
    pg, orc, _ = problem(N, 21)
    worst = 0.0
    done = 0
    for k in (0, 1, 5, 40, 200, 600):
        orc.run(k - done, trace=False)
        done = k
        st = orc.state()
        for key, v in st.items():
            pg.G.arr(key)[:] = v
        with eb.Handle.from_graph(pg.G, engine=eb.ENGINE_PACKING, block_width=bw) as h:
            h.iterate(1)
            h.download(pg.G)
        orc.sweep()
        done += 1
        d = maxdiff(pg.G.state(), orc.state())
        worst = max(worst, d)
        assert d <= TOL_F32, f"k={k}: max diff {d}"
    print(f"teacher-forced worst max|diff| = {worst:.3e}")


@pytest.mark.parametrize("container,exponent", [("triangle", 2.0), ("box", 1.0), ("triangle", 1.5)])
def test_packing_teacher_forced_containers_and_exponents(container, exponent):
    """The demo's triangle container (walls with slanted normals,
    packing/host.c:141-149) and radius exponents 1 (closed-form powers) and
    1.5 (powf Newton steps), teacher-forced like the box case."""
    N, seed = 130, 33
    W, H = (1.0, 0.87) if container == "triangle" else (1.0, 1.0)
    walls = eb.triangle_walls() if container == "triangle" else eb.box_walls(W, H)
    circles = eb.seeded_circles(N, W, H, 0.05, seed)
    pg = eb.PackingGraph(N, walls, exponent)
    pg.init_seeded(circles, RHO, RHO_R, ALPHA)
    orc = oracle_lib.OraclePacking(oracle_lib.best(), N, walls, exponent)
    orc.init(seed, W, H, 0.05, RHO, RHO_R, ALPHA)
    done, checked = 0, 0
    for k in (0, 3, 30, 150):
        orc.run(k - done, trace=False)
        done = k
        st = orc.state()
        if not all(np.isfinite(v).all() for v in st.values()):
            break
        for key, v in st.items():
            pg.G.arr(key)[:] = v
        with eb.Handle.from_graph(pg.G, engine=eb.ENGINE_PACKING) as h:
            h.iterate(1)
            h.download(pg.G)
        orc.sweep()
        done += 1
        ref = orc.state()
        if not all(np.isfinite(v).all() for v in ref.values()):
            break
        d = maxdiff(pg.G.state(), ref)
        assert d <= TOL_F32, f"k={k}: max diff {d}"
        checked += 1
    assert checked >= 2


def test_packing_teacher_forced_every_iterate_to_2000():
    """At every k < 2000: the reference's iterate k uploaded, one engine
    sweep, against the reference's iterate k + 1 (one handle, re-uploaded
    each step), through the chaotic early phase and on to convergence."""
    N = 40
    pg, orc, _ = problem(N, 17)
    worst, worst_k = 0.0, -1
    with eb.Handle.from_graph(pg.G, engine=eb.ENGINE_PACKING) as h:
        for k in range(2000):
            for key, v in orc.state().items():
                pg.G.arr(key)[:] = v
            h.upload(pg.G)
            h.iterate(1)
            h.download(pg.G)
            orc.sweep()
            d = maxdiff(pg.G.state(), orc.state())
            if d > worst:
                worst, worst_k = d, k
            assert d <= TOL_F32, f"k={k}: max diff {d}"
    print(f"teacher-forced, every k < 2000: worst max|diff| = {worst:.3e} at k = {worst_k}")


def test_packing_free_running_from_init():
    """Free-running from the random init.  The early phase is chaotic: an
    FP32 re-evaluation of the same formulas on the CPU leaves 1e-4 of the
    FP64 reference at iterate 9 for this instance, so the horizon is 8."""
    N = 120
    pg, orc, _ = problem(N, 4)
    with eb.Handle.from_graph(pg.G, engine=eb.ENGINE_PACKING) as h:
        for k in range(8):
            h.iterate(1)
            h.download(pg.G)
            orc.sweep()
            d = maxdiff(pg.G.state(), orc.state())
            assert d <= TOL_F32, f"iterate {k + 1}: max diff {d}"


def test_packing_free_running_near_fixed_point():
    """50 free-running FP32 sweeps from the reference's iterate 1500."""
    N = 80
    pg, orc, _ = problem(N, 6)
    orc.run(1500, trace=False)
    for k, v in orc.state().items():
        pg.G.arr(k)[:] = v
    worst = 0.0
    with eb.Handle.from_graph(pg.G, engine=eb.ENGINE_PACKING) as h:
        for k in range(50):
            h.iterate(1)
            h.download(pg.G)
            orc.sweep()
            d = maxdiff(pg.G.state(), orc.state())
            worst = max(worst, d)
            assert d <= TOL_F32, f"iterate {1500 + k + 1}: max diff {d}"
    print(f"near-fixed-point free-running worst max|diff| = {worst:.3e}")


def test_dropin_updateG_runs_packing_engine():
    """updateG / updateGOpenMP (default engine: packing FP32) against the
    reference: 5 single sweeps from the init, then 30 sweeps in one call
    from a near-fixed-point state (the early phase is too chaotic for 35
    free-running FP32 sweeps, see test_packing_free_running_from_init)."""
    pg, orc, _ = problem(40, 2)
    lib = eb.load()
    lib.paradmm_set_sweep_options(None)
    for _ in range(5):
        lib.updateG(C.byref(pg.G))
        assert eb.last_status() == eb.OK, eb.last_error()
        orc.sweep()
    assert maxdiff(pg.G.state(), orc.state()) <= TOL_F32
    orc.run(1500, trace=False)
    for k, v in orc.state().items():
        pg.G.arr(k)[:] = v
    lib.updateGOpenMP(C.byref(pg.G), 30, 8)
    assert eb.last_status() == eb.OK, eb.last_error()
    orc.run(30, trace=False)
    assert maxdiff(pg.G.state(), orc.state()) <= TOL_F32
    lib.closeG(C.byref(pg.G))


def test_upload_download_roundtrip_without_sweep():
    pg, orc, _ = problem(30, 9)
    orc.run(7, trace=False)
    st = orc.state()
    for k, v in st.items():
        pg.G.arr(k)[:] = v
    with eb.Handle.from_graph(pg.G, engine=eb.ENGINE_PACKING) as h:
        for k in ("N", "U", "Z"):
            pg.G.arr(k)[:] = 0.0
        h.download(pg.G)
    got = pg.G.state()
    for k in ("N", "U", "Z"):
        assert np.max(np.abs(got[k] - st[k])) <= 1e-6 * max(1.0, np.max(np.abs(st[k])))


def test_structured_handle_matches_graph_handle():
    N = 90
    pg, orc, circles = problem(N, 13)
    desc = dict(n_circles=N, walls=eb.box_walls(1, 1), exponent=EXP, rho=RHO, rho_radius=RHO_R, alpha=ALPHA,
                init=circles)
    with eb.Handle.packing([desc], block_width=64) as hs, \
            eb.Handle.from_graph(pg.G, engine=eb.ENGINE_PACKING, block_width=64) as hg:
        hs.iterate(100)
        hg.iterate(100)
        hg.download(pg.G)
        a = hs.circles(0, N)
    Z = pg.G.arr("Z")
    b = np.stack([Z[0::2, 0], Z[0::2, 1], Z[1::2, 0]], axis=1)
    assert np.max(np.abs(a - b)) <= 1e-5


def test_batched_equals_single_instances():
    rng = np.random.default_rng(0)
    descs = []
    for i in range(6):
        N = int(rng.integers(20, 150))
        asp = float(rng.uniform(1, 2))
        descs.append(dict(n_circles=N, walls=eb.box_walls(asp, 1.0), exponent=EXP, rho=RHO, rho_radius=RHO_R,
                          alpha=ALPHA, init=eb.seeded_circles(N, asp, 1.0, 0.05, 100 + i)))
    with eb.Handle.packing(descs, block_width=64) as hb:
        hb.iterate(150)
        batched = [hb.circles(i, d["n_circles"]) for i, d in enumerate(descs)]
    for i, d in enumerate(descs):
        with eb.Handle.packing([d], block_width=64) as h1:
            h1.iterate(150)
            single = h1.circles(0, d["n_circles"])
        assert np.array_equal(batched[i], single), f"instance {i} differs"


def test_solve_reaches_tolerance_and_metrics():
    N = 50
    pg, orc, circles = problem(N, 31)
    desc = dict(n_circles=N, walls=eb.box_walls(1, 1), exponent=EXP, rho=RHO, rho_radius=RHO_R, alpha=ALPHA,
                init=circles)
    with eb.Handle.packing([desc]) as h:
        s = h.solve(40000, 1e-5)
        st = h.instance_stats()[0]
    assert s["converged"] == 1, s
    assert st["primal"] + st["dual"] <= 1e-5
    n, tr = orc.run(40000, tol=1e-5)
    m = tr[-1]
    print(f"engine FP32: iters {s['iterations']} r {st['primal']:.2e} s {st['dual']:.2e} "
          f"viol {st['max_violation']:.2e} total radius {st['total_radius']:.6f}")
    print(f"oracle FP64: iters {n} r {m[0]:.2e} s {m[1]:.2e} viol {m[2]:.2e} total radius {m[3]:.6f}")
    assert st["max_violation"] < 5e-3
    assert abs(st["total_radius"] - m[3]) / m[3] < 0.1


def test_nonfinite_is_reported():
    """Two coincident centres make the pair operator divide 0/0 (as the
    reference does, packing/host.c:123): the engine stops with ENONFINITE."""
    N = 10
    circles = eb.seeded_circles(N, 1, 1, 0.3, 1)
    circles[1, :2] = circles[0, :2]
    desc = dict(n_circles=N, walls=eb.box_walls(1, 1), exponent=EXP, rho=RHO, rho_radius=RHO_R, alpha=ALPHA,
                init=circles)
    with eb.Handle.packing([desc]) as h:
        s = h.solve(50, -1.0)
        assert s["status"] == eb.ENONFINITE
        assert eb.last_status() == eb.ENONFINITE


# ------------------------------------------------------ golden fixtures (GPU)
import glob as _glob  # noqa: E402
import os as _os  # noqa: E402

_GOLDEN = sorted(_glob.glob(_os.path.join(_os.path.dirname(__file__), "golden", "*.npz")))


@pytest.mark.parametrize("path", _GOLDEN, ids=[_os.path.basename(p) for p in _GOLDEN])
def test_generic_f64_reproduces_golden(path):
    """The exact engine reproduces the reference's own outputs bit for bit."""
    g = np.load(path)
    N = int(g["N"])
    pg = eb.PackingGraph(N, g["walls"], 2.0, order=int(g["order"]))
    lib = eb.load()
    lib.initialize_X_N_Z_M_U_zeros(C.byref(pg.G))
    lib.initialize_RHOS_APHAS(C.byref(pg.G), float(g["rho"]), float(g["alpha"]))
    pg.G.arr("RHOS")[:] = g["RHOS"]
    for k in ("X", "M", "N", "U", "Z"):
        pg.G.arr(k)[:] = g[f"init_{k}"]
    with eb.Handle.from_graph(pg.G, engine=eb.ENGINE_GENERIC_F64) as h:
        done = 0
        for s in g["snaps"]:
            h.iterate(int(s) - done)
            done = int(s)
            h.download(pg.G)
            st = pg.G.state()
            for k in ("X", "M", "N", "U", "Z"):
                assert np.array_equal(st[k], g[f"it{s}_{k}"]), f"{k} at sweep {s}"


@pytest.mark.parametrize("schedule", [eb.SCHEDULE_GRID, eb.SCHEDULE_INSTANCE])
def test_batched_solve_with_retiring_instances_equals_single(schedule):
    """Instances of a batch stop on their own residual; the ones still
    iterating must evolve exactly as if solved alone (same sweeps, same
    circles), however many of their neighbours have retired -- on both
    schedules (grid-wide persistent loop, one CTA per instance)."""
    rng = np.random.default_rng(11)
    descs = []
    for i in range(96):
        N = int(rng.integers(20, 130))
        asp = float(rng.uniform(1, 2))
        descs.append(dict(n_circles=N, walls=eb.box_walls(asp, 1.0), exponent=EXP, rho=RHO, rho_radius=RHO_R,
                          alpha=ALPHA, init=eb.seeded_circles(N, asp, 1.0, 0.05, 500 + i)))
    with eb.Handle.packing(descs, schedule=schedule) as hb:
        hb.solve(8000, 1e-5)
        batched = hb.instance_stats()
        circ = [hb.circles(i, d["n_circles"]) for i, d in enumerate(descs)]
    n_conv = sum(s["converged"] for s in batched)
    assert n_conv >= len(descs) // 2  # many retire early: that is the case under test
    for i in range(0, len(descs), 5):
        with eb.Handle.packing([descs[i]], schedule=schedule) as h1:
            h1.solve(8000, 1e-5)
            single = h1.instance_stats()[0]
            c1 = h1.circles(0, descs[i]["n_circles"])
        assert batched[i]["iterations"] == single["iterations"], (i, batched[i], single)
        assert batched[i]["converged"] == single["converged"], i
        assert np.array_equal(circ[i], c1), i


def test_autotune_keeps_state_and_picks_a_valid_schedule():
    """The schedule autotuner probes each candidate from a snapshot of the
    state and restores it: a solve after tuning equals the same solve on a
    fresh handle built with the chosen configuration, bit for bit."""
    rng = np.random.default_rng(3)
    descs = []
    for i in range(24):
        n = int(rng.integers(12, 260))
        asp = float(rng.uniform(1, 2))
        descs.append(dict(n_circles=n, walls=eb.box_walls(asp, 1.0), exponent=2.0, rho=10.0, rho_radius=5.0,
                          alpha=1.0, init=eb.seeded_circles(n, asp, 1.0, 0.05, 500 + i)))
    h = eb.Handle.packing(descs)
    t = h.autotune(30)
    assert t["candidates"] >= 2 and t["schedule"] in (eb.SCHEDULE_GRID, eb.SCHEDULE_INSTANCE)
    assert 0 < t["ms"] <= t["worst_ms"]
    s1 = h.solve(200, 1e-5)
    c1 = [h.circles(i, d["n_circles"]) for i, d in enumerate(descs)]
    kw = dict(schedule=t["schedule"])
    if t["schedule"] == eb.SCHEDULE_INSTANCE:
        kw.update(cluster_size=t["cluster_size"], coop_min_n=t["coop_min_n"])
    g = eb.Handle.packing(descs, **kw)
    s2 = g.solve(200, 1e-5)
    c2 = [g.circles(i, d["n_circles"]) for i, d in enumerate(descs)]
    assert s1["iterations"] == s2["iterations"]
    for a, b in zip(c1, c2):
        assert np.array_equal(a, b)
    h.close()
    g.close()


def test_graph_replayed_solves_equal_direct_launches():
    """Per-instance solves replay a captured CUDA graph once their parameters
    repeat; repeated solves give the same results as direct launches, and
    each call launches one kernel."""
    descs = []
    for i in range(10):
        n = 15 + 9 * i
        descs.append(dict(n_circles=n, walls=eb.box_walls(1.3, 1.0), exponent=2.0, rho=10.0, rho_radius=5.0,
                          alpha=1.0, init=eb.seeded_circles(n, 1.3, 1.0, 0.05, 40 + i)))
    out = []
    for no_graphs in (False, True):
        h = eb.Handle.packing(descs, schedule=eb.SCHEDULE_INSTANCE, no_graphs=no_graphs)
        l0 = h.launches()
        res = []
        for _ in range(4):
            h.solve(60, 1e-5)
            res.append([h.circles(i, d["n_circles"]).copy() for i, d in enumerate(descs)])
        assert h.launches() - l0 == 4
        out.append(res)
        h.close()
    for ra, rb in zip(*out):
        for a, b in zip(ra, rb):
            assert np.array_equal(a, b)


def test_config0_fixed_point():
    """Configuration 0 (N = 100, unit square) solved to r + s <= 1e-5: the
    FP64 generic engine stops at the same sweep with the same residuals and
    metrics as the reference's CPU updateG; the FP32 packing engine reaches
    the tolerance too, feasible, with total radius near the FP64 one."""
    N = 100
    pg, orc, circles = problem(N, 3)
    with eb.Handle.from_graph(pg.G, engine=eb.ENGINE_GENERIC_F64) as g:
        s64 = g.solve(20000, 1e-5)
        st64 = g.stats()
    n, tr = orc.run(20000, tol=1e-5)
    m = tr[-1]
    assert s64["converged"] == 1 and s64["iterations"] == n
    assert abs(st64["primal"] - m[0]) <= 1e-12 and abs(st64["dual"] - m[1]) <= 1e-12
    assert abs(st64["max_violation"] - m[2]) <= 1e-12 and abs(st64["total_radius"] - m[3]) <= 1e-9
    desc = dict(n_circles=N, walls=eb.box_walls(1, 1), exponent=EXP, rho=RHO, rho_radius=RHO_R, alpha=ALPHA,
                init=circles)
    with eb.Handle.packing([desc]) as h:
        s32 = h.solve(20000, 1e-5)
        st32 = h.instance_stats()[0]
    assert s32["converged"] == 1 and st32["primal"] + st32["dual"] <= 1e-5
    assert st32["max_violation"] < 2e-3
    assert abs(st32["total_radius"] - m[3]) / m[3] < 0.02


def test_create_packing_tuned_picks_tile_side_and_schedule():
    """paradmm_gpu_create_packing_tuned probes tile sides 64 and 128 and the
    schedules, keeps the fastest handle in its initial state: its solve
    equals a fresh handle built with the chosen configuration."""
    rng = np.random.default_rng(4)
    descs = []
    for i in range(16):
        n = int(rng.integers(20, 200))
        descs.append(dict(n_circles=n, walls=eb.box_walls(1.2, 1.0), exponent=2.0, rho=10.0, rho_radius=5.0,
                          alpha=1.0, init=eb.seeded_circles(n, 1.2, 1.0, 0.05, 900 + i)))
    h, t = eb.Handle.packing_tuned(descs, 20)
    assert t["block_width"] in (64, 128) and t["candidates"] >= 2
    h.solve(150, -1.0)
    c1 = [h.circles(i, d["n_circles"]) for i, d in enumerate(descs)]
    kw = dict(schedule=t["schedule"], block_width=t["block_width"])
    if t["schedule"] == eb.SCHEDULE_INSTANCE:
        kw.update(cluster_size=t["cluster_size"], coop_min_n=t["coop_min_n"])
    g = eb.Handle.packing(descs, **kw)
    g.solve(150, -1.0)
    for i, d in enumerate(descs):
        assert np.array_equal(c1[i], g.circles(i, d["n_circles"]))
    h.close()
    g.close()
