"""GPU: residual balancing of the penalties (paradmm_gpu_set_rho_balance).

The reference has only an empty hook for it (update_outgoing_rhos,
core/paradmm.c:564-566), so the rule is pinned against its restatement over
the reference's own updateG (oracle harness orc_packing_run_balanced):
  * the FP64 generic engine follows it bit for bit through hundreds of
    sweeps with doublings and halvings of the penalties, across calls;
  * the FP32 packing engine follows it within the per-iterate 1e-4 over the
    free-running horizon, a sweep per call (decisions on every third iterate);
  * on either schedule, an instance of a batch evolves exactly as it does
    alone with balancing on, bit for bit.
"""
import numpy as np
import pytest

import engine_b200 as eb
import oracle_lib

pytestmark = pytest.mark.gpu

TOL_F32 = 1e-4
RHO, RHO_R, ALPHA, EXP = 10.0, 5.0, 1.0, 2.0


def _graphs(N, seed):
    walls = eb.box_walls(1.0, 1.0)
    pg = eb.PackingGraph(N, walls, EXP)
    pg.init_seeded(eb.seeded_circles(N, 1.0, 1.0, 0.05, seed), RHO, RHO_R, ALPHA)
    orc = oracle_lib.OraclePacking(oracle_lib.best(), N, walls, EXP)
    orc.init(seed, 1.0, 1.0, 0.05, RHO, RHO_R, ALPHA)
    return pg, orc


def test_generic_f64_balancing_bit_identical_to_the_rule_over_reference_updateG():
    N, period, mu = 24, 25, 2.0
    pg, orc = _graphs(N, 11)
    n, tr = orc.run_balanced(600, period, mu, -1, 4)
    applied = np.nonzero(tr[:, 3])[0]
    assert len(applied) >= 4 and set(tr[applied, 3]) == {-1.0, 1.0}  # both directions happen
    want = orc.state()
    with eb.Handle.from_graph(pg.G, engine=eb.ENGINE_GENERIC_F64) as h:
        h.set_rho_balance(period, mu, -1, 4)
        done = 0
        for chunk in (37, 1, 1, 161, 400):  # ages continue across calls
            h.iterate(chunk)
            done += chunk
        assert done == 600
        assert h.rho_scale(0) == int(tr[-1, 2])
        h.download(pg.G)
    got = pg.G.state()
    for k in ("X", "M", "N", "U", "Z"):
        assert np.array_equal(got[k], want[k]), f"{k} differs (max {np.max(np.abs(got[k] - want[k]))})"


def test_packing_balancing_follows_the_rule_free_running():
    N, period, mu = 40, 3, 1.0
    pg, orc = _graphs(N, 11)
    with eb.Handle.from_graph(pg.G, engine=eb.ENGINE_PACKING) as h:
        h.set_rho_balance(period, mu, -1, 4)
        for k in range(1, 9):
            h.iterate(1)
            h.download(pg.G)
            ref = oracle_lib.OraclePacking(oracle_lib.best(), N, eb.box_walls(1.0, 1.0), EXP)
            ref.init(11, 1.0, 1.0, 0.05, RHO, RHO_R, ALPHA)
            _, tr = ref.run_balanced(k, period, mu, -1, 4)
            got, want = pg.G.state(), ref.state()
            d = max(float(np.max(np.abs(got[q] - want[q]))) for q in ("X", "M", "N", "U", "Z"))
            assert d <= TOL_F32, f"sweep {k}: max |diff| {d}"
            assert h.rho_scale(0) == int(tr[-1, 2]), k
            ref.close()
    assert int(tr[-1, 2]) == 2  # two doublings applied (after sweeps 5 and 8)


@pytest.mark.parametrize("schedule", [eb.SCHEDULE_GRID, eb.SCHEDULE_INSTANCE])
def test_packing_balancing_batched_equals_single(schedule):
    rng = np.random.default_rng(4)
    descs = []
    for i in range(12):
        N = int(rng.integers(20, 160))
        asp = float(rng.uniform(1, 2))
        descs.append(dict(n_circles=N, walls=eb.box_walls(asp, 1.0), exponent=EXP, rho=RHO, rho_radius=RHO_R,
                          alpha=ALPHA, init=eb.seeded_circles(N, asp, 1.0, 0.05, 700 + i)))
    with eb.Handle.packing(descs, schedule=schedule) as hb:
        hb.set_rho_balance(20, 10.0, -1, 3)
        hb.solve(700, -1.0)
        hb.solve(900, -1.0)  # a second call continues the ages
        batched = [hb.circles(i, d["n_circles"]) for i, d in enumerate(descs)]
        scales = [hb.rho_scale(i) for i in range(len(descs))]
    assert any(s != 0 for s in scales)
    for i in range(0, len(descs), 3):
        with eb.Handle.packing([descs[i]], schedule=schedule) as h1:
            h1.set_rho_balance(20, 10.0, -1, 3)
            h1.solve(1600, -1.0)
            assert h1.rho_scale(0) == scales[i]
            assert np.array_equal(batched[i], h1.circles(0, descs[i]["n_circles"])), i


def test_balancing_arguments_are_checked():
    d = dict(n_circles=10, walls=eb.box_walls(1, 1), exponent=EXP, rho=RHO, rho_radius=RHO_R, alpha=ALPHA,
             init=eb.seeded_circles(10, 1, 1, 0.05, 1))
    with eb.Handle.packing([d]) as h:
        for bad in ((2, 10.0, -1, 4), (10, 0.5, -1, 4), (10, 10.0, 1, 4), (10, 10.0, -1, -1)):
            with pytest.raises(eb.ParadmmError):
                h.set_rho_balance(*bad)
        h.set_rho_balance(0)
        assert h.rho_scale(0) == 0
