"""Tail hand-off of the per-instance schedule (paradmm_gpu_set_tail_handoff):
the last few unfinished instances of a solve stop at a sweep boundary and
finish together on the grid-wide schedule.  The sweep arithmetic is the
same on both schedules (only the consensus sums' association differs), so a
handed-over instance follows its per-instance trajectory to rounding, keeps
its own budget of maxiter sweeps and stops on its own residual."""
import numpy as np
import pytest

import engine_b200 as eb

pytestmark = pytest.mark.gpu


def _descs(n, seed, lo=20, hi=220):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        N = int(rng.integers(lo, hi))
        asp = float(rng.uniform(1, 2))
        out.append(dict(n_circles=N, walls=eb.box_walls(asp, 1.0), exponent=2.0, rho=10.0, rho_radius=5.0,
                        alpha=1.0, init=eb.seeded_circles(N, asp, 1.0, 0.05, seed * 1000 + i)))
    return out


def _solve(descs, maxiter, tol, handoff, **kw):
    h = eb.Handle.packing(descs, schedule=eb.SCHEDULE_INSTANCE, **kw)
    if handoff:
        h.set_tail_handoff(handoff)
    s = h.solve(maxiter, tol)
    st = h.instance_stats()
    circ = [h.circles(i, d["n_circles"]) for i, d in enumerate(descs)]
    n = h.tail_handoffs()
    h.close()
    return s, st, circ, n


def test_fixed_sweeps_every_instance_runs_its_budget():
    descs = _descs(48, 1)
    _, st0, c0, n0 = _solve(descs, 400, -1.0, 0)
    _, st1, c1, n1 = _solve(descs, 400, -1.0, 12)
    assert n0 == 0 and 1 <= n1 <= 12
    assert all(s["iterations"] == 400 for s in st1)
    for a, b in zip(c0, c1):
        assert np.abs(a - b).max() <= 1e-6


@pytest.mark.parametrize("cluster,coop", [(1, 0), (2, 100)])
def test_handed_over_instances_stop_on_their_own_residual(cluster, coop):
    descs = _descs(64, 2)
    _, st0, c0, _ = _solve(descs, 20000, 1e-5, 0, cluster_size=cluster, coop_min_n=coop)
    _, st1, c1, n1 = _solve(descs, 20000, 1e-5, 16, cluster_size=cluster, coop_min_n=coop)
    assert n1 >= 1
    for a, b in zip(st0, st1):
        assert a["converged"] == b["converged"]
        if b["converged"]:
            assert b["primal"] + b["dual"] <= 1e-5
        # the grid schedule tests iterate k - 2 at sweep k (the per-instance
        # one k - 1): a handed-over instance may take one sweep more
        assert 0 <= b["iterations"] - a["iterations"] <= 2 or not a["converged"], (a["iterations"], b["iterations"])
    # stopped at r + s <= 1e-5, up to two sweeps apart: the packings agree to
    # the size of a sweep's step there
    for a, b, x, y in zip(st0, st1, c0, c1):
        if a["converged"]:
            assert np.abs(x - y).max() <= 1e-3
    tot0 = sum(c[:, 2].sum() for c in c0)
    tot1 = sum(c[:, 2].sum() for c in c1)
    assert abs(tot1 - tot0) <= 1e-4 * tot0


def test_no_handoff_while_a_fallback_restart_can_happen():
    descs = _descs(24, 3)
    h = eb.Handle.packing(descs, schedule=eb.SCHEDULE_INSTANCE)
    h.set_tail_handoff(8)
    h.set_fallback(5000)  # a budget beyond the call's sweeps: no restart can happen, the hand-off runs
    h.solve(300, -1.0)
    assert h.tail_handoffs() >= 1
    assert all(s["iterations"] == 300 for s in h.instance_stats())
    h.set_fallback(100)  # restarts inside the launch: the per-instance schedule keeps every instance
    h.solve(300, -1.0)
    assert h.tail_handoffs() == 0
    assert all(s["iterations"] == 300 for s in h.instance_stats())
    h.close()
