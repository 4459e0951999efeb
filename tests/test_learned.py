"""The learned warm start: feature kernel, set-MLP gradients against the CPU
FP64 reference, training, and the warm-start path into the packing engine."""
import numpy as np
import pytest

import setmlp_ref

pytestmark = pytest.mark.gpu


def _small_set(seed=0, n=8):
    from engine_b200 import learned
    inst = learned.make_instances(n, seed, nmin=4, nmax=40)
    return inst


def test_features_match_reference():
    from engine_b200 import learned
    inst = _small_set(1)
    net = learned.SetMLP(seed=3)
    net.set_data(inst)
    rows = sum(d["n_circles"] for d in inst)
    f_dev = net.features(rows)
    f_ref = setmlp_ref.features([(d["n_circles"], d["aspect"], 1.0, d["init"]) for d in inst])
    assert np.max(np.abs(f_dev - f_ref)) < 2e-4
    net.close()


@pytest.mark.parametrize("seed", [2, 5])
def test_gradients_match_fp64_reference(seed):
    from engine_b200 import learned
    inst = _small_set(seed)
    rng = np.random.default_rng(seed)
    targets = [np.stack([d["init"][:, 0] + rng.normal(0, 0.02, d["n_circles"]),
                         d["init"][:, 1] + rng.normal(0, 0.02, d["n_circles"]),
                         rng.uniform(0.01, 0.08, d["n_circles"])], 1) for d in inst]
    net = learned.SetMLP(seed=seed)
    net.set_data(inst, targets)
    g_dev, l_dev = net.gradients(0, len(inst))
    rows = sum(d["n_circles"] for d in inst)
    F = net.features(rows)
    sizes = [d["n_circles"] for d in inst]
    T = np.zeros((rows, 4))
    r0 = 0
    for d, t in zip(inst, targets):
        s = np.sqrt(d["aspect"] / d["n_circles"])
        n = d["n_circles"]
        T[r0:r0 + n, 0] = (t[:, 0] - d["init"][:, 0]) / s
        T[r0:r0 + n, 1] = (t[:, 1] - d["init"][:, 1]) / s
        T[r0:r0 + n, 2] = t[:, 2] / s
        r0 += n
    l_ref, g_ref = setmlp_ref.loss_and_grads(net.params(), F, T, sizes)
    assert abs(l_dev - l_ref) <= 1e-4 * abs(l_ref)
    off = 0
    for name, cnt in (("W1", 128 * 32), ("b1", 128), ("W2", 128 * 256), ("b2", 128), ("W3", 4 * 128), ("b3", 4)):
        a, b = g_dev[off:off + cnt], g_ref[off:off + cnt]
        rel = np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30)
        assert rel < 2e-3, f"{name}: relative error {rel:.2e}"
        off += cnt
    net.close()


def test_training_reduces_loss():
    from engine_b200 import learned
    inst = learned.make_instances(64, 11, nmin=10, nmax=60)
    # a smooth synthetic target: each circle moves toward the box centre and
    # takes a radius set by its nearest-neighbour distance
    targets = []
    for d in inst:
        c = d["init"]
        dd = np.sqrt(((c[:, None, :2] - c[None, :, :2]) ** 2).sum(-1)) + np.eye(len(c)) * 9
        tgt = np.stack([c[:, 0] + 0.1 * (d["aspect"] / 2 - c[:, 0]), c[:, 1] + 0.1 * (0.5 - c[:, 1]),
                        0.45 * dd.min(1)], 1)
        targets.append(tgt)
    net = learned.SetMLP(seed=1)
    net.set_data(inst, targets)
    l0 = net.eval()
    losses = net.train(epochs=60, batch_inst=16, lr=2e-3, lr_end=2e-4)
    l1 = net.eval()
    assert l1 < 0.2 * l0, (l0, l1, losses[-5:])
    net.close()


def test_warm_start_from_converged_packing_converges_fast():
    """The warm-start path itself: starting from a converged packing (the
    best possible proposal) converges in far fewer sweeps than the plain
    start, and from a noisy copy of it the residual still decides."""
    from engine_b200 import learned
    inst = learned.make_instances(6, 21, nmin=30, nmax=80)
    plain = learned.solve_plain(inst)
    its_plain = [s["iterations"] for s in plain["stats"]]
    b = learned.Batch(inst)
    b.warm_start(np.concatenate(plain["circles"]), radius_duals=1)
    b.solve(20000, 1e-5)
    st = b.stats()
    assert all(s["converged"] for s in st)
    its_warm = [s["iterations"] for s in st]
    assert sum(its_warm) < 0.5 * sum(its_plain), (its_warm, its_plain)
    b.close()


@pytest.mark.parametrize("cluster", [1, 2])
def test_in_call_fallback_equals_plain_solve(cluster):
    """An instance whose warm start does not converge within the budget
    restarts from its plain start inside the same launch: from there on its
    trajectory is the plain solve's, so it ends on the plain solve's circles
    bit for bit after budget + (plain sweeps) sweeps.  Sizes cover the
    on-chip small-instance path (N <= 40), the tiled one-CTA path and the
    cluster path (N >= 60 here)."""
    from engine_b200 import SCHEDULE_INSTANCE, learned
    inst = learned.make_instances(12, 31, nmin=12, nmax=110)
    budget = 25
    kw = dict(schedule=SCHEDULE_INSTANCE, cluster=cluster, coop_min_n=60)
    bp = learned.Batch(inst, **kw)
    bp.solve(20000, 1e-5)
    st_p, circ_p = bp.stats(), bp.circles()
    bp.close()
    rng = np.random.default_rng(5)
    prop = np.concatenate([d["init"] + rng.normal(0, 0.05, d["init"].shape) * [1, 1, 0.1] for d in inst])
    prop[:, 2] = np.abs(prop[:, 2])
    b = learned.Batch(inst, **kw)
    b.warm_start(prop, radius_duals=1)
    b.set_fallback(budget)
    b.solve(budget + 20000, 1e-5)
    st, circ, fb = b.stats(), b.circles(), b.fallbacks()
    b.close()
    assert fb.sum() > 0
    for i in range(len(inst)):
        if not fb[i]:
            assert st[i]["converged"] and st[i]["iterations"] <= budget
            continue
        assert st[i]["iterations"] == budget + st_p[i]["iterations"], (i, st[i]["iterations"], st_p[i]["iterations"])
        assert st[i]["converged"] == st_p[i]["converged"]
        assert np.array_equal(circ[i], circ_p[i]), i


def test_fallback_needs_instance_schedule():
    from engine_b200 import SCHEDULE_GRID, learned
    from engine_b200 import ParadmmError
    inst = learned.make_instances(2, 3, nmin=10, nmax=20)
    b = learned.Batch(inst, schedule=SCHEDULE_GRID)
    with pytest.raises(ParadmmError):
        b.set_fallback(10)
    b.set_fallback(0)
    b.close()


def test_trained_network_reduces_sweeps():
    """The committed weights on fresh instances of the batched workload
    (N uniform in [20, 400]): the learned warm start (with the in-launch
    fallback) needs fewer sweeps than the plain start, and the packings it
    converges to are no smaller (total radius) and as feasible (the per-instance
    violations at the stopping rule, by quantile)."""
    from engine_b200 import learned
    inst = learned.make_instances(48, 4242)
    net = learned.SetMLP()
    net.load()
    pl = learned.solve_plain(inst)
    le = learned.solve_learned(inst, net, budget=3000)
    net.close()
    its_p = np.array([x["iterations"] for x in pl["stats"]])
    its_l = np.array([x["iterations"] for x in le["stats"]])
    conv_p = np.array([x["converged"] for x in pl["stats"]], bool)
    conv_l = np.array([x["converged"] for x in le["stats"]], bool)
    assert conv_l.sum() >= conv_p.sum() - 1
    assert np.median(its_l) < 0.8 * np.median(its_p), (np.median(its_l), np.median(its_p))
    tot_p = sum(c[:, 2].sum() for c in pl["circles"])
    tot_l = sum(c[:, 2].sum() for c in le["circles"])
    assert (tot_l - tot_p) / tot_p > -1e-3, (tot_l, tot_p)
    # feasibility at the same stopping rule (r + s <= 1e-5): the learned
    # start's violations are distributed like the plain start's -- median and
    # 90th percentile no worse than plain's (10 % slack for 48 instances), the
    # worst instance within 1.5x of plain's worst
    vp = np.array([x["max_violation"] for x, c in zip(pl["stats"], conv_p) if c])
    vl = np.array([x["max_violation"] for x, c in zip(le["stats"], conv_l) if c])
    qp, ql = np.quantile(vp, [0.5, 0.9]), np.quantile(vl, [0.5, 0.9])
    print(f"violation median/p90/max: plain {qp[0]:.2e}/{qp[1]:.2e}/{vp.max():.2e}, "
          f"learned {ql[0]:.2e}/{ql[1]:.2e}/{vl.max():.2e}")
    assert np.all(ql <= 1.1 * qp + 1e-7), (ql, qp)
    assert vl.max() <= 1.5 * vp.max() + 1e-7, (vl.max(), vp.max())
