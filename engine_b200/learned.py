"""Learned warm start for batched circle packing (driver over the C-ABI).

Instances of the batched workload: N uniform in [nmin, nmax] circles in a
box of aspect uniform in [1, 2] (height 1); every circle carries a Gaussian
code of dimension 16 whose first three coordinates, through the normal CDF,
give its plain start (cx, cy, r) = (W Phi(z0), H Phi(z1), rmax Phi(z2)).
So an instance is its codes, the plain start is a function of them, and the
set MLP (paradmm_learned.h) learns the map from that start to the packing
plain ADMM converges to.

solve_plain / solve_learned time both paths on the same instances:
  plain    create the batch handle (plain start) [untimed], then solve;
  learned  features + network forward + warm start + one solve in which an
           instance not converged within the budget restarts from its plain
           start inside the same launch (fallback); the residual decides.
Times are host wall clock around the calls (device work included).
"""
from __future__ import annotations

import ctypes as C
import math
import os
import time

import numpy as np

from . import PackingDesc, Stats, box_walls, check, load

HERE = os.path.dirname(os.path.abspath(__file__))
WEIGHTS = os.path.join(HERE, "weights", "setmlp_packing.f32")
RMAX = 0.05
CODE_DIM = 16
RHO, RHO_R, ALPHA, EXPONENT = 10.0, 5.0, 1.0, 2.0

_P = C.POINTER(C.c_double)


def _bind():
    lib = load()
    sig = {
        "paradmm_setmlp_num_params": (C.c_int64, []),
        "paradmm_setmlp_create": (C.c_int, [C.c_int, C.c_uint64, C.POINTER(C.c_void_p)]),
        "paradmm_setmlp_destroy": (None, [C.c_void_p]),
        "paradmm_setmlp_get_params": (C.c_int, [C.c_void_p, C.POINTER(C.c_float)]),
        "paradmm_setmlp_set_params": (C.c_int, [C.c_void_p, C.POINTER(C.c_float)]),
        "paradmm_setmlp_set_data": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_int), _P, _P, _P, C.c_double]),
        "paradmm_setmlp_train": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_float, C.c_float, _P]),
        "paradmm_setmlp_eval": (C.c_int, [C.c_void_p, _P]),
        "paradmm_setmlp_gradients": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.POINTER(C.c_float), _P]),
        "paradmm_setmlp_features": (C.c_int, [C.c_void_p, C.POINTER(C.c_float)]),
        "paradmm_setmlp_predict": (C.c_int, [C.c_void_p, _P, _P]),
        "paradmm_gpu_warm_start_all": (C.c_int, [C.c_void_p, _P, C.c_int]),
        "paradmm_gpu_warm_start_all_duals": (C.c_int, [C.c_void_p, _P, C.c_int, C.c_int]),
    }
    for k, (r, a) in sig.items():
        f = getattr(lib, k)
        f.restype = r
        f.argtypes = a
    return lib


def _phi(x: np.ndarray) -> np.ndarray:
    return 0.5 * (1.0 + np.vectorize(math.erf)(x / math.sqrt(2.0)))


def make_instances(n: int, seed: int, nmin: int = 20, nmax: int = 400) -> list[dict]:
    """n instances of the batched workload (seeded)."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        N = int(rng.integers(nmin, nmax + 1))
        asp = float(rng.uniform(1.0, 2.0))
        z = rng.standard_normal((N, CODE_DIM))
        init = _phi(z[:, :3]) * np.array([asp, 1.0, RMAX])
        out.append(dict(n_circles=N, aspect=asp, code=z, init=np.ascontiguousarray(init)))
    return out


def _descs(instances):
    arr = (PackingDesc * len(instances))()
    keep = []
    for i, d in enumerate(instances):
        walls = np.ascontiguousarray(box_walls(d["aspect"], 1.0))
        init = np.ascontiguousarray(d["init"], dtype=np.float64)
        keep += [walls, init]
        arr[i].n_circles = d["n_circles"]
        arr[i].n_walls = 4
        arr[i].walls = walls.ctypes.data_as(_P)
        arr[i].exponent = EXPONENT
        arr[i].rho = RHO
        arr[i].rho_radius = RHO_R
        arr[i].alpha = ALPHA
        arr[i].init = init.ctypes.data_as(_P)
    return arr, keep


class Batch:
    """A packing handle over a list of instances (plain start)."""

    def __init__(self, instances, device=0, schedule=0, cluster=0, coop_min_n=0, no_graphs=False, block_width=0,
                 handoff=0):
        from . import opts
        self.lib = load()
        self.instances = instances
        arr, self._keep = _descs(instances)
        o = opts(device=device, schedule=schedule, cluster_size=cluster, block_width=block_width)
        o.reserved[0] = coop_min_n
        o.reserved[1] = 1 if no_graphs else 0
        o.reserved[2] = int(handoff)  # tail hand-off (paradmm_gpu_set_tail_handoff)
        p = C.c_void_p()
        check(self.lib.paradmm_gpu_create_packing(arr, len(instances), C.byref(o), C.byref(p)))
        self.h = p

    def solve(self, maxiter: int, tol: float) -> dict:
        s = Stats()
        rc = self.lib.paradmm_gpu_solve(self.h, maxiter, tol, C.byref(s))
        if rc not in (0, -6):
            check(rc)
        return s.as_dict()

    def stats(self) -> list[dict]:
        n = len(self.instances)
        arr = (Stats * n)()
        check(self.lib.paradmm_gpu_instance_stats(self.h, arr))
        return [a.as_dict() for a in arr]

    def circles(self) -> list[np.ndarray]:
        out = []
        for i, d in enumerate(self.instances):
            c = np.zeros((d["n_circles"], 3))
            check(self.lib.paradmm_gpu_get_circles(self.h, i, c.ctypes.data_as(_P)))
            out.append(c)
        return out

    def autotune(self, sweeps: int = 100, tol: float = -1.0) -> dict:
        from . import Tuning
        t = Tuning()
        check(self.lib.paradmm_gpu_autotune(self.h, int(sweeps), float(tol), C.byref(t)))
        return {k: getattr(t, k) for k, _ in Tuning._fields_ if k != "reserved"}

    def set_fallback(self, after_sweeps: int) -> None:
        check(self.lib.paradmm_gpu_set_fallback(self.h, int(after_sweeps)))

    def set_rho_balance(self, period: int, mu: float = 10.0, log2_min: int = -1, log2_max: int = 4) -> None:
        check(self.lib.paradmm_gpu_set_rho_balance(self.h, int(period), float(mu), int(log2_min), int(log2_max)))

    def set_tail_handoff(self, instances: int) -> None:
        """The last `instances` unfinished instances of a solve finish together
        on the grid-wide schedule (paradmm_gpu_set_tail_handoff)."""
        check(self.lib.paradmm_gpu_set_tail_handoff(self.h, int(instances)))

    def tail_handoffs(self) -> int:
        return self.lib.paradmm_gpu_tail_handoffs(self.h)

    def fallbacks(self) -> np.ndarray:
        out = np.zeros(len(self.instances), dtype=np.int32)
        check(self.lib.paradmm_gpu_instance_fallbacks(self.h, out.ctypes.data_as(C.POINTER(C.c_int))))
        return out

    def warm_start(self, circles: np.ndarray, radius_duals: int = 1, dual_iters: int = 0) -> None:
        """Every instance from `circles`: X = Z, radius duals at the radius
        prox's fixed point (radius_duals = 1) or 0, pair and wall duals 0,
        then dual_iters rounds of the reference's optimal-initialisation map
        on every factor."""
        lib = _bind()
        c = np.ascontiguousarray(circles, dtype=np.float64)
        check(lib.paradmm_gpu_warm_start_all_duals(self.h, c.ctypes.data_as(_P), radius_duals, int(dual_iters)))

    def close(self):
        if self.h:
            self.lib.paradmm_gpu_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class SetMLP:
    """The set MLP of paradmm_learned.h."""

    def __init__(self, device: int = 0, seed: int = 1):
        self.lib = _bind()
        p = C.c_void_p()
        check(self.lib.paradmm_setmlp_create(device, seed, C.byref(p)))
        self.p = p
        self.n_params = int(self.lib.paradmm_setmlp_num_params())

    def params(self) -> np.ndarray:
        out = np.zeros(self.n_params, dtype=np.float32)
        check(self.lib.paradmm_setmlp_get_params(self.p, out.ctypes.data_as(C.POINTER(C.c_float))))
        return out

    def set_params(self, w: np.ndarray) -> None:
        w = np.ascontiguousarray(w, dtype=np.float32)
        assert w.size == self.n_params
        check(self.lib.paradmm_setmlp_set_params(self.p, w.ctypes.data_as(C.POINTER(C.c_float))))

    def load(self, path: str = WEIGHTS) -> None:
        self.set_params(np.fromfile(path, dtype=np.float32))

    def save(self, path: str = WEIGHTS) -> None:
        os.makedirs(os.path.dirname(path), exist_ok=True)
        self.params().tofile(path)

    def set_data(self, instances, targets=None) -> None:
        n = len(instances)
        nc = np.array([d["n_circles"] for d in instances], dtype=np.int32)
        box = np.array([[d["aspect"], 1.0] for d in instances], dtype=np.float64).ravel()
        init = np.ascontiguousarray(np.concatenate([d["init"] for d in instances]), dtype=np.float64)
        tgt = None if targets is None else np.ascontiguousarray(np.concatenate(targets), dtype=np.float64)
        self._init = init
        check(self.lib.paradmm_setmlp_set_data(self.p, n, nc.ctypes.data_as(C.POINTER(C.c_int)), box.ctypes.data_as(_P),
                                               init.ctypes.data_as(_P), None if tgt is None else tgt.ctypes.data_as(_P),
                                               RMAX))

    def train(self, epochs: int, batch_inst: int, lr: float, lr_end: float) -> np.ndarray:
        losses = np.zeros(epochs)
        check(self.lib.paradmm_setmlp_train(self.p, epochs, batch_inst, lr, lr_end, losses.ctypes.data_as(_P)))
        return losses

    def eval(self) -> float:
        l = C.c_double()
        check(self.lib.paradmm_setmlp_eval(self.p, C.byref(l)))
        return l.value

    def gradients(self, b0: int, nb: int) -> tuple[np.ndarray, float]:
        g = np.zeros(self.n_params, dtype=np.float32)
        l = C.c_double()
        check(self.lib.paradmm_setmlp_gradients(self.p, b0, nb, g.ctypes.data_as(C.POINTER(C.c_float)), C.byref(l)))
        return g, l.value

    def features(self, rows: int) -> np.ndarray:
        f = np.zeros((rows, 32), dtype=np.float32)
        check(self.lib.paradmm_setmlp_features(self.p, f.ctypes.data_as(C.POINTER(C.c_float))))
        return f

    def predict(self) -> np.ndarray:
        out = np.zeros_like(self._init)
        check(self.lib.paradmm_setmlp_predict(self.p, self._init.ctypes.data_as(_P), out.ctypes.data_as(_P)))
        return out

    def close(self):
        if self.p:
            self.lib.paradmm_setmlp_destroy(self.p)
            self.p = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ------------------------------------------------------------------ pipelines
def generate(n: int, seed: int, batch: int = 512, maxiter: int = 20000, tol: float = 1e-5, device: int = 0):
    """Converged packings of n instances (only the converged ones are kept)."""
    inst_all, tgt_all = [], []
    done = 0
    while done < n:
        k = min(batch, n - done)
        inst = make_instances(k, seed + done)
        b = Batch(inst, device=device)
        b.solve(maxiter, tol)
        st = b.stats()
        circ = b.circles()
        for d, s, c in zip(inst, st, circ):
            if s["converged"]:
                inst_all.append(d)
                tgt_all.append(c)
        b.close()
        done += k
    return inst_all, tgt_all


def solve_plain(instances, maxiter=20000, tol=1e-5, device=0, **batch_kw):
    b = Batch(instances, device=device, **batch_kw)
    t = time.perf_counter()
    s = b.solve(maxiter, tol)
    wall = time.perf_counter() - t
    st = b.stats()
    circ = b.circles()
    b.close()
    return dict(wall_s=wall, device_ms=s["device_ms"], stats=st, circles=circ)


def solve_learned(instances, net: SetMLP, budget=6000, maxiter=20000, tol=1e-5, radius_duals=1, dual_iters=0, device=0,
                  **batch_kw):
    """Learned path: network proposal -> warm start -> one solve.  With
    budget > 0, every instance still unconverged after `budget` sweeps
    restarts from its plain start (in the same launch) and gets the plain
    path's full maxiter; with budget <= 0 there is no fallback and every
    instance gets maxiter sweeps from the warm start."""
    b = Batch(instances, device=device, **batch_kw)
    t = time.perf_counter()
    net.set_data(instances)
    prop = net.predict()
    b.warm_start(prop, radius_duals, dual_iters)
    b.set_fallback(max(budget, 0))
    s = b.solve((budget if budget > 0 else 0) + maxiter, tol)
    wall = time.perf_counter() - t
    st = b.stats()
    fb = b.fallbacks()
    for i, x in enumerate(st):
        x["fallback"] = int(fb[i])
    circ = b.circles()
    b.close()
    return dict(wall_s=wall, device_ms=s["device_ms"], stats=st, circles=circ, fallbacks=int(fb.sum()), proposal=prop)


def train_weights(n_instances: int = 20000, epochs: int = 40, seed: int = 100000, out: str = WEIGHTS,
                  device: int = 0, net_seeds=(7, 8, 9), val_seed: int = 900001) -> dict:
    """Reproduces the committed weights: converged packings of n_instances
    seeded instances of the batched workload (plain solver, tol 1e-5), 90 %
    for training and 10 % for the validation loss; one network per seed in
    net_seeds, `epochs` Adam passes in batches of 32 instances, learning rate
    1e-3 decaying to 5e-5.  The kept network is the one whose warm start
    solves a separate validation batch (512 instances, seed val_seed, never
    the evaluation batch) fastest, host wall clock, no fallback."""
    t = time.perf_counter()
    inst, tgt = generate(n_instances, seed=seed, device=device)
    t_gen = time.perf_counter() - t
    ntr = int(0.9 * len(inst))
    val = make_instances(512, val_seed)
    kw = dict(cluster=2, coop_min_n=200)
    for _ in range(2):
        plain = solve_plain(val, device=device, **kw)
    best = None
    report = []
    for ns in net_seeds:
        net = SetMLP(device=device, seed=ns)
        net.set_data(inst[:ntr], tgt[:ntr])
        t = time.perf_counter()
        net.train(epochs=epochs, batch_inst=32, lr=1e-3, lr_end=5e-5)
        t_train = time.perf_counter() - t
        train_loss = net.eval()
        net.set_data(inst[ntr:], tgt[ntr:])
        val_loss = net.eval()
        wall = min(solve_learned(val, net, budget=0, device=device, **kw)["wall_s"] for _ in range(2))
        report.append(dict(net_seed=ns, train_loss=train_loss, val_loss=val_loss, train_s=t_train,
                           val_batch_s=wall, val_batch_plain_s=plain["wall_s"]))
        if best is None or wall < best[0]:
            best = (wall, ns, net.params())
        net.close()
    net = SetMLP(device=device, seed=best[1])
    net.set_params(best[2])
    net.save(out)
    net.close()
    return dict(converged=len(inst), requested=n_instances, generate_s=t_gen, kept_net_seed=best[1],
                candidates=report, out=out)


def tune(instances, sweeps: int, tol: float, device: int = 0, handoff: int = 0) -> dict:
    """Tile side and schedule for batches like `instances`
    (paradmm_gpu_create_packing_tuned with probe solve(sweeps, tol)); the
    probes of the per-instance schedule run with the tail hand-off `handoff`."""
    from . import Tuning, opts
    lib = load()
    arr, keep = _descs(instances)
    o = opts(device=device)
    o.reserved[2] = int(handoff)
    p = C.c_void_p()
    t = Tuning()
    check(lib.paradmm_gpu_create_packing_tuned(arr, len(instances), C.byref(o), int(sweeps), float(tol), C.byref(p),
                                               C.byref(t)))
    lib.paradmm_gpu_destroy(p)
    return {k: getattr(t, k) for k, _ in Tuning._fields_ if k != "reserved"}


if __name__ == "__main__":
    import argparse
    import json
    ap = argparse.ArgumentParser(description="train the set-MLP warm start on packings the plain solver produces")
    ap.add_argument("--instances", type=int, default=20000)
    ap.add_argument("--epochs", type=int, default=40)
    ap.add_argument("--out", default=WEIGHTS)
    a = ap.parse_args()
    print(json.dumps(train_weights(a.instances, a.epochs, out=a.out)))
