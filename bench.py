#!/usr/bin/env python
"""Benchmark of the fused circle-packing ADMM sweep (edge-updates/s).

Workload (one "step" = one full sweep X/M/Z/U/N of the factor graph):
  plain circle packing, N = 8000 circles in a 2 x 1 box: 31,996,000 pair
  factors, 32,000 wall factors, 8,000 radius factors, 128,056,000 edges;
  seeded uniform init (centres in the box, radii in [0, 0.01]), rho = 10,
  rho on radius-factor edges = 5, alpha = 1, radius exponent 2.  The FP32
  edge state (U of the pair edges; X and U of wall and radius edges) is
  0.77 GB, larger than the 126 MB L2, so no L2 flush is needed between
  steps.

Arms:
  default           the engine (libparadmm_b200.so).  `value` is device-timed
                    (CUDA events around the persistent launches, inputs
                    resident); `e2e` is the same metric through the drop-in
                    paradmm.h call updateGOpenMP(G, sweeps, threads) on a host
                    graph, with its uploads and downloads in the timed region.
  --impl reference  the reference's own CPU path (updateGOpenMP of
                    core/paradmm.c, compiled from its sources into oracle/_ref
                    with its -Ofast flags) on all host cores, on a bounded
                    sample of the workload.

Also reported (single GPU): time_to_residual, the batched workload (512
instances, N in [20, 400]) solved to r + s <= 1e-5 from the plain start and
from the set-MLP warm start (inference included), host wall clock.

Multi-GPU (torchrun, one process per GPU): every rank solves its own
instance (replicas, weak scaling; the path has no cross-instance exchange);
value = all ranks' edge-updates / max-over-ranks device time.  With
--mode shard the ranks split ONE instance by circle-block rows and sum a
32 B/circle buffer per sweep with an NCCL all-reduce (strong scaling).
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "edge-updates/s"
N_CIRCLES, BOX_W, BOX_H, RMAX, SEED = 8000, 2.0, 1.0, 0.01, 20261203
RHO, RHO_R, ALPHA, EXPONENT = 10.0, 5.0, 1.0, 2.0
N_WALLS = 4


def edges_of(n: int) -> int:
    return n + 2 * N_WALLS * n + 4 * (n * (n - 1) // 2)


def algo_bytes_per_sweep(n: int) -> int:
    """Bytes one sweep must move: pair edges keep only U (X is recomputed
    from the previous consensus and U), so 8 B per live component (U read and
    written), 6 components; wall and radius edges keep X and U, 16 B per
    component (3 and 1 components)."""
    return (n * (n - 1) // 2) * 48 + N_WALLS * n * 48 + n * 16


def measured_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def profiled_traffic():
    """DRAM bytes per sweep from the committed ncu summary, if present."""
    p = os.path.join(ROOT, "profiles", "pk_persistent_n4000_full.md")
    if not os.path.exists(p):
        return None
    for line in open(p):
        if line.startswith("dram_bytes_per_sweep:"):
            return float(line.split(":", 1)[1].split()[0])
    return None


class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpus: str):
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", gpus, f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                       "-lms", "200"], stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None

    def stop(self) -> dict:
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except Exception:
            self.p.kill()
        self.f.flush()
        rows = [r.split(",") for r in open(self.f.name).read().strip().splitlines() if r.count(",") >= 8]
        os.unlink(self.f.name)
        sm = [float(r[1]) for r in rows if r[1].strip().replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].strip().replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if "Active" in r[5 + i] and "Not" not in r[5 + i]})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def dist_init():
    """One process per GPU over NCCL; gloo on a host without CUDA (tests)."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        if torch.cuda.is_available():
            torch.cuda.set_device(local)
            dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                    device_id=torch.device("cuda", local))
        else:
            dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    return world, rank, local


def _on_gpu() -> bool:
    import torch.distributed as dist
    return dist.get_backend() == "nccl"


def barrier(world):
    if world > 1:
        import torch
        import torch.distributed as dist
        dist.barrier()
        if _on_gpu():
            torch.cuda.synchronize()


def allreduce_max(world, x: float) -> float:
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda" if _on_gpu() else "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def seeded_init(n: int, seed: int):
    import numpy as np

    import engine_b200 as eb
    if n <= 20000:
        return eb.seeded_circles(n, BOX_W, BOX_H, RMAX, seed)
    return np.random.default_rng(seed).uniform(size=(n, 3)) * np.array([BOX_W, BOX_H, RMAX])


# ------------------------------------------------------------------ CPU leg
def reference_lib():
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_lib
    for path in (oracle_lib.REF_OFAST, oracle_lib.REF):
        if os.path.exists(path):
            return oracle_lib._load(path), "reference"
    oracle_lib.ensure_built()
    return oracle_lib._load(oracle_lib.PORT), "port"


def reference_rate(n: int, sweeps: int, threads: int):
    """Edge-updates/s of the reference's updateGOpenMP on an n-circle sample of
    the workload (same box, radii and penalties)."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_lib

    import engine_b200 as eb
    lib, kind = reference_lib()
    P = oracle_lib.OraclePacking(lib, n, eb.box_walls(BOX_W, BOX_H), EXPONENT)
    P.init(SEED, BOX_W, BOX_H, RMAX, RHO, RHO_R, ALPHA)
    dt = lib.orc_time_sweeps(P.graph_ptr(), sweeps, threads)
    E = P.G.num_edges
    P.close()
    return E * sweeps / dt, dt, E, kind


def cpu_sample_size(threads: int, budget_s: float, sweeps: int) -> int:
    rate, _, _, _ = reference_rate(400, 2, threads)
    n = int((rate * budget_s / sweeps / 2.0) ** 0.5)
    return max(200, min(n, 4000))


def run_reference_arm(args):
    world, rank, _ = int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")), 0
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    per_step = min(1.0, 150.0 / max(1, args.steps + args.warmup))
    n = cpu_sample_size(threads, per_step, 1)
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_lib

    import engine_b200 as eb
    lib, kind = reference_lib()
    P = oracle_lib.OraclePacking(lib, n, eb.box_walls(BOX_W, BOX_H), EXPONENT)
    P.init(SEED, BOX_W, BOX_H, RMAX, RHO, RHO_R, ALPHA)
    if args.warmup:
        lib.orc_time_sweeps(P.graph_ptr(), args.warmup, threads)
    dt = lib.orc_time_sweeps(P.graph_ptr(), args.steps, threads)
    E = P.G.num_edges
    rate = E * args.steps / dt
    sample = (f"N={n} circles of the workload's distribution ({E} edges), {args.steps} sweeps of "
              f"updateGOpenMP, {threads} threads")
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": rate, "unit": METRIC, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": dt / args.steps * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"plain circle packing N={N_CIRCLES}, {BOX_W:g}x{BOX_H:g} box (CPU leg: bounded sample)",
                   "sample_circles": n, "sample_edges": E},
        "cpu_baseline": {"value": rate, "unit": METRIC, "cores": threads, "kind": kind, "sample": sample},
        "e2e": {"value": rate, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }), flush=True)


# ------------------------------------------------------------------ GPU arm
# learned arm: no fallback budget -- on this workload the warm start converges
# on more instances than the plain start, and restarting slow ones from the
# plain start only lengthened the batch (0.43 s with a 3000-sweep budget, 0.36 s
# without, device time)
TTR_INSTANCES, TTR_SEED, TTR_MAXITER, TTR_TOL, TTR_BUDGET = 512, 900000, 20000, 1e-5, 0


def run_ttr(local: int):
    """Time to residual on the batched workload: 512 instances (N uniform in
    [20, 400], box aspect uniform in [1, 2]), host wall clock from the solve
    call until every instance has r + s <= 1e-5 or used its iteration cap.
    plain: the batch handle's plain start.  learned: set-MLP features and
    forward, warm start, then one solve (TTR_BUDGET > 0 would restart
    instances not converged after that many sweeps from their plain start in
    the same launch).  Both run once untimed first, on
    the schedule the autotuner picked for batches of this distribution."""
    import numpy as np

    from engine_b200 import learned
    inst = learned.make_instances(TTR_INSTANCES, TTR_SEED)
    # schedule from the autotuner, tuned on another seeded batch of the same
    # distribution (probe = full solves to the tolerance; untimed, like
    # creating the handle), used by both arms
    tune = learned.tune(learned.make_instances(TTR_INSTANCES, TTR_SEED + 1), TTR_MAXITER, TTR_TOL, device=local)
    kw = dict(schedule=tune["schedule"], cluster=tune["cluster_size"], coop_min_n=tune["coop_min_n"],
              block_width=tune["block_width"])
    net = learned.SetMLP(device=local)
    net.load()
    for _ in range(2):
        pl = learned.solve_plain(inst, maxiter=TTR_MAXITER, tol=TTR_TOL, device=local, **kw)
        le = learned.solve_learned(inst, net, budget=TTR_BUDGET, maxiter=TTR_MAXITER, tol=TTR_TOL, device=local, **kw)
    net.close()
    tot_p = sum(float(c[:, 2].sum()) for c in pl["circles"])
    tot_l = sum(float(c[:, 2].sum()) for c in le["circles"])
    its_p = np.array([x["iterations"] for x in pl["stats"]])
    its_l = np.array([x["iterations"] for x in le["stats"]])
    return {"workload": f"{TTR_INSTANCES} packing instances, N uniform in [20,400], aspect uniform in [1,2], "
                        f"seeded Gaussian-code plain starts (seed {TTR_SEED})",
            "tol": TTR_TOL, "maxiter": TTR_MAXITER, "learned_budget": TTR_BUDGET,
            "schedule": {"schedule": "instance" if tune["schedule"] == 2 else "grid", "block_width": tune["block_width"],
                         "cluster": tune["cluster_size"],
                         "coop_min_n": tune["coop_min_n"], "autotune_candidates": tune["candidates"],
                         "probe_ms_best": tune["ms"], "probe_ms_worst": tune["worst_ms"]},
            "plain_s": pl["wall_s"], "learned_s": le["wall_s"], "speedup": pl["wall_s"] / le["wall_s"],
            "converged_plain": int(sum(x["converged"] for x in pl["stats"])),
            "converged_learned": int(sum(x["converged"] for x in le["stats"])),
            "fallbacks": le["fallbacks"],
            "median_sweeps_plain": int(np.median(its_p)), "median_sweeps_learned": int(np.median(its_l)),
            "total_radius_rel_diff": (tot_l - tot_p) / tot_p,
            "max_violation_learned": max(float(x["max_violation"]) for x in le["stats"])}


E2E_HOST_BYTES = 15e9  # one rank's host graph of the workload (X, M, N, U, RHOS, ALPHAS, edge lists)


def host_mem_available():
    """Bytes this process may still allocate: MemAvailable, capped by a
    cgroup memory limit when one is set (None if neither can be read)."""
    vals = []
    try:
        with open("/proc/meminfo") as f:
            for line in f:
                if line.startswith("MemAvailable:"):
                    vals.append(int(line.split()[1]) * 1024)
    except OSError:
        pass
    for lim, cur in (("/sys/fs/cgroup/memory.max", "/sys/fs/cgroup/memory.current"),
                     ("/sys/fs/cgroup/memory/memory.limit_in_bytes", "/sys/fs/cgroup/memory/memory.usage_in_bytes")):
        try:
            with open(lim) as f:
                l = f.read().strip()
            with open(cur) as f:
                c = int(f.read().strip())
            if l != "max" and int(l) < (1 << 60):
                vals.append(int(l) - c)
            break
        except (OSError, ValueError):
            continue
    return min(vals) if vals else None


def run_e2e(args, local: int):
    """updateGOpenMP(G, sweeps, threads) on a host graph of the workload."""
    import engine_b200 as eb
    lib = eb.load()
    o = eb.opts(device=local)
    lib.paradmm_set_sweep_options(C.byref(o))
    t0 = time.time()
    pg = eb.PackingGraph(N_CIRCLES, eb.box_walls(BOX_W, BOX_H), EXPONENT)
    pg.init_seeded(seeded_init(N_CIRCLES, SEED + 1000 * local), RHO, RHO_R, ALPHA)
    build_s = time.time() - t0
    G = pg.G
    threads = os.cpu_count() or 1
    S = args.e2e_sweeps
    lib.updateGOpenMP(C.byref(G), S, threads)  # warm-up: analysis, handle, pinning
    eb.check(lib.paradmm_last_status())
    times = []
    for _ in range(args.e2e_steps):
        t = time.perf_counter()
        lib.updateGOpenMP(C.byref(G), S, threads)
        times.append(time.perf_counter() - t)
        eb.check(lib.paradmm_last_status())
    E, V = G.num_edges, G.num_vars
    h2d = 2 * E * 2 * 8 + V * 2 * 8  # N and U (edge state) + Z
    d2h = 4 * E * 2 * 8 + V * 2 * 8  # X, M, N, U + Z
    total = sum(times)
    lib.closeG(C.byref(G))
    return {"value": E * S * len(times) / total, "unit": METRIC, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
            "sweeps_per_step": S, "steps": len(times), "s_per_step": total / len(times), "call": "updateGOpenMP",
            "graph_build_s": round(build_s, 2)}


def run_engine_arm(args):
    import numpy as np

    import engine_b200 as eb
    world, rank, local = dist_init()
    n = args.circles
    desc = dict(n_circles=n, walls=eb.box_walls(BOX_W, BOX_H), exponent=EXPONENT, rho=RHO, rho_radius=RHO_R,
                alpha=ALPHA, init=seeded_init(n, SEED + 1000 * rank))
    h = eb.Handle.packing([desc], device=local, block_width=args.block_width)
    h.iterate(max(3, args.warmup))
    E = edges_of(n)
    barrier(world)
    clocks = Clocks(str(local) if world == 1 else ",".join(str(i) for i in range(world))) if rank == 0 else None
    l0 = h.launches()
    t = time.perf_counter()
    s = h.solve(args.steps, -1.0)
    wall = time.perf_counter() - t
    launches = h.launches() - l0
    barrier(world)
    ck = clocks.stop() if clocks else None
    dev_ms = allreduce_max(world, float(s["device_ms"]))
    st = h.instance_stats()[0]
    value = world * E * args.steps / (dev_ms * 1e-3)
    algo = algo_bytes_per_sweep(n)
    launch_ms = dev_ms / max(1, launches)
    sweeps_per_launch = args.steps / max(1, launches)
    achieved = algo * sweeps_per_launch / (launch_ms * 1e-3) / 1e9
    peak, peak_kind = measured_peak()
    traffic_sweep = profiled_traffic()
    e2e = None
    if not args.no_e2e and n == N_CIRCLES:
        # every rank builds its own FP64 host graph (about 15 GB at N = 8000,
        # page-locked for the copies): skip the leg on all ranks alike rather
        # than drive the host out of memory
        ranks_here = int(os.environ.get("LOCAL_WORLD_SIZE", str(world)))
        need = E2E_HOST_BYTES * ranks_here
        avail = host_mem_available()
        short = avail is not None and avail < 1.25 * need
        if allreduce_max(world, 1.0 if short else 0.0) > 0:
            e2e = {"value": None, "unit": METRIC,
                   "skipped": f"host memory: {ranks_here} host graphs need about {need / 1e9:.0f} GB, "
                              f"{(avail or 0) / 1e9:.0f} GB available"}
        else:
            rate, err = None, None
            try:
                e2e = run_e2e(args, local)
                rate = e2e["value"]
            except Exception as ex:  # report, never fake
                err = str(ex)[:200]
            # the slowest rank sets the aggregate; every rank takes part, a failed one as +inf
            worst = allreduce_max(world, -rate if rate is not None else float("inf"))
            if err is not None or worst == float("inf"):
                e2e = {"value": None, "unit": METRIC, "error": err or "the end-to-end leg failed on another rank"}
            else:
                e2e["value"] = world * (-worst)
    ttr = None
    if world == 1 and not args.no_ttr and n == N_CIRCLES:
        try:
            ttr = run_ttr(local)
        except Exception as ex:  # report, never fake
            ttr = {"error": str(ex)[:200]}
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu and n == N_CIRCLES:
        threads = os.cpu_count() or 1
        nsamp = cpu_sample_size(threads, 12.0, 10)
        rate, dt, Es, kind = reference_rate(nsamp, 10, threads)
        cpu = {"value": rate, "unit": METRIC, "cores": threads, "kind": kind,
               "sample": f"N={nsamp} circles of the workload's distribution ({Es} edges), 10 sweeps of the "
                         f"reference updateGOpenMP ({dt:.1f} s)"}
    if rank == 0:
        out = {
            "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": dev_ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32/f64", "data": "synthetic",
            "config": {"workload": f"plain circle packing N={n}, {BOX_W:g}x{BOX_H:g} box, radii in [0,{RMAX}], "
                                   f"seeded uniform init (per-rank seeds)"
                                   + ("" if n == N_CIRCLES else " [reduced case for profiling]"),
                       "circles": n, "edges": E, "pair_factors": n * (n - 1) // 2, "rho": RHO, "rho_radius": RHO_R,
                       "alpha": ALPHA, "exponent": EXPONENT, "block_width": args.block_width or "tuned",
                       "l2": f"FP32 edge state {algo_bytes_per_sweep(n) / 2e9:.2f} GB vs 126 MB L2; no flush between steps",
                       "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
                       "timing": "CUDA events on the engine stream around the persistent launches"},
            "iterations_per_s": world * args.steps / (dev_ms * 1e-3),
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_kind": peak_kind,
                         "traffic": None if traffic_sweep is None else traffic_sweep * sweeps_per_launch,
                         "algorithmic_bytes_per_sweep": algo, "sweeps_per_launch": sweeps_per_launch,
                         "algorithmic_bytes": "48 B per pair factor (U of 6 live components, read + written; "
                                              "X recomputed), 48 B per wall factor, 16 B per radius factor",
                         "kernel": "pk_persistent"},
            "cpu_baseline": cpu,
            "e2e": e2e,
            "time_to_residual": ttr,
            "gpu_launches": launches,
            "clocks": ck,
            "wall_s": wall,
            "residuals_after": {"primal": st["primal"], "dual": st["dual"]},
        }
        print(json.dumps(out), flush=True)
    h.close()
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def run_shard_arm(args):
    """--mode shard: ONE instance split over the ranks by circle-block rows
    (engine_b200.shard), one all-reduce of 32 B per circle per sweep (NCCL);
    strong scaling.  Device time: CUDA events on the stream that carries the
    kernels and the all-reduce, max over ranks."""
    import torch
    import torch.distributed as dist

    import engine_b200 as eb
    from engine_b200.shard import Shard, run_sharded
    world, rank, local = dist_init()
    torch.cuda.set_device(local)
    n = args.circles
    desc = dict(n_circles=n, walls=eb.box_walls(BOX_W, BOX_H), exponent=EXPONENT, rho=RHO, rho_radius=RHO_R,
                alpha=ALPHA, init=seeded_init(n, SEED))
    sh = Shard(desc, rank, world, device=local, block_width=args.block_width)
    ex = torch.zeros(sh.exchange_bytes // 8, dtype=torch.float64, device=f"cuda:{local}")

    def allreduce(t):
        if world > 1:
            dist.all_reduce(t)

    run_sharded(sh, ex, allreduce, max(3, args.warmup), -1.0, poll_every=64)
    barrier(world)
    clocks = Clocks(str(local) if world == 1 else ",".join(str(i) for i in range(world))) if rank == 0 else None
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    l0 = sh.launches()
    e0.record()
    st = run_sharded(sh, ex, allreduce, args.steps, -1.0, poll_every=max(64, args.steps))
    e1.record()
    torch.cuda.synchronize()
    launches = sh.launches() - l0
    barrier(world)
    ck = clocks.stop() if clocks else None
    dev_ms = allreduce_max(world, e0.elapsed_time(e1))
    E = edges_of(n)
    algo = algo_bytes_per_sweep(n)
    peak, peak_kind = measured_peak()
    achieved = algo * args.steps / (dev_ms * 1e-3) / 1e9 / world  # per GPU
    if rank == 0:
        out = {
            "metric": METRIC, "value": E * args.steps / (dev_ms * 1e-3), "unit": METRIC, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": dev_ms / args.steps, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": "f32/f64", "data": "synthetic",
            "config": {"workload": f"ONE plain circle packing N={n}, {BOX_W:g}x{BOX_H:g} box, radii in [0,{RMAX}], "
                                   f"seeded uniform init, split over the ranks by circle-block rows",
                       "circles": n, "edges": E, "parallelism": f"shard x{world} (all-reduce of {32 * n} B/sweep)",
                       "rows": list(sh.rows), "timing": "CUDA events on torch's stream (kernels + all-reduce)"},
            "iterations_per_s": args.steps / (dev_ms * 1e-3),
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "peak_kind": peak_kind, "traffic": None, "per": "GPU (algorithmic bytes / world)",
                         "kernel": "pk_shard_pass + pk_shard_partial + pk_shard_consensus"},
            "cpu_baseline": None, "e2e": None, "gpu_launches": launches, "clocks": ck,
            "iterations_run": st["iterations"],
        }
        print(json.dumps(out), flush=True)
    sh.close()
    if world > 1:
        dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="engine", choices=["engine", "reference"])
    ap.add_argument("--block-width", type=int, default=0)
    ap.add_argument("--circles", type=int, default=N_CIRCLES,
                    help="instance size (default: the benchmark workload; smaller only for profiling captures)")
    ap.add_argument("--e2e-sweeps", type=int, default=500)
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-ttr", action="store_true", help="skip the batched time-to-residual comparison")
    ap.add_argument("--mode", default="replicas", choices=["replicas", "shard"],
                    help="multi-GPU: one instance per rank (default) or one instance split over the ranks")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference_arm(args)
    elif args.mode == "shard":
        run_shard_arm(args)
    else:
        run_engine_arm(args)


if __name__ == "__main__":
    main()
