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
                    `cpu_baseline` is the reference's updateGOpenMP on the
                    same N = 8000 graph, 10 sweeps, as many host threads as
                    its int loop bounds allow there (8).
  --impl reference  the reference's own CPU path (updateGOpenMP of
                    core/paradmm.c, compiled from its sources into oracle/_ref
                    with its -Ofast flags) on up to all host cores (8 on
                    this graph: past that its int loop bounds overflow), on
                    the same N = 8000 graph: W warm-up sweeps, then K timed sweeps
                    (fewer only when K sweeps would exceed REF_BUDGET_S; the
                    line says how many ran).

Also reported: time_to_residual, the batched workload (512 instances, N in
[20, 400]) solved to r + s <= 1e-5 from the plain start and from the set-MLP
warm start (inference included), host wall clock; with N GPUs the instances
are dealt over the ranks (no communication) and the time is the slowest
rank's.

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
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "edge-updates/s"
N_CIRCLES, BOX_W, BOX_H, RMAX, SEED = 8000, 2.0, 1.0, 0.01, 20261203
RHO, RHO_R, ALPHA, EXPONENT = 10.0, 5.0, 1.0, 2.0
N_WALLS = 4
CPU_SWEEPS = 10         # cpu_baseline leg: sweeps of the reference on the full graph
REF_BUDGET_S = 150.0    # reference arm: cap on the timed sweeps' CPU time

# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) of ONE pk_persistent
# launch of NCU_SWEEPS sweeps of this workload (N = 8000, bench seed), from one
# ncu capture of `bench.py --steps 20 --warmup 3 --no-e2e --no-ttr --no-cpu`;
# profiles/pk_persistent_n8000_dram.md has the command and the figures.
NCU_DRAM_BYTES_N8000 = 15_403_251_456 + 15_773_677_824
NCU_SWEEPS = 20


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


class Clocks:
    """SM clock and throttle reasons sampled through NVML (the data
    nvidia-smi reports) by a thread that polls as fast as NVML answers,
    started before the timed region.  `stop(t0, t1)` keeps the samples whose
    host timestamps fall inside [t0, t1], the timed region; when that region
    holds fewer than three samples it adds the last sample before and the
    first after it, and says so."""

    BITS = (("hw_slowdown", 0x8), ("hw_thermal_slowdown", 0x40), ("sw_thermal_slowdown", 0x20),
            ("sw_power_cap", 0x4))

    def __init__(self, devices: list[int]):
        import threading
        self.rows: list[tuple] = []
        self.err = None
        self.run = False
        try:
            import pynvml
            import torch
            pynvml.nvmlInit()
            self.nv = pynvml
            self.h = []
            for d in devices:
                try:
                    uuid = str(torch.cuda.get_device_properties(d).uuid)
                    self.h.append(pynvml.nvmlDeviceGetHandleByUUID(uuid if uuid.startswith("GPU-") else "GPU-" + uuid))
                except Exception:
                    self.h.append(pynvml.nvmlDeviceGetHandleByIndex(d))
        except Exception as ex:  # report, never fake
            self.err = f"NVML unavailable: {str(ex)[:80]}"
            return
        self.run = True
        self.t = threading.Thread(target=self._poll, daemon=True)
        self.t.start()
        t_wait = time.perf_counter()
        while self.run and len(self.rows) < 3 and time.perf_counter() - t_wait < 2.0:  # sampling under way
            time.sleep(0.001)

    def _poll(self):
        nv = self.nv
        try:
            mx = [nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM) for h in self.h]  # fixed per device
        except Exception as ex:
            self.err = str(ex)[:80]
            self.run = False
            return
        while self.run:
            for h, m in zip(self.h, mx):
                try:
                    sm = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
                    rs = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
                    self.rows.append((time.perf_counter(), sm, m, rs))
                    time.sleep(0.0002)
                except Exception as ex:
                    self.err = str(ex)[:80]
                    self.run = False

    def stop(self, t0: float, t1: float) -> dict:
        if not self.run and not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [self.err or "no samples"], "samples": 0}
        t_wait = time.perf_counter()  # a sample after the region, when the poller is still running
        while self.run and not any(r[0] > t1 for r in self.rows[-4:]) and time.perf_counter() - t_wait < 1.0:
            time.sleep(0.001)
        self.run = False
        self.t.join(timeout=5)
        try:
            self.nv.nvmlShutdown()
        except Exception:
            pass
        rows = sorted(self.rows)
        inside = [r for r in rows if t0 <= r[0] <= t1]
        note = "samples inside the timed region"
        if len(inside) < 3:
            inside = [r for r in rows if r[0] < t0][-1:] + inside + [r for r in rows if r[0] > t1][:1]
            note = "timed region holds fewer than three NVML samples: the samples just before and after it added"
        sm = [r[1] for r in inside]
        reasons = sorted({n for r in inside for n, b in self.BITS if r[3] & b})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(r[2] for r in inside) if inside else None,
                "reasons": reasons, "samples": len(inside), "source": "NVML", "note": note,
                "timed_region_ms": round((t1 - t0) * 1e3, 3)}


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


def reference_run(n: int, warmup: int, sweeps: int, threads: int, budget_s: float | None = None) -> dict:
    """The reference's updateGOpenMP on the workload's graph with n circles
    (same box, radii, penalties and seeded start as the engine arm's rank 0):
    `warmup` untimed sweeps, then `sweeps` timed ones in one call -- fewer
    when budget_s is given and the warm-up rate says they would take longer
    (at least one)."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_lib

    import engine_b200 as eb
    lib, kind = reference_lib()
    t = time.time()
    P = oracle_lib.OraclePacking(lib, n, eb.box_walls(BOX_W, BOX_H), EXPONENT)
    P.init(SEED, BOX_W, BOX_H, RMAX, RHO, RHO_R, ALPHA)
    build_s = time.time() - t
    # the reference's updateGOpenMP overflows its int loop bounds past this
    # many threads on this graph (oracle_lib.omp_threads)
    threads = oracle_lib.omp_threads(P.G, threads)
    run = sweeps
    if warmup:
        wt = lib.orc_time_sweeps(P.graph_ptr(), warmup, threads)
        if budget_s is not None:
            run = max(1, min(sweeps, int(budget_s / (wt / warmup))))
    dt = lib.orc_time_sweeps(P.graph_ptr(), run, threads)
    E = P.G.num_edges
    P.close()
    return {"rate": E * run / dt, "seconds": dt, "edges": E, "kind": kind, "sweeps": run, "build_s": build_s,
            "threads": threads}


def run_reference_arm(args):
    world, rank = int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    n = args.circles
    r = reference_run(n, args.warmup, args.steps, os.cpu_count() or 1, REF_BUDGET_S)
    threads = r["threads"]
    sample = (f"the full N={n} graph ({r['edges']} edges), {args.warmup} warm-up + {r['sweeps']} timed sweeps of "
              f"updateGOpenMP in one call, {threads} threads (nproc {os.cpu_count()}; the reference's int loop "
              f"bounds, id * N / numthreads at core/paradmm.c:990, overflow past {threads} on this graph)")
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": r["rate"], "unit": METRIC, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": r["seconds"] / r["sweeps"] * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"plain circle packing N={n}, {BOX_W:g}x{BOX_H:g} box, radii in [0,{RMAX}], "
                               f"seeded uniform init", "circles": n, "edges": r["edges"],
                   "timed_sweeps": r["sweeps"], "graph_build_s": round(r["build_s"], 2)},
        "cpu_baseline": {"value": r["rate"], "unit": METRIC, "cores": threads, "kind": r["kind"], "sample": sample},
        "e2e": {"value": r["rate"], "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }), flush=True)


# ------------------------------------------------------------------ GPU arm
# learned arm: no fallback budget -- on this workload the warm start converges
# on more instances than the plain start, and restarting slow ones from the
# plain start only lengthened the batch (0.43 s with a 3000-sweep budget, 0.36 s
# without, device time)
TTR_INSTANCES, TTR_SEED, TTR_MAXITER, TTR_TOL, TTR_BUDGET = 512, 900000, 20000, 1e-5, 0
TTR_REPS = 3  # timed rounds of each arm (after one untimed round); the median is reported


def run_ttr(local: int, world: int = 1, rank: int = 0):
    """Time to residual on the batched workload: 512 instances (N uniform in
    [20, 400], box aspect uniform in [1, 2]), host wall clock from the solve
    call until every instance has r + s <= 1e-5 or used its iteration cap.
    plain: the batch handle's plain start.  learned: set-MLP features and
    forward, warm start, then one solve (TTR_BUDGET > 0 would restart
    instances not converged after that many sweeps from their plain start in
    the same launch).  Both run once untimed first, on the schedule the
    autotuner picked for batches of this distribution.  With world > 1 rank r
    solves its share of the instances (engine_b200.shard.split_instances; no
    communication); each arm's time is the slowest rank's and rank 0 gathers
    the per-instance results."""
    import numpy as np

    from engine_b200 import learned
    from engine_b200.shard import gather_instances, split_instances
    inst_all = learned.make_instances(TTR_INSTANCES, TTR_SEED)
    mine = split_instances([d["n_circles"] for d in inst_all], world, rank)
    inst = [inst_all[i] for i in mine]
    # schedule from the autotuner, tuned on another seeded batch of the same
    # distribution (probe = full solves to the tolerance; untimed, like
    # creating the handle), used by both arms
    tune_all = learned.make_instances(TTR_INSTANCES, TTR_SEED + 1)
    # tail hand-off: the last 1/16 of the instances still running finish
    # together on the grid-wide schedule (paradmm_gpu_set_tail_handoff)
    handoff = max(1, len(inst) // 16)
    tune = learned.tune([tune_all[i] for i in split_instances([d["n_circles"] for d in tune_all], world, rank)],
                        TTR_MAXITER, TTR_TOL, device=local, handoff=handoff)
    kw = dict(schedule=tune["schedule"], cluster=tune["cluster_size"], coop_min_n=tune["coop_min_n"],
              block_width=tune["block_width"], handoff=handoff)
    net = learned.SetMLP(device=local)
    net.load()
    # one untimed round, then TTR_REPS timed rounds of both arms, interleaved;
    # each arm's figure is the median round (host wall clock, max over ranks)
    walls_p, walls_l = [], []
    for rep in range(1 + TTR_REPS):
        barrier(world)
        pl = learned.solve_plain(inst, maxiter=TTR_MAXITER, tol=TTR_TOL, device=local, **kw)
        barrier(world)
        le = learned.solve_learned(inst, net, budget=TTR_BUDGET, maxiter=TTR_MAXITER, tol=TTR_TOL, device=local, **kw)
        if rep > 0:
            walls_p.append(allreduce_max(world, pl["wall_s"]))
            walls_l.append(allreduce_max(world, le["wall_s"]))
    net.close()
    plain_s = statistics.median(walls_p)
    learned_s = statistics.median(walls_l)

    def rows(res):
        return [(s["iterations"], int(s["converged"]), float(s["max_violation"]), float(c[:, 2].sum()),
                 int(s.get("fallback", 0))) for s, c in zip(res["stats"], res["circles"])]

    P = gather_instances(mine, rows(pl), TTR_INSTANCES, world)
    L = gather_instances(mine, rows(le), TTR_INSTANCES, world)
    if rank != 0:
        return None
    its_p = np.array([x[0] for x in P])
    its_l = np.array([x[0] for x in L])
    tot_p = sum(x[3] for x in P)
    tot_l = sum(x[3] for x in L)
    return {"workload": f"{TTR_INSTANCES} packing instances, N uniform in [20,400], aspect uniform in [1,2], "
                        f"seeded Gaussian-code plain starts (seed {TTR_SEED})",
            "tol": TTR_TOL, "maxiter": TTR_MAXITER, "learned_budget": TTR_BUDGET,
            "ranks": world, "split": "instances dealt over the ranks by size (snake order), no communication",
            "schedule": {"schedule": {1: "grid", 2: "instance", 3: "onchip"}.get(tune["schedule"], str(tune["schedule"])),
                         "block_width": tune["block_width"],
                         "cluster": tune["cluster_size"],
                         "coop_min_n": tune["coop_min_n"], "tail_handoff": handoff,
                         "autotune_candidates": tune["candidates"],
                         "probe_ms_best": tune["ms"], "probe_ms_worst": tune["worst_ms"]},
            "plain_s": plain_s,
            "plain_s_rounds": walls_p,
            "learned_s_rounds": walls_l, "learned_s": learned_s, "speedup": plain_s / learned_s,
            "converged_plain": int(sum(x[1] for x in P)), "converged_learned": int(sum(x[1] for x in L)),
            "fallbacks": int(sum(x[4] for x in L)),
            "median_sweeps_plain": int(np.median(its_p)), "median_sweeps_learned": int(np.median(its_l)),
            "sweeps_quantiles_plain": [int(q) for q in np.quantile(its_p, [0.1, 0.5, 0.9, 0.99, 1.0])],
            "sweeps_quantiles_learned": [int(q) for q in np.quantile(its_l, [0.1, 0.5, 0.9, 0.99, 1.0])],
            "total_radius_plain": tot_p, "total_radius_learned": tot_l,
            "total_radius_rel_diff": (tot_l - tot_p) / tot_p,
            "max_violation_plain": max(x[2] for x in P), "max_violation_learned": max(x[2] for x in L)}


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
    import engine_b200 as eb
    world, rank, local = dist_init()
    n = args.circles
    desc = dict(n_circles=n, walls=eb.box_walls(BOX_W, BOX_H), exponent=EXPONENT, rho=RHO, rho_radius=RHO_R,
                alpha=ALPHA, init=seeded_init(n, SEED + 1000 * rank))
    h = eb.Handle.packing([desc], device=local, block_width=args.block_width)
    h.iterate(max(3, args.warmup))
    E = edges_of(n)
    barrier(world)
    clocks = Clocks([local] if world == 1 else list(range(world))) if rank == 0 else None
    l0 = h.launches()
    t = time.perf_counter()
    s = h.solve(args.steps, -1.0)
    t_end = time.perf_counter()
    wall = t_end - t
    launches = h.launches() - l0
    barrier(world)
    ck = clocks.stop(t, t_end) if clocks else None
    dev_ms = allreduce_max(world, float(s["device_ms"]))
    st = h.instance_stats()[0]
    value = world * E * args.steps / (dev_ms * 1e-3)
    algo = algo_bytes_per_sweep(n)
    launch_ms = dev_ms / max(1, launches)
    sweeps_per_launch = args.steps / max(1, launches)
    achieved = algo * sweeps_per_launch / (launch_ms * 1e-3) / 1e9
    peak, peak_kind = measured_peak()
    traffic = None
    if NCU_DRAM_BYTES_N8000 is not None and n == N_CIRCLES:
        traffic = NCU_DRAM_BYTES_N8000 / NCU_SWEEPS * sweeps_per_launch
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
    if not args.no_ttr and n == N_CIRCLES:
        try:
            ttr = run_ttr(local, world, rank)
        except Exception as ex:  # report, never fake
            ttr = {"error": str(ex)[:200]}
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        r = reference_run(n, 1, CPU_SWEEPS, os.cpu_count() or 1)
        cpu = {"value": r["rate"], "unit": METRIC, "cores": r["threads"], "kind": r["kind"],
               "sample": f"the same N={n} graph ({r['edges']} edges), 1 warm-up + {r['sweeps']} timed sweeps of "
                         f"the reference updateGOpenMP ({r['seconds']:.1f} s), {r['threads']} threads (nproc "
                         f"{os.cpu_count()}; the reference's int loop bounds, id * N / numthreads at "
                         f"core/paradmm.c:990, overflow past {r['threads']} on this graph)"}
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
                         "traffic": traffic,
                         "traffic_source": (f"ncu dram__bytes_read.sum + dram__bytes_write.sum of one {NCU_SWEEPS}-sweep "
                                            f"launch at N={N_CIRCLES}, scaled to {sweeps_per_launch:g} sweeps")
                         if traffic is not None else None,
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
    clocks = Clocks([local] if world == 1 else list(range(world))) if rank == 0 else None
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    l0 = sh.launches()
    t = time.perf_counter()
    e0.record()
    st = run_sharded(sh, ex, allreduce, args.steps, -1.0, poll_every=max(64, args.steps))
    e1.record()
    torch.cuda.synchronize()
    t_end = time.perf_counter()
    launches = sh.launches() - l0
    barrier(world)
    ck = clocks.stop(t, t_end) if clocks else None
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
                    help="instance size (default: the benchmark workload; smaller only for profiling and tests)")
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
