"""The multi-rank plumbing of bench.py on the host (gloo, world size 2): the
max-over-ranks reduction that sets the job's time, the barrier, and the
reference arm's rule that rank 0 alone measures and prints."""
import json
import os
import socket
import subprocess
import sys


ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank: int, world: int, port: int, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world), RANK=str(rank),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import torch.distributed as dist

    import bench
    w, r, _ = bench.dist_init()
    assert (w, r) == (world, rank)
    # each rank reports its own device time; the job's time is the slowest
    got = bench.allreduce_max(w, 10.0 * (rank + 1))
    bench.barrier(w)
    q.put((rank, got, dist.get_backend()))
    dist.destroy_process_group()


def test_allreduce_max_and_barrier_over_gloo():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=10) for _ in range(2))
    assert [g for _, g, _ in res] == [20.0, 20.0]
    assert all(b == "gloo" for _, _, b in res)


def test_reference_arm_prints_once_under_torchrun():
    env = dict(os.environ, OMP_NUM_THREADS="1")
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(_free_port()),
           os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "3",
           "--circles", "300"]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=600, env=env, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, r.stdout
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["cpu_baseline"]["cores"] >= 1
    assert d["config"]["circles"] == 300 and d["config"]["edges"] == 300 + 8 * 300 + 4 * (300 * 299 // 2)
    assert d["config"]["timed_sweeps"] == 1


def test_host_memory_probe_for_the_end_to_end_leg():
    """bench.py sizes the e2e leg's host graphs against this (bytes the
    process may still allocate; a cgroup limit caps MemAvailable)."""
    sys.path.insert(0, ROOT)
    import bench
    avail = bench.host_mem_available()
    assert avail is None or avail > 0
    assert bench.E2E_HOST_BYTES >= 13.6e9  # measured peak resident size of one N = 8000 host graph


def _split_worker(rank: int, world: int, port: int, q):
    """Rank `rank` solves its share of a batch (here: a stand-in result per
    instance computed from the instance itself) and the shares are gathered
    back into the batch's order, as bench.py's time-to-residual leg does."""
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world), RANK=str(rank),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import numpy as np
    import torch.distributed as dist

    import bench
    from engine_b200.shard import gather_instances, split_instances
    w, r, _ = bench.dist_init()
    sizes = np.random.default_rng(5).integers(20, 401, 512)
    mine = split_instances(sizes, w, r)
    rows = [(int(sizes[i]), i * 7 + 1, r) for i in mine]
    out = gather_instances(mine, rows, len(sizes), w)
    t = bench.allreduce_max(w, float(r + 1))
    q.put((r, mine, out, t))
    dist.destroy_process_group()


def test_batch_split_over_ranks_and_gather_over_gloo():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_split_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=10) for _ in range(2))
    import numpy as np
    sizes = np.random.default_rng(5).integers(20, 401, 512)
    (r0, m0, o0, t0), (r1, m1, o1, t1) = res
    # every instance on exactly one rank, work balanced within 1 %
    assert sorted(m0 + m1) == list(range(512)) and not set(m0) & set(m1)
    w0, w1 = sum(int(sizes[i]) ** 2 for i in m0), sum(int(sizes[i]) ** 2 for i in m1)
    assert abs(w0 - w1) < 0.01 * (w0 + w1)
    # both ranks hold the whole batch's results in the batch's order
    assert o0 == o1
    assert [x[0] for x in o0] == [int(s) for s in sizes] and [x[1] for x in o0] == [i * 7 + 1 for i in range(512)]
    assert all(o0[i][2] == 0 for i in m0) and all(o0[i][2] == 1 for i in m1)
    assert t0 == t1 == 2.0  # the slowest rank sets each arm's time


def test_split_instances_single_rank_and_many():
    sys.path.insert(0, ROOT)
    from engine_b200.shard import gather_instances, split_instances
    sizes = [5, 400, 20, 399, 100]
    assert split_instances(sizes, 1, 0) == [1, 3, 4, 2, 0]
    parts = [split_instances(sizes, 8, r) for r in range(8)]
    assert sorted(sum(parts, [])) == list(range(5)) and sum(1 for p in parts if p) == 5
    import pytest
    with pytest.raises(ValueError):
        gather_instances([0, 1], ["a", "b"], 3, 1)
