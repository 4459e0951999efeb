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
           os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "3"]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=600, env=env, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, r.stdout
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["cpu_baseline"]["cores"] >= 1


def test_host_memory_probe_for_the_end_to_end_leg():
    """bench.py sizes the e2e leg's host graphs against this (bytes the
    process may still allocate; a cgroup limit caps MemAvailable)."""
    sys.path.insert(0, ROOT)
    import bench
    avail = bench.host_mem_available()
    assert avail is None or avail > 0
    assert bench.E2E_HOST_BYTES >= 13.6e9  # measured peak resident size of one N = 8000 host graph
