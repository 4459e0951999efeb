"""Sharding one packing instance over ranks, on the host: the row partition,
and the sweep's exchange run by two gloo ranks through the same driver
(engine_b200.shard.run_sharded) the GPU ranks use.

Each gloo rank holds the oracle's graph of the instance, takes the
reference sweep's X/M phase (core/paradmm.c:569-634), sums rho * M over the
edges its rows own into the exchange layout the shard kernels use (one
(sx, sy, sr, primal) double4 per circle), and the all-reduce of those
buffers must give the reference's consensus (updateZ, core/paradmm.c:
637-672) on every rank."""
import os
import socket
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))

import engine_b200 as eb  # noqa: E402
from engine_b200.shard import shard_rows  # noqa: E402


def _row_cost(N, BW, I):
    nI = min(BW, N - I * BW)
    return nI * (nI - 1) // 2 + nI * max(0, N - (I + 1) * BW) + nI


@pytest.mark.parametrize("N,BW", [(8000, 64), (8000, 128), (2000, 64), (700, 64)])
@pytest.mark.parametrize("R", [1, 2, 3, 4, 8])
def test_rows_cover_every_row_once_and_balance(N, BW, R):
    nb = (N + BW - 1) // BW
    if R > nb:
        return
    b = shard_rows(N, R, BW)
    assert b[0] == 0 and b[-1] == nb and all(b[r] < b[r + 1] for r in range(R))
    cost = [sum(_row_cost(N, BW, I) for I in range(b[r], b[r + 1])) for r in range(R)]
    mean = sum(cost) / R
    row_max = max(_row_cost(N, BW, I) for I in range(nb))
    # the nearest-boundary split is within one row of the even share
    assert max(cost) <= mean + row_max


def test_rows_reject_more_ranks_than_rows():
    with pytest.raises(eb.ParadmmError):
        shard_rows(100, 3, 64)  # 2 circle-block rows


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


class _HostShard:
    """The shard protocol over the oracle graph: begin = X/M phase + this
    rank's partial sums, end = consensus from the summed buffer (and the
    reference's own updateZ to compare with), then the U/N phase."""

    def __init__(self, O, N, walls, rank, R, BW, exchange):
        self.lib = O.port()
        self.orc = O.OraclePacking(self.lib, N, walls)
        self.orc.init(7, 1.0, 1.0, 0.05, 10.0, 5.0, 1.0)
        G = self.orc.G
        self.N, self.ex = N, exchange
        b = shard_rows(N, R, BW)
        lo, hi = b[rank], b[rank + 1]
        ev = np.ctypeslib.as_array(G.edgeix_to_varlistix, shape=(G.num_edges,))
        own = np.zeros(G.num_edges, dtype=bool)
        for f in range(G.num_opts):
            n = G.operatorix_to_numedges[f]
            es = np.array([G.operatorix_to_edgelistix[f][q] for q in range(n)])
            row_block = (ev[es] // 2).min() // BW  # pair (i < j): circle i's row; wall/radius: its circle's
            own[es] = lo <= row_block < hi
        self.own, self.ev = own, ev
        self.rho = G.arr("RHOS").copy()
        rs = np.zeros(G.num_vars)
        np.add.at(rs, ev, self.rho)
        self.rho_sum = rs
        self.sweeps, self.max_err, self.stopped = 0, 0.0, False

    def start(self, maxiter, tol, check_every=1):
        self.maxiter = maxiter

    def begin(self, ptr, stream):
        G = self.orc.G
        self.lib.updateXM(self.orc.graph_ptr())
        M = G.arr("M")
        e = self.own
        part = np.zeros((self.N, 4))
        cen, rad = (self.ev % 2 == 0) & e, (self.ev % 2 == 1) & e
        np.add.at(part[:, 0], self.ev[cen] // 2, self.rho[cen] * M[cen, 0])
        np.add.at(part[:, 1], self.ev[cen] // 2, self.rho[cen] * M[cen, 1])
        np.add.at(part[:, 2], self.ev[rad] // 2, self.rho[rad] * M[rad, 0])
        self.ex.copy_(__import__("torch").from_numpy(part.reshape(-1)))

    def end(self, ptr, stream):
        G = self.orc.G
        tot = self.ex.numpy().reshape(self.N, 4)
        z = np.stack([tot[:, 0] / self.rho_sum[0::2], tot[:, 1] / self.rho_sum[0::2],
                      tot[:, 2] / self.rho_sum[1::2]], axis=1)
        self.lib.updateZ(self.orc.graph_ptr())
        Z = G.arr("Z")
        ref = np.stack([Z[0::2, 0], Z[0::2, 1], Z[1::2, 0]], axis=1)
        self.max_err = max(self.max_err, float(np.abs(z - ref).max()))
        self.last_z = z
        self.lib.updateUN(self.orc.graph_ptr())
        self.sweeps += 1

    def poll(self, stream):
        return self.sweeps < self.maxiter

    def finish(self, stream):
        return {"iterations": self.sweeps}


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import torch
    import torch.distributed as dist

    import oracle_lib as O
    from engine_b200.shard import run_sharded
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        N = 150  # 3 circle-block rows of 64
        ex = torch.zeros(4 * N, dtype=torch.float64)
        sh = _HostShard(O, N, eb.box_walls(1.0, 1.0), rank, world, 64, ex)
        calls = [0]

        def allreduce(t):
            calls[0] += 1
            dist.all_reduce(t)

        st = run_sharded(sh, ex, allreduce, maxiter=40, tol=-1.0, poll_every=8)
        q.put((rank, st["iterations"], calls[0], sh.max_err, sh.last_z.tobytes()))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_reproduce_the_reference_consensus():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(300)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=10) for _ in range(2))
    assert [r[1] for r in res] == [40, 40] and [r[2] for r in res] == [40, 40]
    assert res[0][4] == res[1][4]  # identical consensus on both ranks
    assert max(r[3] for r in res) <= 1e-12  # the sharded sums are the reference's, up to association


def _leaver(rank, world, port, q):
    """Rank 1 runs 10 sweeps and exits; rank 0 asks for 40 and must get an
    error from its next exchange, not wait for ever."""
    import datetime

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import torch
    import torch.distributed as dist

    import oracle_lib as O
    from engine_b200.shard import run_sharded
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=10))
    N = 150
    ex = torch.zeros(4 * N, dtype=torch.float64)
    sh = _HostShard(O, N, eb.box_walls(1.0, 1.0), rank, world, 64, ex)
    try:
        st = run_sharded(sh, ex, lambda t: dist.all_reduce(t), maxiter=10 if rank == 1 else 40, tol=-1.0,
                         poll_every=5)
        q.put((rank, "done", st["iterations"]))
    except Exception as e:  # the failure under test, reported to the parent
        q.put((rank, "error", sh.sweeps, type(e).__name__))
    if rank == 1:
        q.close()
        q.join_thread()  # the report reaches the parent before the process vanishes
        os._exit(0)      # leaves between sweeps, without a goodbye to the group
    dist.destroy_process_group()


def test_a_rank_leaving_ends_the_others_run_with_an_error():
    import time

    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_leaver, args=(r, 2, port, q)) for r in range(2)]
    t0 = time.time()
    for p in procs:
        p.start()
    try:
        res = sorted(q.get(timeout=120) for _ in range(2))
    finally:
        for p in procs:
            p.join(60)
            if p.is_alive():
                p.kill()
    assert res[1][1:] == ("done", 10)
    assert res[0][1] == "error" and res[0][2] == 10  # rank 0 stopped at its first exchange without the peer
    assert time.time() - t0 < 120
