"""One packing instance sharded over ranks, on one GPU.

Ranks whose kernels wait on one another never share a GPU here, and the
shard kernels never wait: a sweep is three launches per rank and an exchange
between them.  So R ranks are emulated on one device by R shard handles
launched one after another on one stream, with the all-reduce done by a
device-side sum of their exchange buffers in rank order.  The kernels are
the ones a multi-GPU run launches; only the sum's transport differs.  One
real single-rank NCCL process group checks the torch.distributed driver.
"""
import numpy as np
import pytest
import torch

import engine_b200 as eb
from engine_b200.shard import Shard, shard_rows

pytestmark = pytest.mark.gpu


def _desc(N, seed, W=1.0, H=1.0, rmax=0.05, rho=10.0, rho_r=5.0):
    return dict(n_circles=N, walls=eb.box_walls(W, H), exponent=2.0, rho=rho, rho_radius=rho_r, alpha=1.0,
                init=eb.seeded_circles(N, W, H, rmax, seed))


def _emulate(desc, R, sweeps, tol=-1.0, poll_every=16, **kw):
    """R ranks on one device; returns (shards, per-rank stats)."""
    N = desc["n_circles"]
    shards = [Shard(desc, r, R, **kw) for r in range(R)]
    st = torch.cuda.Stream()
    with torch.cuda.stream(st):
        sp = st.cuda_stream
        ex = [torch.zeros(4 * N, dtype=torch.float64, device="cuda") for _ in range(R)]
        total = torch.zeros(4 * N, dtype=torch.float64, device="cuda")
        for s in shards:
            s.start(sweeps, tol)
        done = 0
        while done < sweeps:
            n = min(poll_every, sweeps - done)
            for _ in range(n):
                for r, s in enumerate(shards):
                    s.begin(ex[r].data_ptr(), sp)
                total.copy_(ex[0])
                for r in range(1, R):
                    total.add_(ex[r])
                for s in shards:
                    s.end(total.data_ptr(), sp)
            done += n
            act = [s.poll(sp) for s in shards]
            assert len(set(act)) == 1, act  # every rank takes the same decision
            if not act[0]:
                break
        stats = [s.finish(sp) for s in shards]
    return shards, stats


def _unsharded(desc, sweeps, tol=-1.0):
    h = eb.Handle.packing([desc], schedule=eb.SCHEDULE_GRID)
    st = h.solve(sweeps, tol)
    return h, st


@pytest.mark.parametrize("N,bw", [(300, 64), (500, 128)])
def test_one_rank_equals_unsharded_bit_for_bit(N, bw):
    d = _desc(N, 11)
    h = eb.Handle.packing([d], schedule=eb.SCHEDULE_GRID, block_width=bw)
    st = h.solve(150, -1.0)
    (s,), (ss,) = _emulate(d, 1, 150, block_width=bw)
    a, b = h.circles(0, N), s.circles(0, N)
    assert np.array_equal(a, b), np.abs(a - b).max()
    assert ss["iterations"] == 150 and st["iterations"] == 150


@pytest.mark.parametrize("R", [2, 3, 5])
def test_ranks_hold_identical_consensus_close_to_unsharded(R):
    N = 600
    d = _desc(N, 21)
    h1, _ = _unsharded(dict(d), 1)
    shards, _ = _emulate(d, R, 1)
    z = [s.circles(0, N) for s in shards]
    for q in z[1:]:
        assert np.array_equal(z[0], q)  # the same summed buffer -> the same Z on every rank
    # one sweep: only the association of the FP64 sums differs
    assert np.abs(z[0] - h1.circles(0, N)).max() <= 1e-13
    h20, _ = _unsharded(dict(d), 20)
    shards20, _ = _emulate(d, R, 20)
    assert np.abs(shards20[0].circles(0, N) - h20.circles(0, N)).max() <= 1e-9


def test_rows_partition_the_tiles_and_the_memory():
    N, R = 2000, 4
    d = _desc(N, 5)
    b = shard_rows(N, R)
    shards = [Shard(d, r, R) for r in range(R)]
    assert [s.rows for s in shards] == [(int(b[r]), int(b[r + 1])) for r in range(R)]
    h = eb.Handle.packing([d], schedule=eb.SCHEDULE_GRID)
    nb = (N + 63) // 64
    per = [sum(nb - i for i in range(*s.rows)) for s in shards]
    assert sum(per) == nb * (nb + 1) // 2
    # a shard holds its own tiles only, plus the small per-circle tables
    total = nb * (nb + 1) // 2
    for s, p in zip(shards, per):
        assert s.device_bytes() <= h.device_bytes() * p / total + (2 << 20)
    assert sum(s.device_bytes() for s in shards) <= h.device_bytes() + R * (2 << 20)


def test_sharded_solve_converges_like_the_engine():
    N = 200
    d = _desc(N, 31)
    shards, stats = _emulate(d, 2, 20000, tol=1e-5, poll_every=64)
    assert all(s["converged"] for s in stats)
    assert len({s["iterations"] for s in stats}) == 1
    z = shards[0].circles(0, N)
    assert np.array_equal(z, shards[1].circles(0, N))
    ist = shards[0].instance_stats()[0]
    assert ist["primal"] + ist["dual"] <= 1e-5
    assert ist["max_violation"] < 1e-2
    h, st = _unsharded(dict(d), 20000, 1e-5)
    assert st["converged"]
    # both reach a packing of the same quality (the trajectories part after
    # many sweeps: the iteration is chaotic at the FP64 rounding level)
    assert abs(ist["total_radius"] - h.instance_stats()[0]["total_radius"]) <= 0.02 * h.instance_stats()[0]["total_radius"]


def test_warm_start_and_guards():
    N = 150
    d = _desc(N, 41)
    s = Shard(d, 1, 2)
    with pytest.raises(eb.ParadmmError):
        s.solve(10, -1.0)  # shards sweep through begin/end only
    with pytest.raises(eb.ParadmmError):
        s.begin(0)  # no run armed
    s.warm_start(0, eb.seeded_circles(N, 1.0, 1.0, 0.05, 42))
    s.start(3, -1.0)
    buf = torch.zeros(4 * N + 2, dtype=torch.float64, device="cuda")
    with pytest.raises(eb.ParadmmError):
        s.begin(buf.data_ptr() + 8)  # misaligned exchange
    with pytest.raises(eb.ParadmmError):
        eb.check(eb.load().paradmm_gpu_shard_rows(100, 64, 3, (eb.C.c_int * 4)()))  # 2 rows, 3 ranks


def test_torch_distributed_driver_single_rank_nccl():
    import os
    import socket

    import torch.distributed as dist

    from engine_b200 import shard as sh
    with socket.socket() as so:
        so.bind(("127.0.0.1", 0))
        port = so.getsockname()[1]
    os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{port}", rank=0, world_size=1)
    try:
        N = 300
        d = _desc(N, 51)
        s, st = sh.solve(d, 100, -1.0, poll_every=32)
        assert st["iterations"] == 100
        h, _ = _unsharded(dict(d), 100)
        assert np.array_equal(s.circles(0, N), h.circles(0, N))
    finally:
        dist.destroy_process_group()
