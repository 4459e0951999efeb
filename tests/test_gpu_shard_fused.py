"""The sharded instance with its exchange fused into one persistent launch
(paradmm_gpu_shard_run_fused), on one GPU.

All R ranks run in ONE cooperative launch (every CTA co-resident), each
rank's CTAs storing their partial sums into every rank's exchange buffer and
raising their flags there, exactly as one launch per GPU does with peer
pointers; only the memory the stores land in differs.  The reference for it
is the split shard path (tests/test_gpu_shard.py), whose all-reduce is a
device-side sum in rank order -- the order the fused kernel sums the slots
in -- so the two agree bit for bit.
"""
import numpy as np
import pytest
import torch

import engine_b200 as eb
from engine_b200.shard import Shard, run_fused
from test_gpu_shard import _desc, _emulate

pytestmark = pytest.mark.gpu


def _fused(desc, R, sweeps, tol=-1.0, wait_ms=0, **kw):
    shards = [Shard(desc, r, R, **kw) for r in range(R)]
    bufs = [s.fused_buffers() for s in shards]
    for s in shards:
        s.start(sweeps, tol)
    run_fused(shards, [b[0] for b in bufs], [b[1] for b in bufs], wait_ms)
    return shards, [s.finish() for s in shards]


@pytest.mark.parametrize("R", [1, 2, 3, 4])
def test_fused_equals_split_path_bit_for_bit(R):
    N = 600
    d = _desc(N, 21)
    fs, fst = _fused(d, R, 60)
    ss, sst = _emulate(d, R, 60)
    z = fs[0].circles(0, N)
    for q in range(R):
        assert np.array_equal(fs[q].circles(0, N), z)  # every rank holds the same Z
        assert np.array_equal(ss[q].circles(0, N), z), np.abs(ss[q].circles(0, N) - z).max()
        assert fst[q]["iterations"] == sst[q]["iterations"] == 60


def test_one_fused_rank_equals_unsharded_bit_for_bit():
    N = 300
    d = _desc(N, 11)
    h = eb.Handle.packing([d], schedule=eb.SCHEDULE_GRID)
    h.solve(150, -1.0)
    (s,), (st,) = _fused(d, 1, 150)
    assert np.array_equal(h.circles(0, N), s.circles(0, N))
    assert st["iterations"] == 150


def test_fused_run_stops_where_the_split_path_stops():
    N = 200
    d = _desc(N, 31)
    fs, fst = _fused(d, 2, 20000, tol=1e-5)
    ss, sst = _emulate(d, 2, 20000, tol=1e-5, poll_every=1)
    assert all(s["converged"] for s in fst)
    assert len({s["iterations"] for s in fst}) == 1
    assert fst[0]["iterations"] == sst[0]["iterations"], (fst[0]["iterations"], sst[0]["iterations"])
    assert np.array_equal(fs[0].circles(0, N), ss[0].circles(0, N))
    assert np.array_equal(fs[0].circles(0, N), fs[1].circles(0, N))
    # a second armed run continues from there (new flag epoch, same buffers)
    for s in fs:
        s.start(10, -1.0)
    bufs = [s.fused_buffers() for s in fs]
    run_fused(fs, [b[0] for b in bufs], [b[1] for b in bufs])
    st2 = [s.finish() for s in fs]
    assert all(x["iterations"] == 10 for x in st2)
    assert np.array_equal(fs[0].circles(0, N), fs[1].circles(0, N))


def test_a_rank_that_never_runs_ends_the_wait_with_a_timeout():
    """Rank 1's flags are never raised (its kernel is never launched): rank
    0's bounded wait runs out, the call reports PARADMM_ETIMEOUT, and the
    device keeps working."""
    N = 300
    d = _desc(N, 51)
    s0, s1 = Shard(d, 0, 2), Shard(d, 1, 2)
    b0, b1 = s0.fused_buffers(), s1.fused_buffers()
    s0.start(50, -1.0)
    with pytest.raises(eb.ParadmmError) as e:
        run_fused([s0], [b0[0], b1[0]], [b0[1], b1[1]], wait_ms=300)
    assert e.value.status == eb.ETIMEOUT
    h = eb.Handle.packing([d], schedule=eb.SCHEDULE_GRID)
    assert h.solve(20, -1.0)["iterations"] == 20
    torch.cuda.synchronize()


def test_fused_guards():
    N = 150
    d = _desc(N, 41)
    a, b = Shard(d, 0, 2), Shard(d, 1, 2)
    ba, bb = a.fused_buffers(), b.fused_buffers()
    with pytest.raises(eb.ParadmmError):
        run_fused([a, b], [ba[0], bb[0]], [ba[1], bb[1]])  # no run armed
    a.start(5, -1.0)
    b.start(5, -1.0)
    with pytest.raises(eb.ParadmmError):
        run_fused([b, a], [ba[0], bb[0]], [ba[1], bb[1]])  # ranks out of order
    with pytest.raises(eb.ParadmmError):
        run_fused([a, b], [ba[0] + 8, bb[0]], [ba[1], bb[1]])  # misaligned exchange
    a.begin(torch.zeros(4 * N, dtype=torch.float64, device="cuda").data_ptr())
    with pytest.raises(eb.ParadmmError):
        run_fused([a, b], [ba[0], bb[0]], [ba[1], bb[1]])  # a run already stepped by begin/end
