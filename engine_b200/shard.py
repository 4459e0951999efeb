"""One packing instance sharded over ranks, one process per GPU.

Rank r of R stores and sweeps the pair tiles of its circle-block rows (rows
balanced by pair count, paradmm_gpu_shard_rows) and the wall and radius
factors of those rows' circles, and keeps the whole consensus Z.  A sweep is

    shard.begin(exchange)       pass over the rank's tiles, then its partial
                                consensus sums (32 bytes per circle) into
                                `exchange`
    allreduce(exchange)         float64 sum over the ranks, in place
                                (torch.distributed: NCCL over NVLink)
    shard.end(exchange)         Z, residuals and the stop test from the sum

so the only traffic between GPUs is one all-reduce of 32 N bytes per sweep
(256 KB at N = 8000).  Every rank derives Z from the same summed buffer, so
the ranks hold identical Z and stop at the same sweep; with one rank the
sweep equals the unsharded engine's bit for bit.  The reference has no
multi-device path (core/paradmm-gpu.cu runs one graph on one device); the
per-variable consensus it shards is updateZ, core/paradmm.c:637-672.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import ENONFINITE, OK, Handle, Stats, check, load, opts


def shard_rows(n_circles: int, nranks: int, block_width: int = 64) -> np.ndarray:
    """Row bounds [nranks + 1]: rank r owns circle-block rows [b[r], b[r+1])."""
    b = (C.c_int * (nranks + 1))()
    check(load().paradmm_gpu_shard_rows(int(n_circles), int(block_width), int(nranks), b))
    return np.array(list(b), dtype=np.int64)


class Shard(Handle):
    """A paradmm_gpu handle holding rank `rank` of `nranks` of one instance."""

    def __init__(self, desc: dict, rank: int, nranks: int, **kw):
        lib = load()
        arr, keep = Handle._descs([desc])
        p = C.c_void_p()
        o = opts(**kw)
        check(lib.paradmm_gpu_create_packing_shard(arr, int(rank), int(nranks), C.byref(o), C.byref(p)))
        del keep
        super().__init__(p.value, lib)
        self.rank, self.nranks = int(rank), int(nranks)
        self.n_circles = int(desc["n_circles"])
        lo, hi, nb = C.c_int(), C.c_int(), C.c_int64()
        check(lib.paradmm_gpu_shard_info(self.ptr, C.byref(lo), C.byref(hi), C.byref(nb)))
        self.rows = (lo.value, hi.value)
        self.exchange_bytes = nb.value

    def start(self, maxiter: int, tol: float, check_every: int = 1) -> None:
        check(self.lib.paradmm_gpu_shard_start(self.ptr, int(maxiter), float(tol), int(check_every)))

    def begin(self, exchange_ptr: int, stream: int = 0) -> None:
        check(self.lib.paradmm_gpu_shard_begin(self.ptr, C.c_void_p(exchange_ptr), C.c_void_p(stream or None)))

    def end(self, exchange_ptr: int, stream: int = 0) -> None:
        check(self.lib.paradmm_gpu_shard_end(self.ptr, C.c_void_p(exchange_ptr), C.c_void_p(stream or None)))

    def poll(self, stream: int = 0) -> bool:
        a = C.c_int()
        check(self.lib.paradmm_gpu_shard_poll(self.ptr, C.c_void_p(stream or None), C.byref(a)))
        return bool(a.value)

    def fused_buffers(self) -> tuple[int, int]:
        """(exchange, flags) device pointers of this rank for the fused run."""
        ex, fl = C.c_void_p(), C.c_void_p()
        check(self.lib.paradmm_gpu_shard_fused_buffers(self.ptr, C.byref(ex), C.byref(fl)))
        return ex.value, fl.value

    def finish(self, stream: int = 0) -> dict:
        s = Stats()
        rc = self.lib.paradmm_gpu_shard_finish(self.ptr, C.c_void_p(stream or None), C.byref(s))
        if rc not in (OK, ENONFINITE):
            check(rc)
        return s.as_dict()


def run_sharded(shard, exchange, allreduce, maxiter: int, tol: float, poll_every: int = 64,
                check_every: int = 1) -> dict:
    """Drives one run: `poll_every` sweeps of [begin, allreduce, end] between
    polls, until the instance stops or maxiter sweeps ran.  `exchange` is a
    tensor of exchange_bytes on the shard's device (CPU for a host-side
    shard); `allreduce(exchange)` sums it over the ranks in place.  Every
    rank polls after the same sweeps and gets the same answer, so all ranks
    issue the same collectives.  Kernels go to torch's current stream, where
    the collectives are ordered too."""
    import torch

    stream = torch.cuda.current_stream().cuda_stream if exchange.is_cuda else 0
    ptr = exchange.data_ptr()
    shard.start(maxiter, tol, check_every)
    done = 0
    while done < maxiter:
        n = min(poll_every, maxiter - done)
        for _ in range(n):
            shard.begin(ptr, stream)
            allreduce(exchange)
            shard.end(ptr, stream)
        done += n
        if not shard.poll(stream):
            break
    return shard.finish(stream)


def solve(desc: dict, maxiter: int, tol: float, group=None, poll_every: int = 64, **kw) -> tuple[Shard, dict]:
    """Solves one instance over the ranks of `group` (torch.distributed,
    initialised by the caller; one rank per GPU, device = the current CUDA
    device).  Returns this rank's shard (whole consensus: shard.circles(0, N))
    and the run's stats."""
    import torch
    import torch.distributed as dist

    rank = dist.get_rank(group) if dist.is_initialized() else 0
    world = dist.get_world_size(group) if dist.is_initialized() else 1
    dev = torch.cuda.current_device()
    shard = Shard(desc, rank, world, device=dev, **kw)
    exchange = torch.zeros(shard.exchange_bytes // 8, dtype=torch.float64, device=f"cuda:{dev}")

    def allreduce(t):
        if world > 1:
            dist.all_reduce(t, group=group)

    return shard, run_sharded(shard, exchange, allreduce, maxiter, tol, poll_every)


def run_fused(shards, exchanges, flags, wait_ms: int = 0, stream: int = 0) -> None:
    """paradmm_gpu_shard_run_fused: the armed runs of `shards` (consecutive
    ranks on one device) in one persistent launch with the exchange fused in.
    exchanges[q] / flags[q]: rank q's buffers as this device addresses them,
    for every rank q of the split."""
    lib = load()
    n = len(shards)
    hs = (C.c_void_p * n)(*[s.ptr for s in shards])
    R = len(exchanges)
    ex = (C.c_void_p * R)(*exchanges)
    fl = (C.c_void_p * R)(*flags)
    check(lib.paradmm_gpu_shard_run_fused(hs, n, ex, fl, int(wait_ms), C.c_void_p(stream or None)))


def solve_fused(desc: dict, maxiter: int, tol: float, group=None, wait_ms: int = 0, **kw) -> tuple[Shard, dict]:
    """One instance over the ranks of `group` (torch.distributed, one rank per
    GPU) in one persistent launch per GPU: the ranks' exchange buffers and
    flags are shared through CUDA IPC, each rank's kernel stores its partial
    sums into every peer's buffer over NVLink and waits on their flags; the
    only host collectives are the handle exchange before the run and a
    barrier after it."""
    import torch
    import torch.distributed as dist

    lib = load()
    rank = dist.get_rank(group) if dist.is_initialized() else 0
    world = dist.get_world_size(group) if dist.is_initialized() else 1
    dev = torch.cuda.current_device()
    shard = Shard(desc, rank, world, device=dev, **kw)
    ex, fl = shard.fused_buffers()
    mine = [bytes(64), bytes(64)]
    for j, ptr in enumerate((ex, fl)):
        buf = C.create_string_buffer(64)
        check(lib.paradmm_gpu_ipc_export(C.c_void_p(ptr), buf))
        mine[j] = buf.raw
    every = [None] * world
    if world > 1:
        dist.all_gather_object(every, (rank, mine[0], mine[1]), group=group)
    else:
        every = [(rank, mine[0], mine[1])]
    exchanges, flags, opened = [0] * world, [0] * world, []
    try:
        for q, hx, hf in every:
            if q == rank:
                exchanges[q], flags[q] = ex, fl
                continue
            for j, hnd in enumerate((hx, hf)):
                p = C.c_void_p()
                check(lib.paradmm_gpu_ipc_import(dev, C.create_string_buffer(hnd, 64), C.byref(p)))
                opened.append(p.value)
                (exchanges if j == 0 else flags)[q] = p.value
        shard.start(maxiter, tol)
        stream = torch.cuda.current_stream().cuda_stream
        run_fused([shard], exchanges, flags, wait_ms, stream)
        stats = shard.finish(stream)
    finally:
        if world > 1:
            dist.barrier(group=group)  # no rank still writes into a buffer about to be unmapped
        for p in opened:
            lib.paradmm_gpu_ipc_close(dev, C.c_void_p(p))
    return shard, stats


# ------------------------------------------------------- batches over ranks
def split_instances(sizes, world: int, rank: int) -> list[int]:
    """Indices of the instances rank `rank` of `world` solves when a batch of
    independent packing instances is dealt over the ranks (no communication
    between them).  The instances are taken largest first (a sweep's work
    grows with N^2) and dealt in snake order 0, 1, .., R-1, R-1, .., 0, 0, ..
    so every rank gets a near-equal share of the work; each rank's list keeps
    that order (largest first).  Every index goes to exactly one rank."""
    order = sorted(range(len(sizes)), key=lambda i: (-int(sizes[i]), i))
    mine = []
    for k, i in enumerate(order):
        lap, pos = divmod(k, world)
        owner = pos if lap % 2 == 0 else world - 1 - pos
        if owner == rank:
            mine.append(i)
    return mine


def gather_instances(mine: list[int], rows: list, total: int, world: int, group=None):
    """Per-instance results of a batch dealt by split_instances, back in the
    batch's order on every rank: rows[k] belongs to instance mine[k].  With
    world > 1 every rank takes part (torch.distributed all_gather_object)."""
    parts = [(list(mine), list(rows))]
    if world > 1:
        import torch.distributed as dist
        parts = [None] * world
        dist.all_gather_object(parts, (list(mine), list(rows)), group=group)
    out = [None] * total
    for idx, rs in parts:
        for i, r in zip(idx, rs):
            if out[i] is not None:
                raise ValueError(f"instance {i} reported by two ranks")
            out[i] = r
    missing = [i for i, r in enumerate(out) if r is None]
    if missing:
        raise ValueError(f"{len(missing)} instances reported by no rank (first {missing[0]})")
    return out
