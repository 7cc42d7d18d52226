"""Batched systems across GPUs: one process per GPU, each solving whole systems of the batch.

A single triangular solve or factorisation does not shard (its dependency DAG crosses any
partition at every level), but a batch of independent systems does: each rank takes a subset of
the systems, solves them in one batched launch on its own GPU with no communication at all, and a
single gather afterwards brings every system's iterations, residuals and solution to rank 0.

The split is deterministic (every rank computes the same assignment from the systems' sizes):
longest-processing-time first -- systems in decreasing size, each to the rank with the fewest rows
so far (ties to the lower rank) -- so the ranks' row counts differ by at most one system's rows.
"""
from __future__ import annotations

from typing import Callable, Sequence


def split_systems(sizes: Sequence[int], world: int) -> list[list[int]]:
    """Indices of the systems each of `world` ranks solves, each list ascending."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(sizes)), key=lambda q: (-int(sizes[q]), q))
    load = [0] * world
    parts: list[list[int]] = [[] for _ in range(world)]
    for q in order:
        r = min(range(world), key=lambda k: (load[k], k))
        parts[r].append(q)
        load[r] += int(sizes[q])
    return [sorted(p) for p in parts]


def solve_sharded(systems: Sequence, solve: Callable[[list[int]], dict], rank: int, world: int, group=None):
    """Solves this rank's share of `systems` with solve(indices) -> {system index: result} (and
    optionally key -1: a per-rank value such as its launch time) and gathers every rank's results
    to rank 0 (torch.distributed, any backend; world == 1 needs no process group). Returns the
    merged {system index: result} on rank 0, with key -1 mapping rank -> its value; None elsewhere."""
    mine = split_systems([S.n for S in systems], world)[rank]
    local = solve(mine)
    if set(local) - {-1} != set(mine):
        raise RuntimeError("solve() must return one result per system it was given (and optionally key -1)")
    if world == 1:
        out = dict(local)
        if -1 in out:
            out[-1] = {0: out[-1]}
        return out
    import torch.distributed as dist

    gathered = [None] * world if rank == 0 else None
    dist.gather_object(local, gathered, dst=0, group=group)
    if rank != 0:
        return None
    out: dict = {}
    for r, part in enumerate(gathered):
        for q, v in part.items():
            if q == -1:
                out.setdefault(-1, {})[r] = v  # each rank's extra entry (its launch time)
            else:
                out[q] = v
    if len([q for q in out if q != -1]) != len(systems):
        raise RuntimeError("the gathered results do not cover every system")
    return out


def batched_solve(systems: Sequence, idx: Sequence[int], rhs: Callable[[int], "np.ndarray"], device=None,
                  tol: float = 1e-10, maxiter: int = 20000, precision: int = 1, timed: bool = True) -> dict:
    """One rank's share: the systems `idx` concatenated into one batch (BatchSchedule) and solved
    in one launch on `device`; rhs(q) gives system q's right-hand sides (nrhs x n_q). Returns
    {q: {"iterations", "relres", "x"}} per system, plus the launch time in ms under key -1 when
    `timed` (a warm-up solve first, then one timed with CUDA events)."""
    import numpy as np
    import torch

    from . import BatchSchedule, DeviceCSR

    if len(idx) == 0:
        return {-1: 0.0} if timed else {}
    sub = [systems[q] for q in idx]
    s = BatchSchedule(sub, nthread=8)
    dev = torch.device("cuda") if device is None else device
    dA = DeviceCSR.from_host(s.combined, device=dev)
    B = torch.from_numpy(np.concatenate([np.atleast_2d(rhs(q)) for q in idx], axis=1)).to(dev)
    X = torch.zeros_like(B)

    def run():
        X.zero_()
        return s.iccg_batched(dA, B, X, tol=tol, maxiter=maxiter, precision=precision)

    ms = 0.0
    if timed:
        run()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        it, rel = run()
        e1.record()
        e1.synchronize()
        ms = e0.elapsed_time(e1)
    else:
        it, rel = run()
    Xh = X.cpu().numpy()
    off = s.sys_off
    out = {q: {"iterations": it[j].tolist(), "relres": rel[j].tolist(), "x": Xh[:, int(off[j]):int(off[j + 1])]}
           for j, q in enumerate(idx)}
    if timed:
        out[-1] = ms
    return out
