"""Autotuner for a schedule's execution plan.

The sweeps' speed depends on how the rows are cut into CTA partitions and how each CTA's plan is
staged through shared memory; the best choice depends on the matrix (size, level widths, how many
rows of a level fall into one CTA) and on the number of right-hand sides walked together. The
autotuner times a short run of the caller's own solve (a closure) under each candidate and leaves
the schedule on the fastest:

  parts        CTAs the rows are split over: rows per CTA, and so rows per step per CTA
  smem_budget  shared memory for slots, staged right-hand sides and the two plan window buffers:
               decides whether a CTA's plan is resident or streamed, and the L1 left over

Candidates are rebuilt with `Schedule.replan` (baas_replan), which keeps the analysis, so a trial
costs one plan build and one short run.

`tune_walk` searches the other execution knobs of a single-right-hand-side solve the same way:

  walk           which sweep kernel runs (chunked, fetch, level or single-CTA walk)
  small_cluster  for the single-CTA walk, the CTAs of its cluster (1, 2, 4, 8, 16): more SMs keep more
                 loads in flight, at the price of a cluster barrier per level
"""
from __future__ import annotations

import time

from . import BaasError

DEFAULT_PARTS = (64, 96, 128, 148)
DEFAULT_BUDGETS = (0, 96 * 1024, 220 * 1024)


def _sms() -> int:
    import torch

    return torch.cuda.get_device_properties(torch.cuda.current_device()).multi_processor_count


def tune(schedule, run, parts=None, budgets=None, repeats: int = 2, warmup: int = 1) -> dict:
    """Time `run()` (a closure that calls `schedule`) for each (parts, smem_budget) candidate and
    leave `schedule` replanned with the fastest. Returns {"best": {...}, "table": [...]} with each
    candidate's best time in ms (None if the plan did not fit)."""
    import torch

    parts = tuple(p for p in (parts or DEFAULT_PARTS) if p <= min(_sms(), schedule.n))
    budgets = tuple(budgets or DEFAULT_BUDGETS)
    table = []
    best = None
    for p in parts:
        for b in budgets:
            try:
                schedule.replan(parts=p, smem_budget=b)
                for _ in range(warmup):
                    run()
                ts = []
                for _ in range(repeats):
                    e0 = torch.cuda.Event(enable_timing=True)
                    e1 = torch.cuda.Event(enable_timing=True)
                    e0.record()
                    run()
                    e1.record()
                    e1.synchronize()
                    ts.append(e0.elapsed_time(e1))
                ms = min(ts)
            except BaasError as e:
                table.append({"parts": p, "smem_budget": b, "ms": None, "why": str(e)[:80]})
                continue
            table.append({"parts": p, "smem_budget": b, "ms": round(ms, 4)})
            if best is None or ms < best["ms"]:
                best = {"parts": p, "smem_budget": b, "ms": round(ms, 4)}
    if best is None:
        raise RuntimeError("no candidate plan fits")
    t0 = time.time()
    schedule.replan(parts=best["parts"], smem_budget=best["smem_budget"])
    best["replan_s"] = round(time.time() - t0, 3)
    return {"best": best, "table": table}


DEFAULT_WALKS = ((1, 0), (2, 0), (3, 0), (4, 1), (4, 2), (4, 4), (4, 8), (4, 16))  # (walk, small_cluster)


def tune_walk(schedule, run, candidates=None, repeats: int = 2, warmup: int = 1) -> dict:
    """Time `run()` for each (walk, small_cluster) candidate (walks a schedule cannot take are
    recorded with the reason) and leave `schedule` replanned with the fastest. Returns
    {"best": {...}, "table": [...]}."""
    import torch

    table = []
    best = None
    for walk, cs in tuple(candidates or DEFAULT_WALKS):
        try:
            schedule.replan(walk=walk, small_cluster=cs)
            for _ in range(warmup):
                run()
            ts = []
            for _ in range(repeats):
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record()
                run()
                e1.record()
                e1.synchronize()
                ts.append(e0.elapsed_time(e1))
            ms = min(ts)
        except BaasError as e:
            table.append({"walk": walk, "small_cluster": cs, "ms": None, "why": str(e)[:80]})
            continue
        table.append({"walk": walk, "small_cluster": cs, "ms": round(ms, 4)})
        if best is None or ms < best["ms"]:
            best = {"walk": walk, "small_cluster": cs, "ms": round(ms, 4)}
    if best is None:
        raise RuntimeError("no candidate walk runs this schedule")
    schedule.replan(walk=best["walk"], small_cluster=best["small_cluster"])
    return {"best": best, "table": table}
