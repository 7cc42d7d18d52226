"""Benchmark of the BAAS sparse hot path on B200: ICCG time-to-1e-10 on the 64^3 7-point system.

Workload (the configuration the headline metric is quoted on): IC0-preconditioned CG on the 3-D
7-point Laplacian of 64^3 (n = 262,144, nnz(A) = 1,810,432) with diagonal shift 1e-3, natural
ordering, b ~ U(-1,1) with seed 1, x0 = 0, stop at relative residual 1e-10 or 2,000 iterations.
Synthetic inputs (seeded generators in baas_b200/gen.py); no dataset is involved.

A step is one complete solve: IC0 factorisation of A, then the PCG loop until convergence, i.e.
one launch of the persistent ICCG kernel with A, b, x resident in HBM (the schedule analysis is
done once beforehand and reported separately, as the reference separates Scheduling_Time from
Executor_Runtime). L2 (126 MB) is flushed before every timed step; every step is timed with CUDA
events on the launching stream. `e2e` repeats the solve through the public API with pinned host
buffers: A.values, b and x0 copied host->device and x copied back inside the timed region.

`--impl reference` times the reference's own OpenMP ICCG (its Scheduler + runIC0 + p2p sweeps and
its BLAS-1/SpMV, compiled from its sources into oracle/_ref) on the host cores.

Multi-GPU: a single solve does not shard (the triangular sweeps carry a dependence through every
level), so N GPUs run N independent replicas ("replicas only"); the time is the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "ICCG time-to-1e-10 (64^3 7-pt Laplacian + 1e-3 I, IC0-PCG, FP64), 1 B200"
UNIT = "ms"
K_GRID = 64
TOL = 1e-10
MAXITER = 2000
# algorithmic bytes (reference bandwidth model, test/iccg_level_merge.cpp:509-510, written out
# for the 64^3 system): per PCG iteration SpMV 12*nnz(A)+4(n+1)+16n, two sweeps
# 12*nnz(L)+4(n+1)+16n each, vector work 112n; the IC0 factorisation reads A (12*nnz+4(n+1))
# and writes the factor values (8*nnz).
N = K_GRID ** 3
NNZ_A = 1_810_432
NNZ_L = (NNZ_A + N) // 2
SPMV_BYTES = 12 * NNZ_A + 4 * (N + 1) + 16 * N
SWEEP_BYTES = 12 * NNZ_L + 4 * (N + 1) + 16 * N
VEC_BYTES = 112 * N
ITER_BYTES = SPMV_BYTES + 2 * SWEEP_BYTES + VEC_BYTES
IC0_BYTES = 12 * NNZ_A + 4 * (N + 1) + 8 * NNZ_A
CPU_BASELINES = True  # --no-cpu-baseline clears it


def _peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def _host_cores() -> int:
    """Physical cores this process may run on (the reference's OMP_NUM_THREADS)."""
    try:
        import psutil

        phys = psutil.cpu_count(logical=False) or 1
    except Exception:
        phys = os.cpu_count() or 1
    try:
        allowed = len(os.sched_getaffinity(0))
    except Exception:
        allowed = phys
    return max(1, min(phys, allowed))


def _dist():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


class ClockSampler:
    """nvidia-smi samples (200 ms) during the timed region."""

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = Path(os.environ.get("BAAS_CLOCK_LOG", f"/tmp/baas_clocks_{os.getpid()}.csv"))

    def __enter__(self):
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            time.sleep(0.3)
            self.proc.terminate()
            self.proc.wait()

    def summary(self):
        try:
            rows = [r.split(",") for r in self.path.read_text().strip().splitlines() if r.strip()]
        except Exception:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[0]) for r in rows if r[0].strip().replace(".", "").isdigit()]
        mx = [float(r[1]) for r in rows if r[1].strip().replace(".", "").isdigit()]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            for k, nm in enumerate(names):
                if len(r) > 3 + k and "Active" in r[3 + k] and "Not" not in r[3 + k]:
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(rows)}


def reference_arm(args):
    """The reference's OpenMP ICCG on the host cores (rank 0 only)."""
    world, rank, _ = _dist()
    if rank != 0:
        return
    from baas_b200 import gen
    from oracle.oracle import Ref, ref_available

    if not ref_available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libbaas_ref.so was not built"}))
        return
    cores = _host_cores()
    A = gen.laplace3d(K_GRID, 1e-3)
    b = gen.uniform_rhs(A.n, 1)
    for _ in range(args.warmup):
        Ref.pcg(A, b, maxiter=MAXITER, tol=TOL, mode=1, nthread=cores)
    times, iters, pre, rel = [], 0, [], None
    for _ in range(args.steps):
        x, iters, rel, t = Ref.pcg(A, b, maxiter=MAXITER, tol=TOL, mode=1, nthread=cores)
        times.append(t[1] + t[2])  # IC0 + initial residual + PCG loop (analysis excluded, as on the GPU arm)
        pre.append(t[0])
    v = float(np.mean(times))
    line = {
        "impl": "reference", "metric": METRIC, "value": round(v, 3), "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(v, 3), "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "iccg_laplace3d_64_shift1e-3", "n": A.n, "nnz": A.nnz, "tol": TOL,
                   "iterations": int(iters), "relres": rel, "parallelism": f"openmp{cores}",
                   "l2": "host CPU run"},
        "cpu_baseline": {"value": round(v, 3), "unit": UNIT, "cores": cores, "kind": "reference",
                         "sample": f"{args.steps} full solves (IC0 + PCG to 1e-10) with the reference's "
                                   f"Scheduler P2P_RULE at nthread={cores}"},
        "e2e": {"value": round(v, 3), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "analysis_ms": round(float(np.mean(pre)), 3),
    }
    print(json.dumps(line))


def cpu_baseline_sample():
    """Bounded CPU sample of the same workload with the reference library (1 solve)."""
    from baas_b200 import gen
    from oracle.oracle import Ref, ref_available

    cores = _host_cores()
    if not ref_available():
        return None
    A = gen.laplace3d(K_GRID, 1e-3)
    b = gen.uniform_rhs(A.n, 1)
    xr, it, _, t = Ref.pcg(A, b, maxiter=MAXITER, tol=TOL, mode=1, nthread=cores)
    return {"value": round(float(t[1] + t[2]), 3), "unit": UNIT, "cores": cores, "kind": "reference",
            "sample": f"1 full solve (IC0 + {it} PCG iterations to 1e-10) with the reference's OpenMP "
                      f"Scheduler P2P_RULE path, nthread={cores}; analysis {t[0]:.1f} ms excluded"}, xr


def _event_ms(fn, reps=3, flush=None):
    """Best CUDA-event time of fn() over reps runs (after one untimed run)."""
    import torch

    fn()
    ts = []
    for _ in range(reps):
        if flush is not None:
            flush.fill_(1.0)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        fn()
        e1.record()
        e1.synchronize()
        ts.append(e0.elapsed_time(e1))
    return float(min(ts))


# Latency model of a triangular sweep (the sweeps are dependency-chain bound, not bandwidth bound:
# the whole working set stays in L2). A sweep cannot finish before its critical path has run one
# compute step per level of the group DAG and one CTA-to-CTA hop per partition boundary on that
# path. Both constants are B200 measurements of the fetch walk (fetch.cuh): STEP_US is a step of a
# CTA that never waits (the 64^3 FP64 lower sweep's first CTA: 46 steps in 7.3 us, %globaltimer
# stamps); HOP_US is one value crossing between CTAs through L2 (store, then a poll that sees it:
# 889 cycles one way at 1965 MHz, a two-CTA ping-pong).
STEP_US = 0.16
HOP_US = 0.45


def sweep_latency_bound(s):
    """Lower bound (us) of one sweep of schedule s: levels x STEP_US + hops x HOP_US, where hops
    are the box boundaries a monotone path crosses (grid boxes) or the CTA boundaries (ranges)."""
    levels = int(s.export("nlevels")[0])
    parts, box, nbox = s.plan_parts()
    hops = sum(c - 1 for c in nbox) if nbox else max(parts - 1, 0)
    return {"levels": levels, "hops": hops, "step_us": STEP_US, "hop_us": HOP_US,
            "bound_us": round(levels * STEP_US + hops * HOP_US, 2), "parts": parts,
            "box": list(box) if box else None}


def _ref_ms(fn, reps):
    """Mean wall time (ms) of fn() on the host over reps runs, after one untimed run."""
    fn()
    t0 = time.perf_counter()
    for _ in range(reps):
        fn()
    return (time.perf_counter() - t0) * 1e3 / reps


def c1_cpu_baseline(L, b):
    """The reference's BAAS p2p forward sweep (SpTRSV_DUAL_TREE_BFS_WF_Merge_P2P_MapFourRule's
    schedule, merge/SpTRSV.cpp:421-478) on all host cores."""
    from oracle.oracle import Ref, ref_available

    if not ref_available():
        return None
    cores = _host_cores()
    rs = Ref.Schedule(0, L, cores)
    ms = _ref_ms(lambda: rs.forward(L, b), 200)
    return {"value": round(ms, 4), "unit": "ms", "cores": cores, "kind": "reference",
            "sample": f"200 forward sweeps of the 128^2 lower triangle, reference p2p sweep at nthread={cores} (mean)"}


def c1_sptrsv(flush):
    """The 128x128 5-point lower-triangle forward sweep (SpTRSV HBM GB/s)."""
    import torch

    from baas_b200 import KERNEL_SPTRSV, DeviceCSR, Schedule, gen

    L, x_true, b = gen.sptrsv_case(128, 0)
    s = Schedule(L, kind=KERNEL_SPTRSV, nthread=8)
    dL = DeviceCSR.from_host(L)
    db = torch.from_numpy(b).cuda()
    x = torch.zeros_like(db)
    ms = _event_ms(lambda: s.forward(dL, db, x), 10, flush)
    nbytes = 12 * L.nnz + 4 * (L.n + 1) + 16 * L.n
    xg = x.cpu().numpy()
    err = float(np.max(np.abs(xg - x_true)))
    peak, peak_kind = _peaks()
    gbps = nbytes / (ms * 1e-3) / 1e9
    lat = sweep_latency_bound(s)
    lat["frac"] = round(lat["bound_us"] / (ms * 1e3), 4)
    # the single-CTA walk on the same sweep (253 row levels: the automatic choice keeps the fetch walk)
    from baas_b200 import WALK_SMALL

    s1 = Schedule(L, kind=KERNEL_SPTRSV, nthread=8, walk=WALK_SMALL)
    x1 = torch.zeros_like(db)
    ms1 = _event_ms(lambda: s1.forward(dL, db, x1), 10, flush)
    same1 = bool(torch.equal(x1, x))
    out = {"workload": "sptrsv_laplace2d_128_lower", "ms": round(ms, 4), "bytes": nbytes, "gbps": round(gbps, 2),
           "max_abs_err_vs_x_true": err, "walk": s.last_walk,
           "single_cta_walk": {"ms": round(ms1, 4), "bitexact_vs_auto": same1},
           "roofline": {"bound": "hbm", "achieved": round(gbps, 2), "peak": peak, "unit": "GB/s",
                        "frac": round(gbps / peak, 5), "peak_kind": peak_kind, "kernel": "k_sweep_fetch"},
           "latency_bound": lat}
    if CPU_BASELINES:
        out["cpu_baseline"] = c1_cpu_baseline(L, b)
    return out


def c3_ilu(flush):
    """ILU0 of the 96^3 upwind convection-diffusion operator and its apply on 8 right-hand sides."""
    import scipy.sparse as sp
    import torch

    from baas_b200 import KERNEL_ILU0, DeviceCSR, Schedule, gen

    C = gen.convdiff3d(96)
    s = Schedule(C, kind=KERNEL_ILU0, nthread=8)
    dC = DeviceCSR.from_host(C)
    lu = dC.values.clone()
    ilu_ms = _event_ms(lambda: (lu.copy_(dC.values), s.ilu0(dC, lu)), 3, flush)
    M = gen.CSR(C.n, C.rowptr, C.colidx, lu.cpu().numpy()).to_scipy()
    Lo = gen.from_scipy(sp.tril(M, k=-1) + sp.identity(C.n, format="csr"))
    Up = gen.from_scipy(sp.triu(M))
    dL, dU = DeviceCSR.from_host(Lo), DeviceCSR.from_host(Up)
    B = torch.from_numpy(gen.normal_rhs(C.n, 2, nrhs=8)).cuda()
    Y = torch.zeros_like(B)
    Z = torch.zeros_like(B)
    # the sweep plan (CTAs, shared-memory budget) picked by the autotuner on short trial runs
    from baas_b200 import autotune

    tuned = autotune.tune(s, lambda: s.forward(dL, B, Y), parts=(96, 128, 148), budgets=(0, 160 * 1024), repeats=2)
    fwd = _event_ms(lambda: s.forward(dL, B, Y), 5, flush)
    bwd = _event_ms(lambda: s.backward(dU, Y, Z), 5, flush)
    nnz_t = Lo.nnz
    nbytes = 12 * nnz_t + 4 * (C.n + 1) + 16 * C.n * 8
    peak, peak_kind = _peaks()
    gb_f, gb_b = nbytes / (fwd * 1e-3) / 1e9, nbytes / (bwd * 1e-3) / 1e9
    out = {"workload": "ilu0_convdiff3d_96_8rhs", "n": C.n, "nnz": C.nnz, "ilu0_ms": round(ilu_ms, 4),
           "forward_8rhs_ms": round(fwd, 4), "backward_8rhs_ms": round(bwd, 4),
           "total_ms": round(ilu_ms + fwd + bwd, 4),
           "sweep_bytes_8rhs": nbytes, "forward_gbps": round(gb_f, 2), "backward_gbps": round(gb_b, 2),
           "roofline": {"bound": "hbm", "achieved": round(gb_f, 2), "peak": peak, "unit": "GB/s",
                        "frac": round(gb_f / peak, 5), "peak_kind": peak_kind,
                        "kernel": "k_sweep_chunked<multi-RHS> (forward, 8 right-hand sides)"},
           "autotuned": tuned["best"]}
    if CPU_BASELINES:
        out["cpu_baseline"] = c3_cpu_baseline(C, Lo, Up, B.cpu().numpy())
    return out


def c3_cpu_baseline(C, Lo, Up, B):
    """The reference on all host cores: ILU0 (ilu0_p2p_csr_group_merge_no_perm_alloc) and, for
    each of the 8 right-hand sides, its p2p forward and backward sweeps (one right-hand side per
    call, as the reference's sweeps take)."""
    from oracle.oracle import Ref, ref_available

    if not ref_available():
        return None
    cores = _host_cores()
    rs = Ref.Schedule(3, C, cores)
    ilu_ms = _ref_ms(lambda: rs.ilu0(C), 2)
    R = B.shape[0]

    def apply():
        for r in range(R):
            rs.backward(Up, rs.forward(Lo, B[r]))

    sw_ms = _ref_ms(apply, 2)
    return {"value": round(ilu_ms + sw_ms, 3), "unit": "ms", "cores": cores, "kind": "reference",
            "ilu0_ms": round(ilu_ms, 3), "forward_backward_8rhs_ms": round(sw_ms, 3),
            "sample": f"the whole configuration (ILU0 + 8 x forward/backward p2p sweeps), mean of 2, nthread={cores}"}


def _analysis_placements(A, s_host, host_ms):
    """The schedule analysis with its data-parallel stages on the device (ANALYSIS_DEVICE) next to
    the all-host analysis: the time of each (the device one after a first, module-loading run) and
    whether every exported array and the group DAG are identical."""
    from baas_b200 import ANALYSIS_DEVICE, KERNEL_ICCG, Schedule
    from baas_b200._native import FIELDS, GROUP_DAG_FIELDS

    Schedule(A, kind=KERNEL_ICCG, nthread=8, analysis=ANALYSIS_DEVICE)
    sd = Schedule(A, kind=KERNEL_ICCG, nthread=8, analysis=ANALYSIS_DEVICE)
    same = all(np.array_equal(s_host.export(f), sd.export(f)) for f in list(FIELDS) + list(GROUP_DAG_FIELDS))
    return {"host_ms": round(host_ms, 2), "device_stages_ms": round(sd.analysis_ms, 2), "identical": bool(same),
            "device_stages": "transposes, two-hop reduction, group DAGs, level sets"}


def c4_batched():
    """64 variable-coefficient 2-D diffusion systems (k ~ U[64, 512]) x 4 right-hand sides, FP32
    IC0 factors, one launch; plan parameters picked by the autotuner on short trial runs."""
    import torch

    from baas_b200 import PREC_FP32_FACTORS, PREC_FP64, BatchSchedule, DeviceCSR, autotune, gen

    systems = gen.batch_vardiff2d()
    t0 = time.time()
    s = BatchSchedule(systems, nthread=8)
    analysis_s = time.time() - t0
    from baas_b200 import ANALYSIS_DEVICE

    t0 = time.time()
    sd = BatchSchedule(systems, nthread=8, analysis=ANALYSIS_DEVICE)
    analysis_dev_s = time.time() - t0
    del sd
    A = s.combined
    dA = DeviceCSR.from_host(A)
    B = torch.from_numpy(gen.uniform_rhs(A.n, 2, nrhs=4).reshape(4, A.n)).cuda()
    X = torch.zeros_like(B)

    def trial():
        X.zero_()
        s.iccg_batched(dA, B, X, tol=TOL, maxiter=30, precision=PREC_FP32_FACTORS, raise_on_nonconvergence=False)

    tuned = autotune.tune(s, trial, parts=(96, 128, 148), budgets=(0, 160 * 1024), repeats=1)

    def full(prec):
        X.zero_()
        return s.iccg_batched(dA, B, X, tol=TOL, maxiter=20000, precision=prec)

    it32, rel32 = full(PREC_FP32_FACTORS)
    ms32 = _event_ms(lambda: full(PREC_FP32_FACTORS), 2)
    x32 = X.clone()
    it64, rel64 = full(PREC_FP64)
    ms64 = _event_ms(lambda: full(PREC_FP64), 1)
    x64 = X.clone()
    off = s.sys_off
    errs = []
    for q in range(len(systems)):
        a, b = int(off[q]), int(off[q + 1])
        d = torch.linalg.norm(x32[:, a:b] - x64[:, a:b], dim=1) / torch.linalg.norm(x64[:, a:b], dim=1)
        errs.append(float(d.max()))
    # algorithmic bytes (the reference's model, test/iccg_level_merge.cpp:509-510) summed over
    # the (system, right-hand side) instances, each for the iterations it ran: SpMV, two FP32-factor
    # sweeps (8 bytes per factor entry) and the vector work, per iteration
    itm = np.asarray(it32).reshape(len(systems), -1) if np.asarray(it32).size == 4 * len(systems) else None
    nbytes = 0
    for q, S in enumerate(systems):
        nnz_l = (S.nnz + S.n) // 2
        per_it = (12 * S.nnz + 4 * (S.n + 1) + 16 * S.n) + 2 * (8 * nnz_l + 4 * (S.n + 1) + 16 * S.n) + 112 * S.n
        iters_q = int(itm[q].sum()) if itm is not None else int(np.max(it32)) * 4
        nbytes += per_it * iters_q
    peak, peak_kind = _peaks()
    gbps = nbytes / (ms32 * 1e-3) / 1e9
    out = {"workload": "batched_vardiff2d_64sys_k64-512_4rhs", "n_total": A.n, "nnz_total": A.nnz,
           "systems": len(systems), "rhs": 4, "ms_fp32_factors": round(ms32, 3), "ms_fp64": round(ms64, 3),
           "iterations_fp32": {"min": int(it32.min()), "median": float(np.median(it32)), "max": int(it32.max())},
           "max_relres": float(rel32.max()), "rel_err_fp32_vs_fp64_gpu_per_system": {"max": max(errs),
                                                                                     "median": float(np.median(errs))},
           "roofline": {"bound": "hbm", "achieved": round(gbps, 2), "peak": peak, "unit": "GB/s",
                        "frac": round(gbps / peak, 5), "peak_kind": peak_kind, "kernel": "k_iccg_batched<float>",
                        "algorithmic_bytes_per_launch": int(nbytes)},
           "autotuned": tuned["best"], "analysis_s": round(analysis_s, 2),
           "analysis_device_stages_s": round(analysis_dev_s, 2)}
    if CPU_BASELINES:
        out["cpu_baseline"] = c4_cpu_baseline(systems, B.cpu().numpy(), x32.cpu().numpy(), x64.cpu().numpy(), off)
    return out


def c4_cpu_baseline(systems, B, x32, x64, off):
    """The reference's ICCG (Scheduler P2P_RULE IC0 + p2p sweeps, pcg_opt loop) on all host cores,
    on a bounded sample: every 8th system (by size) with its first right-hand side; the time is
    scaled to all 64 systems x 4 right-hand sides by the sample's share of the batch's rows. The
    same FP64 solves are the oracle for the GPU's per-system errors (FP32 factors and FP64)."""
    from oracle.oracle import Ref, ref_available

    if not ref_available():
        return None
    cores = _host_cores()
    order = np.argsort([S.n for S in systems])
    pick = [int(q) for q in order[::8]]
    t_ms, e32, e64, rows = 0.0, [], [], 0
    for q in pick:
        S = systems[q]
        a, b = int(off[q]), int(off[q + 1])
        xr, it, rel, t = Ref.pcg(S, B[0, a:b], maxiter=20000, tol=TOL, mode=1, nthread=cores)
        t_ms += float(t[1] + t[2])
        rows += S.n
        e32.append(float(np.linalg.norm(x32[0, a:b] - xr) / np.linalg.norm(xr)))
        e64.append(float(np.linalg.norm(x64[0, a:b] - xr) / np.linalg.norm(xr)))
    total_rows = sum(S.n for S in systems)
    est = t_ms * (total_rows / rows) * B.shape[0]
    return {"value": round(est, 1), "unit": "ms", "cores": cores, "kind": "reference",
            "sample": f"{len(pick)} of 64 systems (every 8th by size), right-hand side 0: {t_ms:.1f} ms of IC0 + PCG "
                      f"to 1e-10 at nthread={cores}, scaled by rows ({total_rows}/{rows}) and by 4 right-hand sides",
            "rel_err_vs_reference_fp64": {"systems": pick, "fp32_factors_max": max(e32),
                                          "fp32_factors_median": float(np.median(e32)), "fp64_max": max(e64)}}


def _iccg_case(name, A, b_h, flush, reps=3):
    """One ICCG configuration: GPU FP64 solve time (L2 flushed, CUDA events), iterations, the walk
    that ran, and beside it the reference's OpenMP solve of the same system (whose solution is the
    FP64 oracle the GPU's is compared with)."""
    import torch

    from baas_b200 import KERNEL_ICCG, PREC_FP32_FACTORS, PREC_FP64, DeviceCSR, Schedule

    s = Schedule(A, kind=KERNEL_ICCG, nthread=8)
    dA = DeviceCSR.from_host(A)
    b = torch.from_numpy(b_h).cuda()
    x = torch.zeros_like(b)

    def solve(prec):
        x.zero_()
        return s.iccg(dA, b, x, tol=TOL, maxiter=MAXITER, precision=prec)

    it, rel = solve(PREC_FP64)
    ms = _event_ms(lambda: solve(PREC_FP64), reps, flush)
    x64 = x.cpu().numpy()
    it32, _ = solve(PREC_FP32_FACTORS)
    ms32 = _event_ms(lambda: solve(PREC_FP32_FACTORS), reps, flush)
    x32 = x.cpu().numpy()
    out = {"workload": name, "n": A.n, "nnz": A.nnz, "ms_fp64": round(ms, 4), "iterations": int(it), "relres": rel,
           "ms_fp32_factors": round(ms32, 4), "iterations_fp32": int(it32), "walk": s.last_walk,
           "partition": list(s.plan_parts()[1]) if s.plan_parts()[1] else f"ranges x{s.plan_parts()[0]}",
           "analysis_ms": round(s.analysis_ms, 2)}
    if CPU_BASELINES:
        from oracle.oracle import Ref, ref_available

        if ref_available():
            cores = _host_cores()
            xr, itr, relr, t = Ref.pcg(A, b_h, maxiter=MAXITER, tol=TOL, mode=1, nthread=cores)
            out["cpu_baseline"] = {
                "value": round(float(t[1] + t[2]), 3), "unit": "ms", "cores": cores, "kind": "reference",
                "iterations": int(itr),
                "sample": f"1 full solve (IC0 + PCG to 1e-10), Scheduler P2P_RULE at nthread={cores}",
                "rel_err_vs_reference_fp64": {
                    "fp64": float(np.linalg.norm(x64 - xr) / np.linalg.norm(xr)),
                    "fp32_factors": float(np.linalg.norm(x32 - xr) / np.linalg.norm(xr))}}
    return out


def c2_variants(flush):
    """Configuration 2's other inputs: the 64^3 system under the seeded random symmetric
    permutation, and the k-NN (k = 12) 3-dof stiffness-like SPD matrix (n = 12,000)."""
    from baas_b200 import gen

    out = {}
    P = gen.c2_system(permuted=True)
    out["c2_permuted"] = _iccg_case("iccg_laplace3d_64_shift1e-3_permuted", P, gen.uniform_rhs(P.n, 1), flush)
    K = gen.knn_stiffness(nodes=4000, k=12, seed=3)
    out["c2_knn"] = _iccg_case("iccg_knn_stiffness_4000_nodes_k12", K, gen.uniform_rhs(K.n, 1), flush)
    out["c2_knn"]["walk_table"] = _walk_table(K, gen.uniform_rhs(K.n, 1))
    return out


def _walk_table(A, b_h):
    """The same FP64 ICCG under every sweep walk and cluster size (autotune.tune_walk): best of
    three CUDA-event timings after a warm-up, per candidate."""
    import torch

    from baas_b200 import KERNEL_ICCG, DeviceCSR, Schedule, autotune

    s = Schedule(A, kind=KERNEL_ICCG, nthread=8)
    dA = DeviceCSR.from_host(A)
    b = torch.from_numpy(b_h).cuda()
    x = torch.zeros_like(b)

    def run():
        x.zero_()
        s.iccg(dA, b, x, tol=TOL, maxiter=MAXITER)

    names = {1: "chunked", 2: "fetch", 3: "levels", 4: "cluster"}
    table = autotune.tune_walk(s, run, repeats=3)["table"]
    return [{"walk": names[r["walk"]], "ctas": r["small_cluster"] or None, "ms": r["ms"]} for r in table]


def c5_adjoint():
    """Differentiated ICCG on 64^3 variable-coefficient diffusion (face kappa = exp(theta), sigma
    0.5), FP64 CG with FP32 IC0 factors: loss 1/2 ||x - x_obs||^2, gradients w.r.t. theta and b by
    the adjoint kernel, checked against central differences (h = 1e-6) along 32 random directions;
    beside it the 16^3 gradient against an FP64 CPU gradient built on the reference's own PCG."""
    import torch

    from baas_b200 import PREC_FP32_FACTORS, gen
    from baas_b200.autograd import DiffIccg, FaceDiffusion3D, face_shapes

    def theta_of(k, seed, sigma=0.5):
        return np.concatenate([gen.gaussian_field(shp, sigma, 4.0, seed + j).ravel()
                               for j, shp in enumerate(face_shapes(k))])

    def problem(k, tol):
        op = FaceDiffusion3D(k)
        solver = DiffIccg(op, tol=tol, maxiter=20000, precision=PREC_FP32_FACTORS)
        theta = torch.from_numpy(theta_of(k, 11)).cuda()
        b = torch.from_numpy(gen.uniform_rhs(op.n, 4)).cuda()
        with torch.no_grad():
            xp = solver.solve(theta + torch.from_numpy(theta_of(k, 23, 0.1)).cuda(), b)
        x_obs = xp + torch.from_numpy(np.random.default_rng(5).normal(0.0, 1e-3, op.n)).cuda()
        return op, solver, theta, b, x_obs

    def grads(solver, theta, b, x_obs):
        th = theta.clone().requires_grad_(True)
        bb = b.clone().requires_grad_(True)
        x = solver.solve(th, bb)
        (0.5 * ((x - x_obs) ** 2).sum()).backward()
        return th.grad.detach(), bb.grad.detach()

    op, solver, theta, b, x_obs = problem(64, 1e-14)
    gth, gb = grads(solver, theta, b, x_obs)  # warm-up
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    gth, gb = grads(solver, theta, b, x_obs)
    e1.record()
    e1.synchronize()
    grad_ms = e0.elapsed_time(e1)
    rng = np.random.default_rng(7)
    h = 1e-6
    ad, fd = [], []
    with torch.no_grad():
        x0 = solver.solve(theta, b)

        def perturbed(sign, vt, vb):
            x = x0.clone()
            vals = op.values(torch.exp(theta + sign * h * vt))
            solver.sched.iccg(op.device_csr(vals), b + sign * h * vb, x, tol=1e-12, maxiter=20000,
                              precision=PREC_FP32_FACTORS)
            return x

        for _ in range(32):
            vt = torch.from_numpy(rng.standard_normal(theta.numel())).cuda()
            vb = torch.from_numpy(rng.standard_normal(b.numel())).cuda()
            vt /= vt.norm()
            vb /= vb.norm()
            xp, xm = perturbed(1.0, vt, vb), perturbed(-1.0, vt, vb)
            fd.append(float(0.5 * ((xp - xm) * (xp + xm - 2.0 * x_obs)).sum() / (2 * h)))
            ad.append(float((gth * vt).sum() + (gb * vb).sum()))
    ad, fd = np.array(ad), np.array(fd)
    out = {"workload": "adjoint_iccg_vardiff3d_64_fp32_factors", "n": op.n,
           "forward_plus_adjoint_ms": round(grad_ms, 3),
           "fd_rel_err_32_directions": float(np.linalg.norm(ad - fd) / np.linalg.norm(ad)), "fd_h": h}
    if CPU_BASELINES:
        out["cpu_baseline"] = c5_cpu_gradient(problem, grads)
    return out


def c5_cpu_gradient(problem, grads):
    """FP64 CPU gradient at 16^3: forward and adjoint solves with the reference's PCG (pcg_opt
    structure, Scheduler P2P_RULE), then dL/dtheta_f = -kappa_f (lam_p - lam_q)(x_p - x_q) for each
    interior face and dL/db = lam; compared with the GPU adjoint's gradients."""
    import torch

    from baas_b200 import gen
    from oracle.oracle import Ref, ref_available

    if not ref_available():
        return None
    cores = _host_cores()
    op, solver, theta, b, x_obs = problem(16, 1e-12)
    gth, gb = grads(solver, theta, b, x_obs)
    kappa = np.exp(theta.cpu().numpy())
    A = gen.CSR(op.n, op.pattern.rowptr, op.pattern.colidx, op.values(torch.from_numpy(kappa).cuda()).cpu().numpy())
    t0 = time.perf_counter()
    x, _, _, _ = Ref.pcg(A, b.cpu().numpy(), maxiter=20000, tol=1e-14, mode=1, nthread=cores)
    lam, _, _, _ = Ref.pcg(A, x - x_obs.cpu().numpy(), maxiter=20000, tol=1e-14, mode=1, nthread=cores)
    rows = np.repeat(np.arange(op.n), np.diff(A.rowptr))
    p, q = rows[op.pq], A.colidx[op.pq]
    gth_ref = -kappa * (lam[p] - lam[q]) * (x[p] - x[q])
    cpu_ms = (time.perf_counter() - t0) * 1e3
    return {"value": round(cpu_ms, 3), "unit": "ms", "cores": cores, "kind": "reference",
            "sample": "16^3 forward + adjoint FP64 solves (reference PCG) and the face-gradient formula",
            "grad_theta_rel_err": float(np.linalg.norm(gth.cpu().numpy() - gth_ref) / np.linalg.norm(gth_ref)),
            "grad_b_rel_err": float(np.linalg.norm(gb.cpu().numpy() - lam) / np.linalg.norm(lam))}


def c4_sharded(rank, world, dev):
    """Configuration 4 split across the ranks by whole systems (baas_b200.distributed): each rank
    solves its share in one batched launch, with no communication during the solve, then one
    gather of every system's iterations, residuals and solution to rank 0. The time is the max
    over ranks of their launch times (CUDA events); total work is fixed, so the scaling is strong."""
    from baas_b200 import PREC_FP32_FACTORS, gen
    from baas_b200.distributed import batched_solve, solve_sharded

    systems = gen.batch_vardiff2d()
    rhs = lambda q: gen.uniform_rhs(systems[q].n, 1000 + q, nrhs=4)  # noqa: E731
    got = solve_sharded(systems, lambda idx: batched_solve(systems, idx, rhs, device=dev, tol=TOL,
                                                           precision=PREC_FP32_FACTORS), rank, world)
    if got is None:
        return None
    times = got.pop(-1)
    it = np.array([got[q]["iterations"] for q in range(len(systems))])
    rel = np.array([got[q]["relres"] for q in range(len(systems))])
    return {"workload": "batched_vardiff2d_64sys_k64-512_4rhs_sharded", "ranks": world, "scaling": "strong",
            "ms_fp32_factors": round(max(times.values()), 3),
            "ms_per_rank": {int(r): round(t, 3) for r, t in sorted(times.items())},
            "iterations": {"min": int(it.min()), "max": int(it.max())}, "max_relres": float(rel.max())}


def gpu_arm(args):
    import torch

    world, rank, local = _dist()
    if world > 1:
        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    dev = torch.device("cuda", local if world > 1 else 0)
    torch.cuda.set_device(dev)
    from baas_b200 import KERNEL_ICCG, PREC_FP32_FACTORS, PREC_FP64, DeviceCSR, Schedule, gen

    A = gen.laplace3d(K_GRID, 1e-3)
    b_h = gen.uniform_rhs(A.n, 1)
    s = Schedule(A, kind=KERNEL_ICCG, nthread=8)
    analysis_ms = s.analysis_ms
    analysis = _analysis_placements(A, s, analysis_ms) if rank == 0 else None
    dA = DeviceCSR.from_host(A, device=dev)
    b = torch.from_numpy(b_h).to(dev)
    x = torch.zeros_like(b)
    stream = torch.cuda.current_stream(dev)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)  # 256 MB > L2

    def solve(prec):
        x.zero_()
        return s.iccg(dA, b, x, tol=TOL, maxiter=MAXITER, precision=prec)

    for _ in range(max(args.warmup, 3)):
        solve(PREC_FP64)
    it, rel = solve(PREC_FP64)

    def timed(prec, steps):
        ts = []
        for _ in range(steps):
            flush.fill_(1.0)
            x.zero_()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            s.iccg(dA, b, x, tol=TOL, maxiter=MAXITER, precision=prec)
            e1.record(stream)
            e1.synchronize()
            ts.append(e0.elapsed_time(e1))
        return ts

    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    with ClockSampler(dev.index) as clk:
        t0 = time.time()
        ts64 = timed(PREC_FP64, args.steps)
        wall = time.time() - t0
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    ms64 = float(np.mean(ts64))

    # FP32-factor form (same solve, factors stored and applied in FP32)
    solve(PREC_FP32_FACTORS)
    it32, rel32 = solve(PREC_FP32_FACTORS)
    ts32 = timed(PREC_FP32_FACTORS, max(3, args.steps // 2))
    ms32 = float(np.mean(ts32))
    err32 = 0.0
    x64 = torch.zeros_like(b)
    s.iccg(dA, b, x64, tol=TOL, maxiter=MAXITER, precision=PREC_FP64)
    x32 = torch.zeros_like(b)
    s.iccg(dA, b, x32, tol=TOL, maxiter=MAXITER, precision=PREC_FP32_FACTORS)
    err32 = float(torch.linalg.norm(x32 - x64) / torch.linalg.norm(x64))

    # standalone forward sweep of the IC0 factor (SpTRSV GB/s)
    lu = dA.values.clone()
    s.ic0(dA, lu)
    lo = gen.CSR(A.n, A.rowptr, A.colidx, lu.cpu().numpy()).lower()
    dL = DeviceCSR.from_host(lo, device=dev)
    y = torch.zeros_like(b)
    for _ in range(3):
        s.forward(dL, b, y)
    sw = []
    for _ in range(10):
        flush.fill_(1.0)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        s.forward(dL, b, y)
        e1.record(stream)
        e1.synchronize()
        sw.append(e0.elapsed_time(e1))
    sweep_ms = float(np.min(sw))

    # e2e through the public API with pinned host buffers
    vals_h = torch.from_numpy(A.values).pin_memory()
    b_pin = torch.from_numpy(b_h).pin_memory()
    x_pin = torch.zeros(A.n, dtype=torch.float64).pin_memory()
    x0_pin = torch.zeros(A.n, dtype=torch.float64).pin_memory()
    ee = []
    for _ in range(max(3, args.steps // 2)):
        flush.fill_(1.0)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        dA.values.copy_(vals_h, non_blocking=True)
        b.copy_(b_pin, non_blocking=True)
        x.copy_(x0_pin, non_blocking=True)
        s.iccg(dA, b, x, tol=TOL, maxiter=MAXITER, precision=PREC_FP64)
        x_pin.copy_(x, non_blocking=True)
        e1.record(stream)
        e1.synchronize()
        ee.append(e0.elapsed_time(e1))
    e2e_ms = float(np.mean(ee))

    # the other configurations (1 GPU only: replicas would repeat them)
    extras = {}
    if world == 1 and not args.headline_only:
        for name, fn in (("sptrsv_c1", lambda: c1_sptrsv(flush)), ("c2_variants", lambda: c2_variants(flush)),
                         ("ilu0_c3", lambda: c3_ilu(flush)), ("batched_c4", c4_batched), ("adjoint_c5", c5_adjoint)):
            try:
                r = fn()
                if name == "c2_variants":
                    extras.update(r)
                else:
                    extras[name] = r
            except Exception as e:  # a failure here must not cost the headline line
                extras[name] = {"error": f"{type(e).__name__}: {str(e)[:160]}"}

    if world > 1 and not args.headline_only:
        # the configuration that shards: the batch split by whole systems (every rank takes part)
        try:
            r = c4_sharded(rank, world, dev)
            if r is not None:
                extras["batched_c4_sharded"] = r
        except Exception as e:
            extras["batched_c4_sharded"] = {"error": f"{type(e).__name__}: {str(e)[:160]}"}

    vals = torch.tensor([ms64, e2e_ms, ms32], dtype=torch.float64, device=dev)
    if world > 1:
        torch.distributed.all_reduce(vals, op=torch.distributed.ReduceOp.MAX)
    ms64, e2e_ms, ms32 = [float(v) for v in vals.cpu()]

    peak, peak_kind = _peaks()
    launch_bytes = IC0_BYTES + it * ITER_BYTES
    # latency bounds: one sweep; the ICCG launch = two sweeps per preconditioner apply (it + 1
    # applies) plus the IC0 walk, each at the sweep bound
    sweep_lat = sweep_latency_bound(s)
    sweep_lat["frac"] = round(sweep_lat["bound_us"] / (sweep_ms * 1e3), 4)
    iccg_bound_ms = (2 * (it + 1) + 1) * sweep_lat["bound_us"] * 1e-3
    iccg_lat = {"bound_ms": round(iccg_bound_ms, 3), "sweeps": 2 * (it + 1) + 1, "per_sweep_us": sweep_lat["bound_us"],
                "frac": round(iccg_bound_ms / ms64, 4)}
    achieved = launch_bytes / (ms64 * 1e-3) / 1e9
    # DRAM bytes of one launch, from the ncu capture summarised in profiles/
    traffic = None
    tp = ROOT / "profiles" / "k_iccg_fetch_laplace3d_64.md"
    if tp.exists():
        for line in tp.read_text().splitlines():
            if line.startswith("traffic_bytes_per_launch:"):
                traffic = int(line.split(":")[1])
    if rank == 0:
        cpu, xref = None, None
        if world == 1 and not args.no_cpu_baseline:
            got = cpu_baseline_sample()
            if got is not None:
                cpu, xref = got
                # the reference's FP64 solution is the oracle for both GPU forms' errors
                cpu["rel_err_vs_reference_fp64"] = {
                    "fp64": float(np.linalg.norm(x64.cpu().numpy() - xref) / np.linalg.norm(xref)),
                    "fp32_factors": float(np.linalg.norm(x32.cpu().numpy() - xref) / np.linalg.norm(xref))}
        clocks = clk.summary()
        line = {
            "metric": METRIC, "value": round(ms64, 4), "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": max(args.warmup, 3), "ms_per_step": round(ms64, 4), "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "iccg_laplace3d_64_shift1e-3", "n": A.n, "nnz": A.nnz, "tol": TOL,
                       "iterations": int(it), "relres": rel, "parallelism": f"replicas{world}",
                       "l2": "flushed (256 MB write) before every timed step"},
            "e2e": {"value": round(e2e_ms, 4), "unit": UNIT,
                    "h2d_bytes_per_step": int(A.values.nbytes + b_h.nbytes + 8 * A.n),
                    "d2h_bytes_per_step": int(8 * A.n)},
            "gpu_launches": int(args.steps),
            "roofline": {"bound": "hbm", "achieved": round(achieved, 2), "peak": peak, "unit": "GB/s",
                         "frac": round(achieved / peak, 5), "traffic": traffic,
                         "peak_kind": peak_kind, "kernel": "k_iccg_chunked<double, fetch walk>",
                         "algorithmic_bytes_per_launch": int(launch_bytes),
                         "latency_bound": iccg_lat},
            "cpu_baseline": cpu,
            "clocks": clocks,
            "fp32_factors": {"ms": round(ms32, 4), "iterations": int(it32), "relres": rel32,
                             "rel_err_vs_fp64": err32},
            "sptrsv": {"ms": round(sweep_ms, 4), "bytes": SWEEP_BYTES,
                       "gbps": round(SWEEP_BYTES / (sweep_ms * 1e-3) / 1e9, 2),
                       "hbm_frac": round(SWEEP_BYTES / (sweep_ms * 1e-3) / 1e9 / peak, 5),
                       "latency_bound": sweep_lat},
            "analysis_ms": round(analysis_ms, 2),
            "analysis": analysis,
            "configs": extras,
            "wall_s_timed_region": round(wall, 3),
        }
        print(json.dumps(line))
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()


def profile_case(args):
    """One kernel of the bench workload, `--warmup` untimed then `--steps` timed launches, for
    ncu captures (`-k` on the kernel name). Prints one JSON line with the mean launch time."""
    import torch

    from baas_b200 import KERNEL_ICCG, PREC_FP32_FACTORS, PREC_FP64, DeviceCSR, Schedule, gen

    A = gen.laplace3d(K_GRID, 1e-3)
    s = Schedule(A, kind=KERNEL_ICCG, nthread=8)
    dA = DeviceCSR.from_host(A)
    b = torch.from_numpy(gen.uniform_rhs(A.n, 1)).cuda()
    x = torch.zeros_like(b)
    case = args.profile_case
    if case in ("sweep_lower", "sweep_upper"):
        lu = dA.values.clone()
        s.ic0(dA, lu)
        lo = gen.CSR(A.n, A.rowptr, A.colidx, lu.cpu().numpy()).lower()
        dT = DeviceCSR.from_host(lo if case == "sweep_lower" else lo.transpose())
        run = (lambda: s.forward(dT, b, x)) if case == "sweep_lower" else (lambda: s.backward(dT, b, x))
    elif case == "batched_small":
        from baas_b200 import BatchSchedule

        sb = BatchSchedule(gen.batch_vardiff2d(nsys=8, kmin=64, kmax=128), nthread=8)
        dB = DeviceCSR.from_host(sb.combined)
        Bb = torch.from_numpy(gen.uniform_rhs(sb.n, 2, nrhs=4).reshape(4, sb.n)).cuda()
        Xb = torch.zeros_like(Bb)
        run = lambda: (Xb.zero_(), sb.iccg_batched(dB, Bb, Xb, tol=TOL, maxiter=20000,  # noqa: E731
                                                    precision=PREC_FP32_FACTORS))
    elif case == "knn_iccg":
        # the k-NN stiffness matrix (n = 12,000): the cluster walk the library picks for it
        K = gen.knn_stiffness(nodes=4000)
        sk = Schedule(K, kind=KERNEL_ICCG, nthread=8)
        dK = DeviceCSR.from_host(K)
        bk = torch.from_numpy(gen.uniform_rhs(K.n, gen.C2_RHS_SEED)).cuda()
        xk = torch.zeros_like(bk)
        run = lambda: (xk.zero_(), sk.iccg(dK, bk, xk, tol=TOL, maxiter=MAXITER, precision=PREC_FP64))  # noqa: E731
    elif case == "ic0":
        lu = dA.values.clone()
        run = lambda: (lu.copy_(dA.values), s.ic0(dA, lu))  # noqa: E731
    else:
        prec = PREC_FP32_FACTORS if case == "iccg_fp32" else PREC_FP64
        run = lambda: (x.zero_(), s.iccg(dA, b, x, tol=TOL, maxiter=MAXITER, precision=prec))  # noqa: E731
    for _ in range(args.warmup):
        run()
    ts = []
    for _ in range(args.steps):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        run()
        e1.record()
        e1.synchronize()
        ts.append(e0.elapsed_time(e1))
    print(json.dumps({"profile_case": case, "ms_mean": round(float(np.mean(ts)), 4), "launches": args.steps}))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="baas_b200", choices=["baas_b200", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--headline-only", action="store_true", help="skip the other configurations")
    ap.add_argument("--profile-case", default=None,
                    choices=["iccg", "iccg_fp32", "ic0", "sweep_lower", "sweep_upper", "batched_small", "knn_iccg"],
                    help="run one kernel of the workload only (for ncu captures)")
    args = ap.parse_args()
    global CPU_BASELINES
    CPU_BASELINES = not args.no_cpu_baseline
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        # one process per GPU: relaunch this command under torchrun (rendezvous on 127.0.0.1)
        cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={args.gpus}",
               "--master-addr", "127.0.0.1", "--master-port", os.environ.get("BAAS_BENCH_PORT", "29531"),
               str(Path(__file__).resolve())] + sys.argv[1:]
        raise SystemExit(subprocess.call(cmd))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if args.gpus != world and args.impl != "reference":
        raise SystemExit(f"--gpus {args.gpus} but WORLD_SIZE={world}")
    if args.impl == "reference":
        reference_arm(args)
    elif args.profile_case:
        profile_case(args)
    else:
        gpu_arm(args)


if __name__ == "__main__":
    main()
