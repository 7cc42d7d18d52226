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
    times, iters, pre = [], 0, []
    for _ in range(args.steps):
        x, iters, rel, t = Ref.pcg(A, b, maxiter=MAXITER, tol=TOL, mode=1, nthread=cores)
        times.append(t[1] + t[2])  # IC0 + PCG loop (analysis excluded, as on the GPU arm)
        pre.append(t[0])
    v = float(np.mean(times))
    line = {
        "impl": "reference", "metric": METRIC, "value": round(v, 3), "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(v, 3), "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "iccg_laplace3d_64_shift1e-3", "n": A.n, "nnz": A.nnz, "tol": TOL,
                   "iterations": int(iters), "l2": "host CPU run"},
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
    _, it, _, t = Ref.pcg(A, b, maxiter=MAXITER, tol=TOL, mode=1, nthread=cores)
    return {"value": round(float(t[1] + t[2]), 3), "unit": UNIT, "cores": cores, "kind": "reference",
            "sample": f"1 full solve (IC0 + {it} PCG iterations to 1e-10) with the reference's OpenMP "
                      f"Scheduler P2P_RULE path, nthread={cores}; analysis {t[0]:.1f} ms excluded"}


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
    err = float(np.max(np.abs(x.cpu().numpy() - x_true)))
    return {"workload": "sptrsv_laplace2d_128_lower", "ms": round(ms, 4), "bytes": nbytes,
            "gbps": round(nbytes / (ms * 1e-3) / 1e9, 2), "max_abs_err_vs_x_true": err}


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
    fwd = _event_ms(lambda: s.forward(dL, B, Y), 5, flush)
    bwd = _event_ms(lambda: s.backward(dU, Y, Z), 5, flush)
    nnz_t = Lo.nnz
    nbytes = 12 * nnz_t + 4 * (C.n + 1) + 16 * C.n * 8
    return {"workload": "ilu0_convdiff3d_96_8rhs", "n": C.n, "nnz": C.nnz, "ilu0_ms": round(ilu_ms, 4),
            "forward_8rhs_ms": round(fwd, 4), "backward_8rhs_ms": round(bwd, 4),
            "sweep_bytes_8rhs": nbytes, "forward_gbps": round(nbytes / (fwd * 1e-3) / 1e9, 2),
            "backward_gbps": round(nbytes / (bwd * 1e-3) / 1e9, 2)}


def c4_batched():
    """64 variable-coefficient 2-D diffusion systems (k ~ U[64, 512]) x 4 right-hand sides, FP32
    IC0 factors, one launch; plan parameters picked by the autotuner on short trial runs."""
    import torch

    from baas_b200 import PREC_FP32_FACTORS, PREC_FP64, BatchSchedule, DeviceCSR, autotune, gen

    t0 = time.time()
    systems = gen.batch_vardiff2d()
    s = BatchSchedule(systems, nthread=8)
    analysis_s = time.time() - t0
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
    return {"workload": "batched_vardiff2d_64sys_k64-512_4rhs", "n_total": A.n, "nnz_total": A.nnz,
            "systems": len(systems), "rhs": 4, "ms_fp32_factors": round(ms32, 3), "ms_fp64": round(ms64, 3),
            "iterations_fp32": {"min": int(it32.min()), "median": float(np.median(it32)), "max": int(it32.max())},
            "max_relres": float(rel32.max()), "rel_err_vs_fp64_per_system": {"max": max(errs),
                                                                              "median": float(np.median(errs))},
            "autotuned": tuned["best"], "analysis_s": round(analysis_s, 2)}


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
        for name, fn in (("sptrsv_c1", lambda: c1_sptrsv(flush)), ("ilu0_c3", lambda: c3_ilu(flush)),
                         ("batched_c4", c4_batched)):
            try:
                extras[name] = fn()
            except Exception as e:  # a failure here must not cost the headline line
                extras[name] = {"error": f"{type(e).__name__}: {str(e)[:160]}"}

    vals = torch.tensor([ms64, e2e_ms, ms32], dtype=torch.float64, device=dev)
    if world > 1:
        torch.distributed.all_reduce(vals, op=torch.distributed.ReduceOp.MAX)
    ms64, e2e_ms, ms32 = [float(v) for v in vals.cpu()]

    peak, peak_kind = _peaks()
    launch_bytes = IC0_BYTES + it * ITER_BYTES
    achieved = launch_bytes / (ms64 * 1e-3) / 1e9
    # DRAM bytes of one launch, from the ncu capture summarised in profiles/
    traffic = None
    tp = ROOT / "profiles" / "k_iccg_chunked_laplace3d_64.md"
    if tp.exists():
        for line in tp.read_text().splitlines():
            if line.startswith("traffic_bytes_per_launch:"):
                traffic = int(line.split(":")[1])
    if rank == 0:
        cpu = None
        if world == 1 and not args.no_cpu_baseline:
            cpu = cpu_baseline_sample()
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
                         "peak_kind": peak_kind, "kernel": "k_iccg_chunked<double>",
                         "algorithmic_bytes_per_launch": int(launch_bytes)},
            "cpu_baseline": cpu,
            "clocks": clocks,
            "fp32_factors": {"ms": round(ms32, 4), "iterations": int(it32), "relres": rel32,
                             "rel_err_vs_fp64": err32},
            "sptrsv": {"ms": round(sweep_ms, 4), "bytes": SWEEP_BYTES,
                       "gbps": round(SWEEP_BYTES / (sweep_ms * 1e-3) / 1e9, 2)},
            "analysis_ms": round(analysis_ms, 2),
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
                    choices=["iccg", "iccg_fp32", "ic0", "sweep_lower", "sweep_upper", "batched_small"],
                    help="run one kernel of the workload only (for ncu captures)")
    args = ap.parse_args()
    if args.impl == "reference":
        reference_arm(args)
    elif args.profile_case:
        profile_case(args)
    else:
        gpu_arm(args)


if __name__ == "__main__":
    main()
