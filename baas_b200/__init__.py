"""B200-native BAAS sparse hot path: Python binding over the C ABI (include/baas_b200.h).

The compute runs in ``baas_b200/_lib/libbaas_b200.so`` (hand-written sm_100a kernels). This
module only marshals arrays: host numpy arrays for the analysis, torch CUDA tensors for the
device calls. There is no CPU fallback -- every compute call goes to the CUDA library and raises
if it is missing or fails.

Names follow the reference's runtime surface (test/Schedule.hpp:39-178): a :class:`Schedule`
is built once from a matrix pattern (``Scheduler::preprocessing``) and then drives
``ic0`` / ``ilu0`` (``runIC0``), ``forward`` / ``backward`` (``runForwardTRSVNoPerm`` /
``runBackwardTRSVNoPerm``) and ``iccg`` (the ``pcg_opt`` loop).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _native
from ._native import (KERNEL_IC0, KERNEL_ICCG, KERNEL_ILU0, KERNEL_SPTRSV, MAPPING_COST_SPLIT,
                      MAPPING_AFFINITY, MAPPING_COST_SPLIT_BARRIER, MAPPING_FINISH_TIME, MAPPING_FOUR_RULE, PARTITION_BAAS_THREADS, PARTITION_CUSTOM,
                      PARTITION_RANGES, PARTITION_BLOCKS, PARTITION_AUTO, WALK_AUTO, WALK_CHUNKED, WALK_FETCH, WALK_LEVELS, WALK_SMALL,
                      ANALYSIS_HOST, ANALYSIS_DEVICE, ABLATION_NONE, ABLATION_WOS, ABLATION_WOA, ABLATION_WOAS,
                      PREC_FP32_FACTORS, PREC_FP64, BaasError)
from .gen import CSR

__all__ = ["Schedule", "BatchSchedule", "batch_concat", "DeviceCSR", "BaasError", "CSR", "KERNEL_SPTRSV",
           "KERNEL_ICCG", "KERNEL_IC0", "KERNEL_ILU0", "PREC_FP64", "PREC_FP32_FACTORS", "PARTITION_RANGES",
           "PARTITION_BAAS_THREADS", "PARTITION_CUSTOM", "MAPPING_FOUR_RULE", "MAPPING_COST_SPLIT",
           "MAPPING_COST_SPLIT_BARRIER", "MAPPING_FINISH_TIME", "MAPPING_AFFINITY", "WALK_AUTO", "WALK_CHUNKED",
           "WALK_FETCH", "WALK_LEVELS", "WALK_SMALL", "PARTITION_BLOCKS", "PARTITION_AUTO", "ANALYSIS_HOST", "ANALYSIS_DEVICE",
           "ABLATION_NONE", "ABLATION_WOS", "ABLATION_WOA", "ABLATION_WOAS", "version"]


def version() -> str:
    return _native.lib().baas_version().decode()


def _ptr(a) -> int:
    """Address of a numpy array or a torch tensor."""
    if isinstance(a, np.ndarray):
        return a.ctypes.data
    return a.data_ptr()


def _stream_ptr(stream) -> int | None:
    if stream is None:
        import torch

        return torch.cuda.current_stream().cuda_stream
    return getattr(stream, "cuda_stream", stream)


@dataclass
class DeviceCSR:
    """A CSR matrix resident on the GPU (torch tensors)."""
    n: int
    rowptr: "object"
    colidx: "object"
    values: "object"

    @property
    def nnz(self) -> int:
        return int(self.colidx.numel())

    @staticmethod
    def from_host(m: CSR, device="cuda") -> "DeviceCSR":
        import torch

        return DeviceCSR(m.n, torch.from_numpy(m.rowptr).to(device), torch.from_numpy(m.colidx).to(device),
                         torch.from_numpy(m.values).to(device))

    def c(self) -> _native.BaasCsr:
        return _native.BaasCsr(self.n, self.nnz, _ptr(self.rowptr), _ptr(self.colidx), _ptr(self.values))


class Schedule:
    """BAAS schedule + device plan for one sparsity pattern.

    kind: KERNEL_SPTRSV (input is the lower triangle L), KERNEL_ICCG (full SPD A, as
    ``Scheduler(A, true, false, P2P_RULE, nthread)``), KERNEL_IC0, KERNEL_ILU0.
    """

    def __init__(self, A: CSR, kind: int = KERNEL_ICCG, nthread: int = 8, spin_limit: int = 0,
                 parts: int = 0, partition: int = PARTITION_AUTO, smem_budget: int = 0, mapping: int = 0,
                 walk: int = 0, analysis: int = ANALYSIS_HOST, ablation: int = ABLATION_NONE,
                 small_cluster: int = 0, scoring: dict | None = None):
        L = _native.lib()
        self._rowptr = np.ascontiguousarray(A.rowptr, dtype=np.int32)
        self._colidx = np.ascontiguousarray(A.colidx, dtype=np.int32)
        c = _native.BaasCsr(A.n, int(self._rowptr[-1]), _ptr(self._rowptr), _ptr(self._colidx), None)
        opt = _native.BaasOptions()
        L.baas_options_default(C.byref(opt))
        opt.nthread = nthread
        opt.spin_limit = spin_limit
        opt.parts = parts
        opt.partition = partition
        opt.smem_budget = smem_budget
        opt.mapping = mapping
        opt.walk = walk
        opt.analysis = analysis
        opt.ablation = ablation
        opt.small_cluster = small_cluster
        # the four-rule mapping's scoring constants (level_window, amplify, over_gamma,
        # award_alpha, load_beta); unnamed ones keep the reference's values
        for key, val in (scoring or {}).items():
            if key not in ("level_window", "amplify", "over_gamma", "award_alpha", "load_beta"):
                raise KeyError(key)
            setattr(opt, key, val)
        h = C.c_void_p()
        _native.check(L.baas_analyze(C.byref(c), kind, C.byref(opt), C.byref(h)), "baas_analyze")
        self._h = h
        self.n = A.n
        self.nnz = int(self._rowptr[-1])
        self.kind = kind
        self.nthread = nthread
        self.mapping = mapping

    def save(self, path) -> None:
        """Write the analysed schedule to `path` (baas_schedule_save): a later `Schedule.load`
        skips the analysis."""
        _native.check(_native.lib().baas_schedule_save(self._h, str(path).encode()), "baas_schedule_save")

    @classmethod
    def load(cls, path) -> "Schedule":
        """A schedule read from a file written by `save` (baas_schedule_load), ready for GPU calls."""
        h = C.c_void_p()
        _native.check(_native.lib().baas_schedule_load(str(path).encode(), C.byref(h)), "baas_schedule_load")
        s = cls.__new__(cls)
        s._h = h
        info = np.zeros(6, dtype=np.int32)
        _native.lib().baas_schedule_info(h, info.ctypes.data)
        s.n, s.nnz, s.kind, s.nthread, s.mapping = (int(v) for v in info[:5])
        return s

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                _native.lib().baas_destroy(h)
            except Exception:
                pass
            self._h = None

    # ---- schedule export (host only) ----
    def export(self, field: str) -> np.ndarray:
        L = _native.lib()
        fid = _native.FIELDS[field] if field in _native.FIELDS else _native.GROUP_DAG_FIELDS[field]
        n = L.baas_schedule_export(self._h, fid, None)
        if n < 0:
            raise KeyError(field)
        out = np.zeros(max(n, 1), dtype=np.int32)
        L.baas_schedule_export(self._h, fid, out.ctypes.data)
        return out[:n]

    def arrays(self) -> dict:
        return {k: self.export(k) for k in _native.FIELDS}

    def plan_parts(self):
        """(CTAs of the current device plan, grid box shape, boxes per axis); shapes are None
        unless the plan uses grid boxes, and the count is 0 before a plan exists."""
        box = np.zeros(6, dtype=np.int32)
        P = int(_native.lib().baas_plan_parts(self._h, box.ctypes.data))
        if box[0] == 0:
            return P, None, None
        return P, tuple(int(v) for v in box[:3]), tuple(int(v) for v in box[3:])

    @property
    def last_walk(self) -> int:
        """WALK_CHUNKED or WALK_FETCH: the sweep kernel of the last sweep / ICCG call (0 before)."""
        return int(_native.lib().baas_schedule_last_walk(self._h))

    def inject_unsatisfiable_wait(self, row: int) -> None:
        """Test hook: the next forward sweep waits on a value nothing writes (BAAS_ERR_TIMEOUT)."""
        _native.check(_native.lib().baas_test_inject_unsatisfiable_wait(self._h, row), "inject")

    def replan(self, parts: int = 0, smem_budget: int = 0, partition: int = PARTITION_AUTO, spin_limit: int = 0,
               walk: int = 0, small_cluster: int = 0) -> None:
        """Rebuild the device plan with other execution options (baas_replan), keeping the analysis."""
        opt = _native.BaasOptions()
        _native.lib().baas_options_default(C.byref(opt))
        opt.nthread = self.nthread
        opt.mapping = self.mapping
        opt.parts = parts
        opt.smem_budget = smem_budget
        opt.partition = partition
        opt.spin_limit = spin_limit
        opt.walk = walk
        opt.small_cluster = small_cluster
        _native.check(_native.lib().baas_replan(self._h, C.byref(opt)), "baas_replan")

    def replan_custom(self, row_part, parts: int | None = None, smem_budget: int = 0) -> None:
        """Rebuild the device plan with row i owned by CTA row_part[i] (baas_replan_custom); parts
        defaults to max(row_part) + 1."""
        rp = np.ascontiguousarray(row_part, dtype=np.int32)
        if rp.shape != (self.n,):
            raise ValueError("row_part needs one entry per row")
        if parts is None:
            parts = int(rp.max()) + 1
        _native.check(_native.lib().baas_replan_custom(self._h, _ptr(rp), int(parts), int(smem_budget)),
                      "baas_replan_custom")

    def emulate_sweep(self, T: CSR, b: np.ndarray, upper: bool = False, parts: int = 0,
                      smem_budget: int = 0) -> np.ndarray:
        """Test hook: run the chunked sweep plan on the host (no GPU) and return x."""
        tv = np.ascontiguousarray(T.values, dtype=np.float64)
        bb = np.ascontiguousarray(b, dtype=np.float64)
        x = np.zeros(self.n)
        _native.check(_native.lib().baas_test_emulate_sweep(self._h, parts, smem_budget, int(upper), _ptr(tv),
                                                             _ptr(bb), _ptr(x)), "emulate_sweep")
        return x

    def emulate_fetch(self, T: CSR, b: np.ndarray, upper: bool = False, parts: int = 0) -> np.ndarray:
        """Test hook: run the fetch-walk plan on the host (no GPU) and return x."""
        tv = np.ascontiguousarray(T.values, dtype=np.float64)
        bb = np.ascontiguousarray(b, dtype=np.float64)
        x = np.zeros(self.n)
        _native.check(_native.lib().baas_test_emulate_fetch(self._h, parts, int(upper), _ptr(tv), _ptr(bb), _ptr(x)),
                      "emulate_fetch")
        return x

    @property
    def analysis_ms(self) -> float:
        return _native.lib().baas_schedule_analysis_ms(self._h)

    # ---- device compute (torch CUDA tensors) ----
    def sptrsv(self, T: DeviceCSR, b, x, upper: bool, stream=None) -> None:
        """x = T^-1 b for T lower (diagonal last) or upper (diagonal first); b, x are (n,) or
        (nrhs, n) contiguous float64 CUDA tensors (rows of a 2-D tensor are right-hand sides)."""
        nrhs = 1 if b.dim() == 1 else int(b.shape[0])
        c = T.c()
        st = _native.lib().baas_sptrsv(self._h, C.byref(c), int(upper), _ptr(b), _ptr(x), nrhs, self.n,
                                       _stream_ptr(stream))
        _native.check(st, "baas_sptrsv")

    def forward(self, L: DeviceCSR, b, x, stream=None) -> None:
        self.sptrsv(L, b, x, False, stream)

    def backward(self, U: DeviceCSR, b, x, stream=None) -> None:
        self.sptrsv(U, b, x, True, stream)

    def ic0(self, A: DeviceCSR, lu, stream=None) -> None:
        """IC0 in place on lu (pre-filled with A.values)."""
        c = A.c()
        _native.check(_native.lib().baas_ic0(self._h, C.byref(c), _ptr(lu), _stream_ptr(stream)), "baas_ic0")

    def ic0_noalloc(self, A: DeviceCSR, lu, stream=None) -> None:
        """IC0 that allocates no device memory (static scratch inside the library; at most
        2,097,152 rows). The schedule must have run one ordinary GPU call first."""
        c = A.c()
        _native.check(_native.lib().baas_ic0_noalloc(self._h, C.byref(c), _ptr(lu), _stream_ptr(stream)),
                      "baas_ic0_noalloc")

    def ilu0(self, A: DeviceCSR, lu, stream=None) -> None:
        """ILU0 in place on lu (pre-filled with A.values)."""
        c = A.c()
        _native.check(_native.lib().baas_ilu0(self._h, C.byref(c), _ptr(lu), _stream_ptr(stream)), "baas_ilu0")

    def iccg(self, A: DeviceCSR, b, x, tol: float = 1e-10, maxiter: int = 2000, precision: int = PREC_FP64,
             stream=None, raise_on_nonconvergence: bool = True, raise_on_zero_pivot: bool = True):
        """IC0-PCG solve; x holds the initial guess. Returns (iterations, relative residual).
        raise_on_zero_pivot=False accepts a factor with non-positive pivots, which IC0 leaves
        unchanged as the reference does (merge/IC.cpp:371-378), and returns the solve's result."""
        c = A.c()
        it = C.c_int(0)
        rr = C.c_double(0.0)
        st = _native.lib().baas_iccg(self._h, C.byref(c), _ptr(b), _ptr(x), tol, maxiter, precision,
                                     C.byref(it), C.byref(rr), _stream_ptr(stream))
        if (st == 5 and not raise_on_nonconvergence) or (st == 4 and not raise_on_zero_pivot):
            return it.value, rr.value
        _native.check(st, "baas_iccg")
        return it.value, rr.value

    def iccg_adjoint(self, A: DeviceCSR, g, lam, x=None, grad_a=None, tol: float = 1e-10, maxiter: int = 2000,
                     precision: int = PREC_FP64, stream=None, raise_on_nonconvergence: bool = True):
        """Adjoint solve A^T lam = g with the factors of the previous `iccg` call; if x and grad_a
        are given, grad_a[e] = -lam_i x_j on A's pattern. Returns (iterations, relative residual)."""
        c = A.c()
        it = C.c_int(0)
        rr = C.c_double(0.0)
        st = _native.lib().baas_iccg_adjoint(self._h, C.byref(c), _ptr(g), _ptr(lam),
                                             _ptr(x) if x is not None else None,
                                             _ptr(grad_a) if grad_a is not None else None, tol, maxiter, precision,
                                             C.byref(it), C.byref(rr), _stream_ptr(stream))
        if st == 5 and not raise_on_nonconvergence:
            return it.value, rr.value
        _native.check(st, "baas_iccg_adjoint")
        return it.value, rr.value


def batch_concat(systems) -> tuple[CSR, np.ndarray]:
    """The block-diagonal concatenation of CSR systems and their row offsets (baas_batch_concat)."""
    ns = len(systems)
    arrs = [(np.ascontiguousarray(m.rowptr, dtype=np.int32), np.ascontiguousarray(m.colidx, dtype=np.int32),
             np.ascontiguousarray(m.values, dtype=np.float64)) for m in systems]
    cs = (_native.BaasCsr * ns)(*[_native.BaasCsr(m.n, int(a[0][-1]), _ptr(a[0]), _ptr(a[1]), _ptr(a[2]))
                                  for m, a in zip(systems, arrs)])
    ptrs = (C.POINTER(_native.BaasCsr) * ns)(*[C.pointer(cs[k]) for k in range(ns)])
    L = _native.lib()
    nnz = L.baas_batch_concat(ns, ptrs, None, None, None, None)
    if nnz < 0:
        raise ValueError("bad systems")
    n = sum(m.n for m in systems)
    rowptr = np.zeros(n + 1, dtype=np.int32)
    colidx = np.zeros(nnz, dtype=np.int32)
    values = np.zeros(nnz, dtype=np.float64)
    off = np.zeros(ns + 1, dtype=np.int32)
    L.baas_batch_concat(ns, ptrs, _ptr(rowptr), _ptr(colidx), _ptr(values), _ptr(off))
    return CSR(n, rowptr, colidx, values), off


class BatchSchedule(Schedule):
    """One ICCG schedule for a batch of independent SPD systems (block-diagonal concatenation)."""

    def __init__(self, systems, nthread: int = 8, spin_limit: int = 0, parts: int = 0, smem_budget: int = 0,
                 analysis: int = ANALYSIS_HOST):
        A, off = batch_concat(systems)
        self.combined = A
        self.sys_off = off
        self.nsys = len(systems)
        L = _native.lib()
        self._rowptr, self._colidx = A.rowptr, A.colidx
        c = _native.BaasCsr(A.n, A.nnz, _ptr(A.rowptr), _ptr(A.colidx), None)
        opt = _native.BaasOptions()
        L.baas_options_default(C.byref(opt))
        opt.nthread = nthread
        opt.spin_limit = spin_limit
        opt.parts = parts
        opt.smem_budget = smem_budget
        opt.analysis = analysis
        h = C.c_void_p()
        _native.check(L.baas_analyze_batch(C.byref(c), _ptr(off), self.nsys, C.byref(opt), C.byref(h)),
                      "baas_analyze_batch")
        self._h = h
        self.n = A.n
        self.nnz = A.nnz
        self.kind = KERNEL_ICCG
        self.nthread = nthread
        self.mapping = MAPPING_FOUR_RULE  # batched analyses use the four-rule mapping

    def iccg_batched(self, A: DeviceCSR, B, X, tol: float = 1e-10, maxiter: int = 2000,
                     precision: int = PREC_FP64, stream=None, raise_on_nonconvergence: bool = True):
        """B, X: (nrhs, n) CUDA float64 tensors (row r = right-hand side r). Returns per-instance
        iterations and relative residuals as (nsys, nrhs) arrays."""
        nrhs = int(B.shape[0]) if B.dim() == 2 else 1
        it = np.zeros(self.nsys * nrhs, dtype=np.int32)
        rr = np.zeros(self.nsys * nrhs, dtype=np.float64)
        c = A.c()
        st = _native.lib().baas_iccg_batched(self._h, C.byref(c), _ptr(B), _ptr(X), nrhs, self.n, tol, maxiter,
                                             precision, _ptr(it), _ptr(rr), _stream_ptr(stream))
        if not (st == 5 and not raise_on_nonconvergence):
            _native.check(st, "baas_iccg_batched")
        return it.reshape(self.nsys, nrhs), rr.reshape(self.nsys, nrhs)
