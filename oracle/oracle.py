"""ctypes access to the two checkers -- TEST INFRASTRUCTURE ONLY.

* :class:`Ref` -- the reference itself, compiled from its own sources into
  ``oracle/_ref/libbaas_ref.so`` by ``oracle/Makefile`` (present wherever that library was
  built; the reference tree is not needed at run time).
* :class:`Port` -- ``oracle/baas_oracle.c``, our plain-C restatement of the reference's serial
  numeric routines and of the pcg loop, each function citing the reference line it follows.

Only tests/, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline / reference arms
import this module, and only to check or to time the CPU path -- never as the product.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REF_LIB = HERE / "_ref" / "libbaas_ref.so"
PORT_LIB = HERE / "_lib" / "libbaas_oracle.so"

FIELDS = {
    "ngroups": 0, "nlevels": 1, "ntasks": 2, "group_ptr": 3, "group_set": 4, "level_ptr": 5,
    "perm_to_orig": 6, "node_to_level": 7, "nthread_per_level": 8, "thread_boundaries": 9,
    "task_boundaries": 10, "thread_cont_to_orig": 11, "orig_to_thread_cont": 12, "task_ptr": 13,
    "task_set": 14, "btask_ptr": 15, "btask_set": 16, "cost": 17,
}

_vp, _i, _d = C.c_void_p, C.c_int, C.c_double


def _p(a: np.ndarray) -> int:
    return a.ctypes.data


def ref_available() -> bool:
    return REF_LIB.exists()


class Ref:
    """The reference's own routines (schedule, p2p executors, serial routines, pcg)."""

    _lib = None

    @classmethod
    def lib(cls):
        if cls._lib is None:
            if not REF_LIB.exists():
                raise RuntimeError(f"{REF_LIB} not built (make -C oracle ref)")
            L = C.CDLL(str(REF_LIB))
            L.ref_schedule_build.argtypes = [_i, _i, _vp, _vp, _i]
            L.ref_schedule_build.restype = _vp
            L.ref_schedule_get.argtypes = [_vp, _i, _vp]
            L.ref_schedule_get.restype = _i
            L.ref_schedule_free.argtypes = [_vp]
            L.ref_schedule_analysis_ms.argtypes = [_vp]
            L.ref_schedule_analysis_ms.restype = _d
            for name in ("ref_sptrsv_forward", "ref_sptrsv_backward"):
                getattr(L, name).argtypes = [_vp, _i, _vp, _vp, _vp, _vp, _vp]
            for name in ("ref_ic0", "ref_ilu0"):
                getattr(L, name).argtypes = [_vp, _i, _vp, _vp, _vp, _vp]
            for name in ("ref_sptrsv_serial", "ref_upper_serial"):
                getattr(L, name).argtypes = [_i, _vp, _vp, _vp, _vp, _vp]
            for name in ("ref_ic0_serial", "ref_ilu0_serial"):
                getattr(L, name).argtypes = [_i, _vp, _vp, _vp, _vp]
            L.ref_spmv.argtypes = [_i, _vp, _vp, _vp, _vp, _vp, _d, _d]
            L.ref_dot.argtypes = [_vp, _vp, _i]
            L.ref_dot.restype = _d
            L.ref_pcg.argtypes = [_i, _i, _i, _vp, _vp, _vp, _vp, _vp, _i, _d, _vp, _vp]
            L.ref_pcg.restype = _i
            L.ref_set_mapping.argtypes = [_i]
            L.ref_set_ablation.argtypes = [_i]
            L.ref_mtx_read.argtypes = [C.c_char_p, _vp, _vp]
            L.ref_mtx_read.restype = _vp
            L.ref_mtx_copy.argtypes = [_vp, _vp, _vp, _vp]
            L.ref_mtx_free.argtypes = [_vp]
            cls._lib = L
        return cls._lib

    @staticmethod
    def read_mtx(path):
        """The reference's own MatrixMarket reader (SPM::CSR(fileName), spm/CSR.cpp:90-112)."""
        from baas_b200.gen import CSR as _CSR

        L = Ref.lib()
        n, nnz = C.c_int(0), C.c_int(0)
        h = L.ref_mtx_read(str(path).encode(), C.byref(n), C.byref(nnz))
        try:
            rowptr = np.zeros(n.value + 1, dtype=np.int32)
            colidx = np.zeros(nnz.value, dtype=np.int32)
            values = np.zeros(nnz.value, dtype=np.float64)
            L.ref_mtx_copy(h, _p(rowptr), _p(colidx), _p(values))
        finally:
            L.ref_mtx_free(h)
        return _CSR(n.value, rowptr, colidx, values)

    class Schedule:
        def __init__(self, kind: int, A, nthread: int, mapping: int = 0, ablation: int = 0):
            """ablation (kind SPTRSV): 0 BAAS, 1 BAASWOS, 2 BAASWOA, 3 BAASWOAS -- the SpTRSV
            runtime's ablation classes (test/SpTRSV_level_merge.cpp:156-299)."""
            L = Ref.lib()
            self.rowptr = np.ascontiguousarray(A.rowptr, dtype=np.int32)
            self.colidx = np.ascontiguousarray(A.colidx, dtype=np.int32)
            self.n = A.n
            L.ref_set_mapping(mapping)
            L.ref_set_ablation(ablation)
            try:
                self.h = L.ref_schedule_build(kind, A.n, _p(self.rowptr), _p(self.colidx), nthread)
            finally:
                L.ref_set_mapping(0)
                L.ref_set_ablation(0)

        def __del__(self):
            if getattr(self, "h", None):
                Ref.lib().ref_schedule_free(self.h)
                self.h = None

        @property
        def analysis_ms(self) -> float:
            return Ref.lib().ref_schedule_analysis_ms(self.h)

        def export(self, field: str) -> np.ndarray:
            L = Ref.lib()
            n = L.ref_schedule_get(self.h, FIELDS[field], None)
            out = np.zeros(max(n, 1), dtype=np.int32)
            L.ref_schedule_get(self.h, FIELDS[field], _p(out))
            return out[:n]

        def arrays(self) -> dict:
            return {k: self.export(k) for k in FIELDS}

        def forward(self, L, b: np.ndarray) -> np.ndarray:
            x = np.zeros(L.n)
            bc = np.ascontiguousarray(b, dtype=np.float64)
            Ref.lib().ref_sptrsv_forward(self.h, L.n, _p(L.rowptr), _p(L.colidx), _p(L.values), _p(x),
                                         _p(bc))
            return x

        def backward(self, U, b: np.ndarray) -> np.ndarray:
            x = np.zeros(U.n)
            bc = np.ascontiguousarray(b, dtype=np.float64)
            Ref.lib().ref_sptrsv_backward(self.h, U.n, _p(U.rowptr), _p(U.colidx), _p(U.values), _p(x),
                                          _p(bc))
            return x

        def ic0(self, A) -> np.ndarray:
            lu = A.values.copy()
            Ref.lib().ref_ic0(self.h, A.n, _p(A.rowptr), _p(A.colidx), _p(A.values), _p(lu))
            return lu

        def ilu0(self, A) -> np.ndarray:
            lu = A.values.copy()
            Ref.lib().ref_ilu0(self.h, A.n, _p(A.rowptr), _p(A.colidx), _p(A.values), _p(lu))
            return lu

    @staticmethod
    def sptrsv_serial(L, b) -> np.ndarray:
        x = np.zeros(L.n)
        bc = np.ascontiguousarray(b, dtype=np.float64)
        Ref.lib().ref_sptrsv_serial(L.n, _p(L.rowptr), _p(L.colidx), _p(L.values), _p(x), _p(bc))
        return x

    @staticmethod
    def upper_serial(U, b) -> np.ndarray:
        x = np.zeros(U.n)
        bc = np.ascontiguousarray(b, dtype=np.float64)
        Ref.lib().ref_upper_serial(U.n, _p(U.rowptr), _p(U.colidx), _p(U.values), _p(x), _p(bc))
        return x

    @staticmethod
    def ic0_serial(A) -> np.ndarray:
        lu = A.values.copy()
        Ref.lib().ref_ic0_serial(A.n, _p(A.rowptr), _p(A.colidx), _p(A.values), _p(lu))
        return lu

    @staticmethod
    def ilu0_serial(A) -> np.ndarray:
        lu = A.values.copy()
        Ref.lib().ref_ilu0_serial(A.n, _p(A.rowptr), _p(A.colidx), _p(A.values), _p(lu))
        return lu

    @staticmethod
    def pcg(A, b, x0=None, maxiter=2000, tol=1e-10, mode=1, nthread=8):
        """mode 0 = pcg_ref structure (serial), 1 = pcg_opt structure (BAAS p2p).
        Returns (x, iterations, relres, times_ms[pre, ic, loop, total, trsv])."""
        x = np.zeros(A.n) if x0 is None else np.array(x0, dtype=np.float64)
        rel = C.c_double(0.0)
        t = np.zeros(5)
        bc = np.ascontiguousarray(b, dtype=np.float64)
        it = Ref.lib().ref_pcg(mode, nthread, A.n, _p(A.rowptr), _p(A.colidx), _p(A.values),
                               _p(bc), _p(x), maxiter, tol, C.addressof(rel), _p(t))
        return x, it, rel.value, t


class Port:
    """Plain-C restatement of the reference's serial numeric routines (oracle/baas_oracle.c)."""

    _lib = None

    @classmethod
    def lib(cls):
        if cls._lib is None:
            if not PORT_LIB.exists():
                raise RuntimeError(f"{PORT_LIB} not built (make -C oracle oracle)")
            L = C.CDLL(str(PORT_LIB))
            L.orc_lower_solve.argtypes = [_i, _vp, _vp, _vp, _vp, _vp]
            L.orc_upper_solve_desc.argtypes = [_i, _vp, _vp, _vp, _vp, _vp]
            L.orc_upper_solve_asc.argtypes = [_i, _vp, _vp, _vp, _vp, _vp]
            L.orc_ic0.argtypes = [_i, _vp, _vp, _vp, _vp]
            L.orc_ic0.restype = _i
            L.orc_ilu0.argtypes = [_i, _vp, _vp, _vp, _vp]
            L.orc_ilu0.restype = _i
            L.orc_spmv.argtypes = [_i, _vp, _vp, _vp, _vp, _vp, _d, _d]
            L.orc_pcg.argtypes = [_i, _vp, _vp, _vp, _vp, _vp, _i, _d, _vp, _vp]
            L.orc_pcg.restype = _i
            cls._lib = L
        return cls._lib

    @staticmethod
    def lower_solve(L, b):
        x = np.zeros(L.n)
        bc = np.ascontiguousarray(b, dtype=np.float64)
        Port.lib().orc_lower_solve(L.n, _p(L.rowptr), _p(L.colidx), _p(L.values), _p(bc), _p(x))
        return x

    @staticmethod
    def upper_solve(U, b, descending=True):
        x = np.zeros(U.n)
        bc = np.ascontiguousarray(b, dtype=np.float64)
        f = Port.lib().orc_upper_solve_desc if descending else Port.lib().orc_upper_solve_asc
        f(U.n, _p(U.rowptr), _p(U.colidx), _p(U.values), _p(bc), _p(x))
        return x

    @staticmethod
    def ic0(A):
        lu = A.values.copy()
        dp = A.diagptr()
        bad = Port.lib().orc_ic0(A.n, _p(A.rowptr), _p(A.colidx), _p(dp), _p(lu))
        return lu, bad

    @staticmethod
    def ilu0(A):
        lu = A.values.copy()
        dp = A.diagptr()
        bad = Port.lib().orc_ilu0(A.n, _p(A.rowptr), _p(A.colidx), _p(dp), _p(lu))
        return lu, bad

    @staticmethod
    def spmv(A, x, y=None, alpha=1.0, beta=0.0):
        y = np.zeros(A.n) if y is None else np.array(y, dtype=np.float64)
        xc = np.ascontiguousarray(x, dtype=np.float64)
        Port.lib().orc_spmv(A.n, _p(A.rowptr), _p(A.colidx), _p(A.values), _p(xc), _p(y), alpha, beta)
        return y

    @staticmethod
    def pcg(A, b, x0=None, maxiter=2000, tol=1e-10):
        """IC0-PCG with serial IC0 and serial sweeps; returns (x, iterations, relres)."""
        x = np.zeros(A.n) if x0 is None else np.array(x0, dtype=np.float64)
        rel = C.c_double(0.0)
        bc = np.ascontiguousarray(b, dtype=np.float64)
        it = Port.lib().orc_pcg(A.n, _p(A.rowptr), _p(A.colidx), _p(A.values), _p(bc), _p(x),
                                maxiter, tol, C.addressof(rel), None)
        return x, it, rel.value


def _pcg_job(job):
    """One oracle PCG solve in a worker process (top level, so a spawned worker can import it)."""
    from baas_b200.gen import CSR as _CSR

    n, rowptr, colidx, values, b, tol, maxiter = job
    return Port.pcg(_CSR(n, rowptr, colidx, values), b, tol=tol, maxiter=maxiter)


def pcg_many(jobs, workers=None):
    """Port.pcg over many (A, b, tol, maxiter) jobs in a pool of spawned worker processes (spawned,
    not forked, so a caller that already holds a CUDA context can use it). Returns the
    (x, iterations, relres) triples in job order."""
    import multiprocessing as mp
    import os

    packed = [(A.n, A.rowptr, A.colidx, A.values, np.ascontiguousarray(b, dtype=np.float64), tol, maxiter)
              for A, b, tol, maxiter in jobs]
    workers = max(1, min(len(packed), workers or os.cpu_count() or 1))
    if workers == 1:
        return [_pcg_job(j) for j in packed]
    with mp.get_context("spawn").Pool(workers) as pool:
        return pool.map(_pcg_job, packed, chunksize=1)
