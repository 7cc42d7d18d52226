"""ctypes binding of the in-tree C ABI (include/baas_b200.h).

The library is ``baas_b200/_lib/libbaas_b200.so`` built by :mod:`baas_b200.build`. Importing
this module never falls back to anything else: if the library is missing, :func:`lib` raises.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

# BAAS_LIB=bounds selects the bounds-checked build (python -m baas_b200.build --debug-bounds)
_LIB_PATH = Path(__file__).resolve().parent / "_lib" / (
    "libbaas_b200_bounds.so" if os.environ.get("BAAS_LIB") == "bounds" else "libbaas_b200.so")
_lib = None

BAAS_OK = 0
STATUS_NAMES = {
    0: "BAAS_OK",
    1: "BAAS_ERR_BAD_ARG",
    2: "BAAS_ERR_CUDA",
    3: "BAAS_ERR_TIMEOUT",
    4: "BAAS_ERR_ZERO_PIVOT",
    5: "BAAS_ERR_NOT_CONVERGED",
    6: "BAAS_ERR_NO_DEVICE",
    7: "BAAS_ERR_STATE",
}

KERNEL_SPTRSV, KERNEL_ICCG, KERNEL_IC0, KERNEL_ILU0 = 0, 1, 2, 3
PREC_FP64, PREC_FP32_FACTORS = 0, 1
PARTITION_RANGES, PARTITION_BAAS_THREADS, PARTITION_CUSTOM, PARTITION_BLOCKS, PARTITION_AUTO = 0, 1, 2, 3, 4
WALK_AUTO, WALK_CHUNKED, WALK_FETCH, WALK_LEVELS, WALK_SMALL = 0, 1, 2, 3, 4
ANALYSIS_HOST, ANALYSIS_DEVICE = 0, 1
ABLATION_NONE, ABLATION_WOS, ABLATION_WOA, ABLATION_WOAS = 0, 1, 2, 3
MAPPING_FOUR_RULE, MAPPING_COST_SPLIT, MAPPING_COST_SPLIT_BARRIER, MAPPING_FINISH_TIME, MAPPING_AFFINITY = 0, 1, 2, 3, 4

FIELDS = {
    "ngroups": 0, "nlevels": 1, "ntasks": 2, "group_ptr": 3, "group_set": 4, "level_ptr": 5,
    "perm_to_orig": 6, "node_to_level": 7, "nthread_per_level": 8, "thread_boundaries": 9,
    "task_boundaries": 10, "thread_cont_to_orig": 11, "orig_to_thread_cont": 12, "task_ptr": 13,
    "task_set": 14, "btask_ptr": 15, "btask_set": 16, "cost": 17,
}
# the final group DAG (CSC, each group's column: its children and itself, ascending): not one of
# the reference's exported arrays, but what the device plans are built from
GROUP_DAG_FIELDS = {"group_dag_ptr": 18, "group_dag_set": 19}

# every symbol include/baas_b200.h declares
EXPORTS = [
    "baas_options_default", "baas_analyze", "baas_schedule_export", "baas_schedule_analysis_ms",
    "baas_destroy", "baas_sptrsv", "baas_ic0", "baas_ilu0", "baas_iccg", "baas_last_error_string",
    "baas_version", "baas_test_inject_unsatisfiable_wait", "baas_ic0_noalloc", "baas_test_emulate_sweep", "baas_iccg_adjoint", "baas_batch_concat", "baas_analyze_batch", "baas_iccg_batched", "baas_replan", "baas_test_divide", "baas_replan_custom", "baas_csr_read_mtx", "baas_csr_free",
    "baas_schedule_last_walk", "baas_test_emulate_fetch", "baas_plan_parts", "baas_schedule_save",
    "baas_schedule_load", "baas_schedule_info",
]


class BaasCsr(C.Structure):
    _fields_ = [("n", C.c_int), ("nnz", C.c_int), ("rowptr", C.c_void_p), ("colidx", C.c_void_p),
                ("values", C.c_void_p)]


class BaasOptions(C.Structure):
    _fields_ = [("nthread", C.c_int), ("spin_limit", C.c_int), ("parts", C.c_int),
                ("partition", C.c_int), ("smem_budget", C.c_int), ("mapping", C.c_int), ("walk", C.c_int),
                ("analysis", C.c_int), ("ablation", C.c_int),
                ("small_cluster", C.c_int), ("level_window", C.c_int), ("amplify", C.c_double),
                ("over_gamma", C.c_double), ("award_alpha", C.c_double), ("load_beta", C.c_double)]


class BaasError(RuntimeError):
    def __init__(self, status: int, where: str, detail: str):
        self.status = status
        self.status_name = STATUS_NAMES.get(status, str(status))
        super().__init__(f"{where}: {self.status_name}: {detail}")


def lib_path() -> Path:
    return _LIB_PATH


def lib():
    """Load the CUDA library (raises if it was not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not _LIB_PATH.exists():
        raise RuntimeError(f"{_LIB_PATH} is missing: run `python -m baas_b200.build` (no CPU fallback exists)")
    L = C.CDLL(str(_LIB_PATH))
    vp, i, d = C.c_void_p, C.c_int, C.c_double
    L.baas_options_default.argtypes = [C.POINTER(BaasOptions)]
    L.baas_options_default.restype = None
    L.baas_analyze.argtypes = [C.POINTER(BaasCsr), i, C.POINTER(BaasOptions), C.POINTER(vp)]
    L.baas_analyze.restype = i
    L.baas_schedule_export.argtypes = [vp, i, vp]
    L.baas_schedule_export.restype = i
    L.baas_schedule_analysis_ms.argtypes = [vp]
    L.baas_schedule_analysis_ms.restype = d
    L.baas_schedule_last_walk.argtypes = [vp]
    L.baas_schedule_last_walk.restype = i
    L.baas_plan_parts.argtypes = [vp, vp]
    L.baas_plan_parts.restype = i
    L.baas_schedule_save.argtypes = [vp, C.c_char_p]
    L.baas_schedule_save.restype = i
    L.baas_schedule_load.argtypes = [C.c_char_p, C.POINTER(vp)]
    L.baas_schedule_load.restype = i
    L.baas_schedule_info.argtypes = [vp, vp]
    L.baas_schedule_info.restype = i
    L.baas_destroy.argtypes = [vp]
    L.baas_destroy.restype = None
    L.baas_sptrsv.argtypes = [vp, C.POINTER(BaasCsr), i, vp, vp, i, i, vp]
    L.baas_sptrsv.restype = i
    L.baas_ic0.argtypes = [vp, C.POINTER(BaasCsr), vp, vp]
    L.baas_ic0.restype = i
    L.baas_ic0_noalloc.argtypes = [vp, C.POINTER(BaasCsr), vp, vp]
    L.baas_ic0_noalloc.restype = i
    L.baas_ilu0.argtypes = [vp, C.POINTER(BaasCsr), vp, vp]
    L.baas_ilu0.restype = i
    L.baas_iccg.argtypes = [vp, C.POINTER(BaasCsr), vp, vp, d, i, i, C.POINTER(C.c_int), C.POINTER(C.c_double), vp]
    L.baas_iccg.restype = i
    L.baas_last_error_string.argtypes = []
    L.baas_last_error_string.restype = C.c_char_p
    L.baas_version.argtypes = []
    L.baas_version.restype = C.c_char_p
    L.baas_test_inject_unsatisfiable_wait.argtypes = [vp, i]
    L.baas_test_inject_unsatisfiable_wait.restype = i
    L.baas_iccg_adjoint.argtypes = [vp, C.POINTER(BaasCsr), vp, vp, vp, vp, d, i, i, C.POINTER(C.c_int),
                                    C.POINTER(C.c_double), vp]
    L.baas_iccg_adjoint.restype = i
    L.baas_replan.argtypes = [vp, C.POINTER(BaasOptions)]
    L.baas_replan.restype = i
    L.baas_batch_concat.argtypes = [i, vp, vp, vp, vp, vp]
    L.baas_batch_concat.restype = i
    L.baas_analyze_batch.argtypes = [C.POINTER(BaasCsr), vp, i, C.POINTER(BaasOptions), C.POINTER(vp)]
    L.baas_analyze_batch.restype = i
    L.baas_iccg_batched.argtypes = [vp, C.POINTER(BaasCsr), vp, vp, i, i, d, i, i, vp, vp, vp]
    L.baas_iccg_batched.restype = i
    L.baas_test_emulate_sweep.argtypes = [vp, i, i, i, vp, vp, vp]
    L.baas_test_emulate_sweep.restype = i
    L.baas_test_emulate_fetch.argtypes = [vp, i, i, vp, vp, vp]
    L.baas_test_emulate_fetch.restype = i
    L.baas_test_divide.argtypes = [vp, vp, vp, C.c_longlong, i, vp]
    L.baas_test_divide.restype = i
    L.baas_replan_custom.argtypes = [vp, vp, i, i]
    L.baas_replan_custom.restype = i
    L.baas_csr_read_mtx.argtypes = [C.c_char_p, C.POINTER(BaasCsr)]
    L.baas_csr_read_mtx.restype = i
    L.baas_csr_free.argtypes = [C.POINTER(BaasCsr)]
    L.baas_csr_free.restype = None
    _lib = L
    return L


def check(status: int, where: str) -> None:
    if status != BAAS_OK:
        raise BaasError(status, where, lib().baas_last_error_string().decode())
