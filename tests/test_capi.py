"""The C-ABI library: it loads without a GPU, exports every symbol include/baas_b200.h
declares, and rejects bad input on the host with BAAS_ERR_BAD_ARG (no compute without a GPU)."""
import ctypes as C
import re
from pathlib import Path

import numpy as np
import pytest

from baas_b200 import KERNEL_ICCG, KERNEL_SPTRSV, BaasError, Schedule, _native, gen

HEADER = Path(__file__).resolve().parents[1] / "include" / "baas_b200.h"


def _declared():
    text = HEADER.read_text()
    return sorted(set(re.findall(r"^\s*(?:baas_status|void|int|double|const char \*)\s*\*?\s*(baas_\w+)\s*\(", text, re.M)))


def test_library_loads_and_exports_every_declared_symbol():
    L = _native.lib()
    names = _declared()
    assert len(names) >= 10
    for n in names:
        assert hasattr(L, n), n
    assert set(names) == set(_native.EXPORTS)
    assert _native.lib().baas_version().decode().startswith("baas_b200")


def _bad(A, kind=KERNEL_ICCG, **kw):
    with pytest.raises(BaasError) as e:
        Schedule(A, kind=kind, **kw)
    assert e.value.status_name == "BAAS_ERR_BAD_ARG"
    return str(e.value)


def test_rejects_missing_diagonal():
    import scipy.sparse as sp

    m = sp.csr_matrix(np.array([[1.0, 0, 0], [1.0, 0, 0], [0, 1.0, 1.0]]))
    assert "diagonal" in _bad(gen.from_scipy(m), kind=KERNEL_SPTRSV)


def test_rejects_upper_entries_for_sptrsv():
    assert "lower" in _bad(gen.laplace2d(4), kind=KERNEL_SPTRSV)


def test_rejects_unsorted_rows():
    A = gen.laplace2d(4)
    col = A.colidx.copy()
    col[0], col[1] = col[1], col[0]
    assert "ascending" in _bad(gen.CSR(A.n, A.rowptr, col, A.values))


def test_rejects_nonsymmetric_pattern():
    import scipy.sparse as sp

    m = sp.csr_matrix(np.array([[2.0, 0, 0], [1.0, 2.0, 0], [0, 0, 2.0]]))
    assert "symmetric" in _bad(gen.from_scipy(m))


def test_rejects_bad_options():
    _bad(gen.laplace2d(4), nthread=0)


def test_bad_arg_on_null_and_size_mismatch():
    L = _native.lib()
    s = Schedule(gen.laplace2d(5).lower(), kind=KERNEL_SPTRSV, nthread=2)
    # a factor with the wrong nnz is rejected before any GPU work
    bad = _native.BaasCsr(s.n, 3, None, None, None)
    st = L.baas_sptrsv(s._h, C.byref(bad), 0, C.c_void_p(8), C.c_void_p(16), 1, s.n, None)
    assert st == 1
    assert L.baas_schedule_export(s._h, 99, None) == -1


def test_ic0_noalloc_refuses_patterns_above_its_scratch_size():
    # the allocation-free IC0's static scratch holds one ready flag per row, at most 2,097,152;
    # a larger pattern is refused on the host, before any device call (a diagonal keeps the
    # analysis cheap)
    n = (1 << 21) + 1
    A = gen.CSR(n, np.arange(n + 1, dtype=np.int32), np.arange(n, dtype=np.int32), np.ones(n))
    s = Schedule(A, kind=KERNEL_ICCG, nthread=2)
    L = _native.lib()
    c = _native.BaasCsr(n, n, A.rowptr.ctypes.data, A.colidx.ctypes.data, A.values.ctypes.data)
    lu = np.ones(n)
    assert L.baas_ic0_noalloc(s._h, C.byref(c), lu.ctypes.data, None) == 1  # BAAS_ERR_BAD_ARG
    assert "at most 2097152 rows" in L.baas_last_error_string().decode()


def test_analysis_time_reported():
    s = Schedule(gen.laplace3d(8, 1e-3), kind=KERNEL_ICCG, nthread=4)
    assert s.analysis_ms > 0.0


def test_analysis_placement_option():
    from baas_b200 import ANALYSIS_DEVICE, BaasError

    _bad(gen.laplace2d(4), analysis=7)
    import torch

    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present: the device analysis runs (test_gpu_analysis.py)")
    with pytest.raises(BaasError) as e:
        Schedule(gen.laplace2d(4), kind=KERNEL_ICCG, nthread=2, analysis=ANALYSIS_DEVICE)
    assert e.value.status_name == "BAAS_ERR_NO_DEVICE"


def test_scoring_constants():
    """The four-rule mapping's scoring constants (the reference's MergeMarco.hpp macros): the
    defaults are the reference's values, so naming them changes nothing; other values change the
    mapping but not the level sets; out-of-range values are refused."""
    A = gen.knn_stiffness(nodes=600, k=12, seed=3)
    base = Schedule(A, kind=KERNEL_ICCG, nthread=8).arrays()
    same = Schedule(A, kind=KERNEL_ICCG, nthread=8,
                    scoring={"level_window": 6, "amplify": 2.0, "over_gamma": 6.0, "award_alpha": 1.0,
                             "load_beta": 0.1}).arrays()
    assert all(np.array_equal(base[f], same[f]) for f in base)
    other = Schedule(A, kind=KERNEL_ICCG, nthread=8, scoring={"award_alpha": 0.0, "level_window": 2}).arrays()
    assert np.array_equal(base["level_ptr"], other["level_ptr"])
    assert not np.array_equal(base["thread_cont_to_orig"], other["thread_cont_to_orig"])
    _bad(A, scoring={"level_window": -1})
    _bad(A, scoring={"amplify": float("nan")})


def test_execution_option_checks():
    """walk, small_cluster and ablation values outside their sets are refused at analysis time."""
    A = gen.laplace2d(6)
    _bad(A, walk=9)
    _bad(A, small_cluster=3)
    _bad(A, small_cluster=32)
    _bad(gen.laplace2d(6).lower(), kind=KERNEL_SPTRSV, ablation=4)
    from baas_b200 import WALK_SMALL

    s = Schedule(A, kind=KERNEL_ICCG, nthread=2, walk=WALK_SMALL, small_cluster=16)
    with pytest.raises(BaasError):
        s.replan(walk=WALK_SMALL, small_cluster=5)
