"""The chunked sweep plan (the layout the sweep kernels read), checked on the host: the plan is
run CTA by CTA by the library's emulator, which validates every offset, size and index, and
the result must equal the oracle bit for bit. Covers partitions, window budgets (resident and
streamed plans), both sweep directions and every matrix family."""
import numpy as np
import pytest

from baas_b200 import KERNEL_ICCG, KERNEL_ILU0, KERNEL_SPTRSV, PARTITION_BAAS_THREADS, Schedule, gen
from oracle.oracle import Port


def _ic_lu(A):
    lu, _ = Port.ic0(A)
    Lo = gen.CSR(A.n, A.rowptr, A.colidx, lu).lower()
    return Lo, Lo.transpose()


@pytest.mark.parametrize("parts", [1, 5, 32, 0])
def test_c1_plan(parts):
    L, _, b = gen.sptrsv_case(128, 0)
    s = Schedule(L, kind=KERNEL_SPTRSV, nthread=8)
    assert np.array_equal(s.emulate_sweep(L, b, parts=parts), Port.lower_solve(L, b))


@pytest.mark.parametrize("budget", [20 * 1024, 28 * 1024, 0])
@pytest.mark.parametrize("upper", [False, True])
def test_ic_plan_budgets(budget, upper):
    A = gen.laplace3d(20, 1e-3)
    Lo, Up = _ic_lu(A)
    s = Schedule(A, kind=KERNEL_ICCG, nthread=8)
    r = gen.uniform_rhs(A.n, 1)
    if upper:
        want = Port.upper_solve(Up, r, descending=True)
        got = s.emulate_sweep(Up, r, upper=True, parts=6, smem_budget=budget)
    else:
        want = Port.lower_solve(Lo, r)
        got = s.emulate_sweep(Lo, r, parts=6, smem_budget=budget)
    assert np.array_equal(got, want)


def test_knn_and_permuted_plans():
    for A in (gen.knn_stiffness(nodes=500, k=12, seed=3),
              gen.laplace3d(12, 1e-3).permuted(gen.random_symmetric_permutation(12 ** 3, 7))):
        Lo, Up = _ic_lu(A)
        s = Schedule(A, kind=KERNEL_ICCG, nthread=8)
        r = gen.uniform_rhs(A.n, 1)
        for parts in (3, 16):
            assert np.array_equal(s.emulate_sweep(Lo, r, parts=parts), Port.lower_solve(Lo, r))
            assert np.array_equal(s.emulate_sweep(Up, r, upper=True, parts=parts),
                                  Port.upper_solve(Up, r, descending=True))


def test_ilu_plan():
    import scipy.sparse as sp

    C = gen.convdiff3d(10)
    lu, _ = Port.ilu0(C)
    M = gen.CSR(C.n, C.rowptr, C.colidx, lu).to_scipy()
    Lo = gen.from_scipy(sp.tril(M, k=-1) + sp.identity(C.n, format="csr"))
    Up = gen.from_scipy(sp.triu(M))
    s = Schedule(C, kind=KERNEL_ILU0, nthread=6)
    b = gen.normal_rhs(C.n, 2)
    assert np.array_equal(s.emulate_sweep(Lo, b, parts=7), Port.lower_solve(Lo, b))
    assert np.array_equal(s.emulate_sweep(Up, b, upper=True, parts=7), Port.upper_solve(Up, b, descending=True))


def test_baas_threads_partition_plan():
    A = gen.laplace3d(10, 1e-3)
    Lo, Up = _ic_lu(A)
    s = Schedule(A, kind=KERNEL_ICCG, nthread=12, partition=PARTITION_BAAS_THREADS)
    r = gen.uniform_rhs(A.n, 1)
    assert np.array_equal(s.emulate_sweep(Lo, r), Port.lower_solve(Lo, r))
    assert np.array_equal(s.emulate_sweep(Up, r, upper=True), Port.upper_solve(Up, r, descending=True))


def test_plan_rejects_tiny_budget():
    from baas_b200 import BaasError

    A = gen.laplace3d(20, 1e-3)
    Lo, _ = _ic_lu(A)
    s = Schedule(A, kind=KERNEL_ICCG, nthread=8)
    with pytest.raises(BaasError):
        s.emulate_sweep(Lo, np.zeros(A.n), parts=1, smem_budget=2048)


def test_liveness_slots_let_one_cta_stream_a_large_plan():
    """Slots live only until a row's last local reader, so one CTA holding all 8,000 rows (one
    slot per row would need 64 KB for the slots alone) fits a 40 KB budget and streams its plan in windows."""
    A = gen.laplace3d(20, 1e-3)
    Lo, Up = _ic_lu(A)
    s = Schedule(A, kind=KERNEL_ICCG, nthread=8)
    r = gen.uniform_rhs(A.n, 1)
    assert np.array_equal(s.emulate_sweep(Lo, r, parts=1, smem_budget=40 * 1024), Port.lower_solve(Lo, r))
    assert np.array_equal(s.emulate_sweep(Up, r, upper=True, parts=1, smem_budget=40 * 1024),
                          Port.upper_solve(Up, r, descending=True))
