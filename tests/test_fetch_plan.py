"""The fetch-walk plan (rows of at most 3 off-diagonal entries, one right-hand side), checked on the
host: the library's emulator runs it step by step, each step only once the producers of its
staged values are written, validating every record, slot, fetch-list entry and value code; the
result must equal the oracle bit for bit. Covers the stencil families, a random symmetric
permutation, custom and BAAS-thread partitions, and both sweep directions; wide rows are refused."""
import numpy as np
import pytest

from baas_b200 import BaasError, KERNEL_ICCG, KERNEL_SPTRSV, PARTITION_BAAS_THREADS, Schedule, gen
from oracle.oracle import Port


def _ic_lu(A):
    lu, _ = Port.ic0(A)
    Lo = gen.CSR(A.n, A.rowptr, A.colidx, lu).lower()
    return Lo, Lo.transpose()


def _both(s, A, r, parts):
    Lo, Up = _ic_lu(A)
    assert np.array_equal(s.emulate_fetch(Lo, r, parts=parts), Port.lower_solve(Lo, r))
    assert np.array_equal(s.emulate_fetch(Up, r, upper=True, parts=parts), Port.upper_solve(Up, r, descending=True))


@pytest.mark.parametrize("parts", [8, 16, 0])
def test_c1_fetch_plan(parts):
    L, _, b = gen.sptrsv_case(128, 0)
    s = Schedule(L, kind=KERNEL_SPTRSV, nthread=8)
    assert np.array_equal(s.emulate_fetch(L, b, parts=parts), Port.lower_solve(L, b))


@pytest.mark.parametrize("parts", [2, 7, 27, 0])
def test_laplace3d_fetch_plan(parts):
    A = gen.laplace3d(18, 1e-3)
    s = Schedule(A, kind=KERNEL_ICCG, nthread=8)
    _both(s, A, gen.uniform_rhs(A.n, 1), parts)


def test_varcoef_fetch_plan():
    rng = np.random.default_rng(5)
    k = 10
    theta = tuple(rng.normal(0.0, 0.5, size=s) for s in ((k, k, k - 1), (k, k - 1, k), (k - 1, k, k)))
    B = gen.vardiff3d_faces(k, theta)
    _both(Schedule(B, kind=KERNEL_ICCG, nthread=4), B, gen.uniform_rhs(B.n, 2), 5)


def test_baas_threads_and_custom_fetch_plans():
    A = gen.laplace3d(10, 1e-3)
    r = gen.uniform_rhs(A.n, 1)
    _both(Schedule(A, kind=KERNEL_ICCG, nthread=12, partition=PARTITION_BAAS_THREADS), A, r, 0)
    s = Schedule(A, kind=KERNEL_ICCG, nthread=8)
    k = 10
    ijk = np.arange(A.n)
    i, j, kk = ijk % k, (ijk // k) % k, ijk // (k * k)
    s.replan_custom((i // 5) + 2 * (j // 5) + 4 * (kk // 5))  # 2x2x2 blocks of 5^3 rows
    _both(s, A, r, 0)


def test_oversized_cta_is_refused():
    L, _, b = gen.sptrsv_case(128, 0)
    s = Schedule(L, kind=KERNEL_SPTRSV, nthread=8)
    with pytest.raises(BaasError, match="does not fit shared memory"):
        s.emulate_fetch(L, b, parts=1)


@pytest.mark.parametrize("which", ["knn", "permuted"])
def test_wide_rows_are_refused(which):
    # a k-NN stiffness matrix, and a 7-point stencil under a random symmetric permutation (a row's
    # lower part then holds up to 6 neighbours), have rows of more than 3 off-diagonal entries
    if which == "knn":
        A = gen.knn_stiffness(nodes=300, k=12, seed=3)
    else:
        A = gen.laplace3d(12, 1e-3).permuted(gen.random_symmetric_permutation(12 ** 3, 7))
    Lo, _ = _ic_lu(A)
    s = Schedule(A, kind=KERNEL_ICCG, nthread=8)
    with pytest.raises(BaasError, match="does not qualify"):
        s.emulate_fetch(Lo, gen.uniform_rhs(A.n, 1), parts=8)
