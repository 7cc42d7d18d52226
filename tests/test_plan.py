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


def _column_blocks(k, bi, bj):
    """Row (i, j, l) of a k^3 grid (row = i + k*j + k*k*l) to the CTA of its (i // bi, j // bj)
    block of grid columns."""
    r = np.arange(k ** 3)
    i, j = r % k, (r // k) % k
    return (i // bi + ((k + bi - 1) // bi) * (j // bj)).astype(np.int32)


@pytest.mark.parametrize("budget", [24 * 1024, 0])
def test_custom_partition_plan(budget):
    """A caller's row-to-CTA map (baas_replan_custom): blocks of grid columns, so cross-CTA
    dependencies point both ways between CTAs."""
    A = gen.laplace3d(14, 1e-3)
    Lo, Up = _ic_lu(A)
    s = Schedule(A, kind=KERNEL_ICCG, nthread=8)
    rp = _column_blocks(14, 4, 5)
    s.replan_custom(rp, smem_budget=budget)
    r = gen.uniform_rhs(A.n, 1)
    assert np.array_equal(s.emulate_sweep(Lo, r, smem_budget=budget), Port.lower_solve(Lo, r))
    assert np.array_equal(s.emulate_sweep(Up, r, upper=True, smem_budget=budget),
                          Port.upper_solve(Up, r, descending=True))


def test_custom_partition_checks():
    from baas_b200 import PARTITION_CUSTOM, BaasError

    A = gen.laplace3d(6, 1e-3)
    s = Schedule(A, kind=KERNEL_ICCG, nthread=4)
    rp = np.zeros(A.n, dtype=np.int32)
    rp[::2] = 3
    with pytest.raises(BaasError):
        s.replan_custom(rp, parts=3)  # entries out of [0, parts)
    with pytest.raises(ValueError):
        s.replan_custom(rp[:-1])
    with pytest.raises(BaasError):
        s.replan(partition=PARTITION_CUSTOM)  # no map stored yet
    s.replan_custom(rp)  # parts = 4, CTAs 1 and 2 own no rows
    Lo, _ = _ic_lu(A)
    b = gen.uniform_rhs(A.n, 3)
    assert np.array_equal(s.emulate_sweep(Lo, b), Port.lower_solve(Lo, b))
    s.replan(parts=4, partition=PARTITION_CUSTOM)  # keeps the map
    assert np.array_equal(s.emulate_sweep(Lo, b), Port.lower_solve(Lo, b))


@pytest.mark.parametrize("mapping", [1, 2, 3, 4])
def test_scheduler_mapping_thread_partition_plan(mapping):
    """CTA t runs virtual thread t of the Scheduler's P2P (cost split per merged level, both task
    layouts), P2P_TIME or P2P_MAPPING mapping."""
    A = gen.laplace3d(10, 1e-3)
    Lo, Up = _ic_lu(A)
    s = Schedule(A, kind=KERNEL_ICCG, nthread=12, partition=PARTITION_BAAS_THREADS, mapping=mapping)
    r = gen.uniform_rhs(A.n, 1)
    assert np.array_equal(s.emulate_sweep(Lo, r), Port.lower_solve(Lo, r))
    assert np.array_equal(s.emulate_sweep(Up, r, upper=True), Port.upper_solve(Up, r, descending=True))


def test_batch_schedule_replan_keeps_analysis():
    """BatchSchedule.replan (the autotuner's call) rebuilds only the device plan."""
    from baas_b200 import BatchSchedule

    bs = BatchSchedule([gen.laplace2d(8), gen.vardiff2d(10, seed=1)], parts=3)
    bs.replan(parts=2, smem_budget=64 * 1024)
    bs.replan(parts=3)
