"""The analysis's data-parallel stages on the GPU (BAAS_ANALYSIS_DEVICE, baas_b200/csrc/analysis.cu):
transposes, the two-hop reduction, the group DAGs and the level sets run as CUDA kernels while the
BFS coarsenings and mappings stay on the host. The schedule must be the host analysis's, array for
array -- every field the reference exports plus the final group DAG the device plans are built
from -- on the benchmark's matrices at full size, under every mapping, and on patterns whose
shape stresses one stage (a dense first row and column, a diagonal-only matrix, a chain)."""
import numpy as np
import pytest

from baas_b200 import (ANALYSIS_DEVICE, KERNEL_ICCG, KERNEL_ILU0, KERNEL_SPTRSV, BatchSchedule, Schedule, gen)
from baas_b200._native import FIELDS, GROUP_DAG_FIELDS

pytestmark = pytest.mark.gpu

ALL = list(FIELDS) + list(GROUP_DAG_FIELDS)


def _same(a, b, what):
    for f in ALL:
        x, y = a.export(f), b.export(f)
        assert np.array_equal(x, y), f"{what}: field {f}"


def _arrow(n):
    """Row 0 couples to every row: one column of the lower DAG holds n entries."""
    rows = [[0] + list(range(1, n))] + [[0, i] for i in range(1, n)]
    rowptr = np.zeros(n + 1, dtype=np.int32)
    rowptr[1:] = np.cumsum([len(r) for r in rows])
    colidx = np.concatenate(rows).astype(np.int32)
    return gen.CSR(n, rowptr, colidx, np.ones(colidx.size))


def _diagonal(n):
    return gen.CSR(n, np.arange(n + 1, dtype=np.int32), np.arange(n, dtype=np.int32), np.ones(n))


def _tridiag(n):
    cols = [[j for j in (i - 1, i, i + 1) if 0 <= j < n] for i in range(n)]
    rowptr = np.zeros(n + 1, dtype=np.int32)
    rowptr[1:] = np.cumsum([len(c) for c in cols])
    colidx = np.concatenate(cols).astype(np.int32)
    return gen.CSR(n, rowptr, colidx, np.ones(colidx.size))


FULL = [
    ("c2_natural_64", KERNEL_ICCG, lambda: gen.c2_system(False), (8, 16)),
    ("c2_permuted_64", KERNEL_ICCG, lambda: gen.c2_system(True), (8,)),
    ("c2_knn_12000", KERNEL_ICCG, lambda: gen.knn_stiffness(nodes=4000), (8,)),
    ("c3_ilu0_96", KERNEL_ILU0, lambda: gen.convdiff3d(96), (8,)),
    ("c1_lower_128", KERNEL_SPTRSV, lambda: gen.laplace2d(128).lower(), (1, 8)),
]


@pytest.mark.parametrize("case", [c[0] for c in FULL])
def test_device_analysis_equals_host_at_full_size(case):
    _, kind, mk, threads = next(c for c in FULL if c[0] == case)
    A = mk()
    for nt in threads:
        h = Schedule(A, kind=kind, nthread=nt)
        d = Schedule(A, kind=kind, nthread=nt, analysis=ANALYSIS_DEVICE)
        _same(h, d, f"{case} nthread={nt}")
        assert d.analysis_ms > 0


@pytest.mark.parametrize("mapping", [1, 2, 3, 4])
def test_device_analysis_under_every_mapping(mapping):
    for A in (gen.laplace3d(12, 1e-3), gen.knn_stiffness(nodes=600, k=12, seed=3)):
        for nt in (3, 8):
            h = Schedule(A, kind=KERNEL_ICCG, nthread=nt, mapping=mapping)
            d = Schedule(A, kind=KERNEL_ICCG, nthread=nt, mapping=mapping, analysis=ANALYSIS_DEVICE)
            _same(h, d, f"mapping={mapping} nthread={nt}")


@pytest.mark.parametrize("name,mk", [("arrow", lambda: _arrow(3000)), ("diagonal", lambda: _diagonal(1000)),
                                     ("chain", lambda: _tridiag(5000)), ("one_row", lambda: _diagonal(1))])
def test_device_analysis_on_edge_patterns(name, mk):
    A = mk()
    for kind in (KERNEL_ICCG, KERNEL_ILU0):
        h = Schedule(A, kind=kind, nthread=4)
        d = Schedule(A, kind=kind, nthread=4, analysis=ANALYSIS_DEVICE)
        _same(h, d, f"{name} kind={kind}")


def test_device_analysis_of_a_batch():
    systems = gen.batch_vardiff2d(nsys=8, kmin=64, kmax=128)
    h = BatchSchedule(systems, nthread=8)
    d = BatchSchedule(systems, nthread=8, analysis=ANALYSIS_DEVICE)
    _same(h, d, "batch of 8")


def test_device_analysed_schedule_solves_like_the_host_one():
    import torch

    from baas_b200 import DeviceCSR

    A = gen.laplace3d(24, 1e-3)
    b = torch.from_numpy(gen.uniform_rhs(A.n, 7)).cuda()
    out = []
    for analysis in (0, ANALYSIS_DEVICE):
        s = Schedule(A, kind=KERNEL_ICCG, nthread=8, analysis=analysis)
        dA = DeviceCSR.from_host(A)
        x = torch.zeros_like(b)
        it, rel = s.iccg(dA, b, x, tol=1e-10, maxiter=500)
        out.append((it, x.cpu().numpy()))
    assert out[0][0] == out[1][0]
    assert np.array_equal(out[0][1], out[1][1])


@pytest.mark.parametrize("ablation", [1, 2, 3])
def test_device_analysis_of_ablation_schedules(ablation):
    L = gen.laplace2d(128).lower()
    for nt in (1, 8):
        h = Schedule(L, kind=KERNEL_SPTRSV, nthread=nt, ablation=ablation)
        d = Schedule(L, kind=KERNEL_SPTRSV, nthread=nt, ablation=ablation, analysis=ANALYSIS_DEVICE)
        _same(h, d, f"ablation={ablation} nthread={nt}")
