"""The fetch walk on the GPU (stencil rows, one right-hand side): it must be the walk that runs
by default on these systems, and every result must be bit-identical to the chunked walk's on the
same partition and, for the sweeps, to the oracle's."""
import numpy as np
import pytest

from baas_b200 import (KERNEL_ICCG, KERNEL_SPTRSV, PARTITION_BLOCKS, PREC_FP32_FACTORS, PREC_FP64, WALK_CHUNKED,
                       WALK_FETCH, WALK_SMALL, BaasError, DeviceCSR, Schedule, gen)
from oracle.oracle import Port

pytestmark = pytest.mark.gpu


def _t(a):
    import torch

    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _ic_lu(A):
    lu, _ = Port.ic0(A)
    Lo = gen.CSR(A.n, A.rowptr, A.colidx, lu).lower()
    return Lo, Lo.transpose()


@pytest.mark.parametrize("parts", [8, 16, 0])
def test_c1_sweep_fetch_walk(parts):
    L, _, b = gen.sptrsv_case(128, 0)
    s = Schedule(L, kind=KERNEL_SPTRSV, nthread=8, parts=parts)
    x = _t(np.zeros(L.n))
    s.forward(DeviceCSR.from_host(L), _t(b), x)
    assert s.last_walk == WALK_FETCH
    assert np.array_equal(x.cpu().numpy(), Port.lower_solve(L, b))


@pytest.mark.parametrize("k", [24, 64])
def test_ic_sweeps_both_directions(k):
    A = gen.laplace3d(k, 1e-3)
    Lo, Up = _ic_lu(A)
    r = gen.uniform_rhs(A.n, 1)
    s = Schedule(A, kind=KERNEL_ICCG, nthread=8)
    y, z = _t(np.zeros(A.n)), _t(np.zeros(A.n))
    s.forward(DeviceCSR.from_host(Lo), _t(r), y)
    assert s.last_walk == WALK_FETCH
    s.backward(DeviceCSR.from_host(Up), _t(r), z)
    assert np.array_equal(y.cpu().numpy(), Port.lower_solve(Lo, r))
    assert np.array_equal(z.cpu().numpy(), Port.upper_solve(Up, r, descending=True))


@pytest.mark.parametrize("precision", [PREC_FP64, PREC_FP32_FACTORS])
@pytest.mark.parametrize("k", [16, 64])
def test_iccg_fetch_walk_bitexact_vs_chunked(k, precision):
    A = gen.laplace3d(k, 1e-3)
    b = gen.uniform_rhs(A.n, 1)
    dA, db = DeviceCSR.from_host(A), _t(b)
    out = {}
    # the same grid-box partition for both walks: the ICCG sums its dot products CTA by CTA, so
    # its iterates depend on the partition in the last bits (its sweeps and factor do not)
    for walk in (0, WALK_CHUNKED):
        s = Schedule(A, kind=KERNEL_ICCG, nthread=8, walk=walk, partition=PARTITION_BLOCKS)
        x = _t(np.zeros(A.n))
        it, rel = s.iccg(dA, db, x, tol=1e-10, maxiter=2000, precision=precision)
        assert s.last_walk == (WALK_FETCH if walk == 0 else WALK_CHUNKED)
        out[walk] = (it, rel, x.cpu().numpy())
    assert out[0][0] == out[WALK_CHUNKED][0]
    assert out[0][1] == out[WALK_CHUNKED][1]
    assert np.array_equal(out[0][2], out[WALK_CHUNKED][2])


def test_adjoint_fetch_walk_bitexact_vs_chunked():
    A = gen.laplace3d(12, 1e-3)
    b = gen.uniform_rhs(A.n, 1)
    g = gen.uniform_rhs(A.n, 3)
    dA = DeviceCSR.from_host(A)
    out = {}
    for walk in (0, WALK_CHUNKED):
        s = Schedule(A, kind=KERNEL_ICCG, nthread=8, walk=walk, partition=PARTITION_BLOCKS)
        x = _t(np.zeros(A.n))
        s.iccg(dA, _t(b), x, tol=1e-10, precision=PREC_FP32_FACTORS)
        lam = _t(np.zeros(A.n))
        s.iccg_adjoint(dA, _t(g), lam, tol=1e-10, precision=PREC_FP32_FACTORS)
        out[walk] = lam.cpu().numpy()
    assert np.array_equal(out[0], out[WALK_CHUNKED])


def test_forced_fetch_walk_refuses_wide_rows():
    A = gen.knn_stiffness(nodes=400, k=12, seed=3)
    s = Schedule(A, kind=KERNEL_ICCG, nthread=8, walk=WALK_FETCH)
    x = _t(np.zeros(A.n))
    with pytest.raises(BaasError, match="fetch walk"):
        s.iccg(DeviceCSR.from_host(A), _t(gen.uniform_rhs(A.n, 1)), x)
    s2 = Schedule(A, kind=KERNEL_ICCG, nthread=8)  # automatic: a small shallow system takes one CTA
    it, rel = s2.iccg(DeviceCSR.from_host(A), _t(gen.uniform_rhs(A.n, 1)), x)
    assert s2.last_walk == WALK_SMALL and rel < 1e-10


def test_fetch_walk_timeout_leaves_context_usable():
    L, _, b = gen.sptrsv_case(32, 0)
    dL = DeviceCSR.from_host(L)
    s = Schedule(L, kind=KERNEL_SPTRSV, nthread=2, spin_limit=1 << 14, parts=4, walk=WALK_FETCH)
    s.inject_unsatisfiable_wait(300)  # the row then waits, through the fetcher, on its own result
    x = _t(np.zeros(L.n))
    with pytest.raises(BaasError) as e:
        s.forward(dL, _t(b), x)
    assert e.value.status_name == "BAAS_ERR_TIMEOUT"
    s2 = Schedule(L, kind=KERNEL_SPTRSV, nthread=2, parts=4, walk=WALK_FETCH)
    x2 = _t(np.zeros(L.n))
    s2.forward(dL, _t(b), x2)
    assert np.array_equal(x2.cpu().numpy(), Port.lower_solve(L, b))
