"""GPU parity of the sweeps and factorisations against the oracle (bit-exact: the CUDA path
follows the reference's operation order with correctly rounded FP64 operations)."""
import numpy as np
import pytest

from baas_b200 import (KERNEL_IC0, KERNEL_ICCG, KERNEL_ILU0, KERNEL_SPTRSV, BaasError, DeviceCSR, Schedule, gen)
from oracle.oracle import Port

pytestmark = pytest.mark.gpu


def _t(a):
    import torch

    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _ic_factors(A):
    """Split an IC0 factor (lu on A's pattern) into L (diagonal last) and U = L^T (diagonal
    first), as IC0_preconditioner does (test/iccg_level_merge.cpp:874-891)."""
    lu, _ = Port.ic0(A)
    Lo = gen.CSR(A.n, A.rowptr, A.colidx, lu).lower()
    Up = gen.from_scipy(Lo.to_scipy().T.tocsr())
    return Lo, Up


@pytest.mark.parametrize("k,nthread", [(16, 1), (32, 4), (128, 8)])
def test_forward_sweep_c1_bitexact(k, nthread):
    L, x_true, b = gen.sptrsv_case(k, 0)
    s = Schedule(L, kind=KERNEL_SPTRSV, nthread=nthread)
    x = _t(np.zeros(L.n))
    s.forward(DeviceCSR.from_host(L), _t(b), x)
    got = x.cpu().numpy()
    want = Port.lower_solve(L, b)
    assert np.array_equal(got, want)
    assert np.max(np.abs(got - x_true)) < 1e-12


@pytest.mark.parametrize("kind", [KERNEL_ICCG, KERNEL_IC0])
def test_ic_sweeps_bitexact(kind):
    A = gen.laplace3d(12, 1e-3)
    Lo, Up = _ic_factors(A)
    s = Schedule(A, kind=kind, nthread=8)
    r = gen.uniform_rhs(A.n, 1)
    y = _t(np.zeros(A.n))
    z = _t(np.zeros(A.n))
    s.forward(DeviceCSR.from_host(Lo), _t(r), y)
    s.backward(DeviceCSR.from_host(Up), y, z)
    ywant = Port.lower_solve(Lo, r)
    zwant = Port.upper_solve(Up, ywant, descending=True)
    assert np.array_equal(y.cpu().numpy(), ywant)
    assert np.array_equal(z.cpu().numpy(), zwant)


def test_multi_rhs_sweep():
    A = gen.laplace3d(10, 1e-3)
    Lo, Up = _ic_factors(A)
    s = Schedule(A, kind=KERNEL_ICCG, nthread=4)
    B = gen.normal_rhs(A.n, 2, nrhs=8)
    X = _t(np.zeros_like(B))
    s.forward(DeviceCSR.from_host(Lo), _t(B), X)
    got = X.cpu().numpy()
    for r in range(8):
        assert np.array_equal(got[r], Port.lower_solve(Lo, B[r]))


def test_ic0_bitexact():
    A = gen.laplace3d(16, 1e-3)
    s = Schedule(A, kind=KERNEL_IC0, nthread=8)
    dA = DeviceCSR.from_host(A)
    lu = dA.values.clone()
    s.ic0(dA, lu)
    want, bad = Port.ic0(A)
    assert bad == 0
    assert np.array_equal(lu.cpu().numpy(), want)


def test_ic0_knn_bitexact():
    A = gen.knn_stiffness(nodes=800, k=12, seed=3)
    s = Schedule(A, kind=KERNEL_ICCG, nthread=8)
    dA = DeviceCSR.from_host(A)
    lu = dA.values.clone()
    s.ic0(dA, lu)
    want, _ = Port.ic0(A)
    assert np.array_equal(lu.cpu().numpy(), want)


def test_ilu0_bitexact():
    A = gen.convdiff3d(14)
    s = Schedule(A, kind=KERNEL_ILU0, nthread=8)
    dA = DeviceCSR.from_host(A)
    lu = dA.values.clone()
    s.ilu0(dA, lu)
    want, bad = Port.ilu0(A)
    assert bad == 0
    assert np.array_equal(lu.cpu().numpy(), want)


def test_ic0_nonpositive_pivot_status():
    # an indefinite matrix: IC0 leaves the offending diagonals unchanged (merge/IC.cpp:371-378)
    # and the library reports it; the factor still equals the oracle's
    A = gen.laplace2d(8, diag=1.0)
    s = Schedule(A, kind=KERNEL_IC0, nthread=2)
    dA = DeviceCSR.from_host(A)
    lu = dA.values.clone()
    with pytest.raises(BaasError) as e:
        s.ic0(dA, lu)
    assert e.value.status_name == "BAAS_ERR_ZERO_PIVOT"
    want, bad = Port.ic0(A)
    assert bad > 0
    assert np.array_equal(lu.cpu().numpy(), want)
