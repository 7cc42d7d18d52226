"""GPU ICCG (one persistent kernel: IC0 + PCG loop) against the oracle's pcg_opt loop."""
import numpy as np
import pytest

from baas_b200 import KERNEL_ICCG, PREC_FP32_FACTORS, PREC_FP64, DeviceCSR, Schedule, gen
from oracle.oracle import Port

pytestmark = pytest.mark.gpu


def _t(a):
    import torch

    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


@pytest.mark.parametrize("k", [12, 24])
def test_iccg_matches_oracle(k):
    A = gen.laplace3d(k, 1e-3)
    b = gen.uniform_rhs(A.n, 1)
    s = Schedule(A, kind=KERNEL_ICCG, nthread=8)
    x = _t(np.zeros(A.n))
    it, rel = s.iccg(DeviceCSR.from_host(A), _t(b), x, tol=1e-10, maxiter=2000)
    xo, ito, relo = Port.pcg(A, b, tol=1e-10)
    assert abs(it - ito) <= 1
    assert rel < 1e-10
    xg = x.cpu().numpy()
    # both iterates converge to the same solution; the dot products differ only in summation order
    assert np.linalg.norm(xg - xo) / np.linalg.norm(xo) <= 1e-12
    res = np.linalg.norm(b - A.to_scipy() @ xg) / np.linalg.norm(b)
    assert res < 1e-9


def test_iccg_fp32_factors():
    A = gen.laplace3d(20, 1e-3)
    b = gen.uniform_rhs(A.n, 1)
    s = Schedule(A, kind=KERNEL_ICCG, nthread=8)
    x = _t(np.zeros(A.n))
    it, rel = s.iccg(DeviceCSR.from_host(A), _t(b), x, tol=1e-10, maxiter=2000, precision=PREC_FP32_FACTORS)
    xo, ito, _ = Port.pcg(A, b, tol=1e-10)
    assert rel < 1e-10
    assert it <= ito + max(3, ito // 10)
    xg = x.cpu().numpy()
    assert np.linalg.norm(xg - xo) / np.linalg.norm(xo) <= 1e-9  # FP32 factors vs the FP64 oracle


def test_iccg_knn_stiffness():
    A = gen.knn_stiffness(nodes=1000, k=12, seed=3)
    b = gen.uniform_rhs(A.n, 1)
    s = Schedule(A, kind=KERNEL_ICCG, nthread=8)
    x = _t(np.zeros(A.n))
    it, rel = s.iccg(DeviceCSR.from_host(A), _t(b), x, tol=1e-10, maxiter=2000, precision=PREC_FP64)
    xo, ito, _ = Port.pcg(A, b, tol=1e-10)
    assert abs(it - ito) <= 1
    assert np.linalg.norm(x.cpu().numpy() - xo) / np.linalg.norm(xo) <= 1e-12


def test_iccg_repeat_and_permuted():
    A = gen.laplace3d(16, 1e-3)
    P = A.permuted(gen.random_symmetric_permutation(A.n, 5))
    b = gen.uniform_rhs(A.n, 1)
    for M in (A, P):
        s = Schedule(M, kind=KERNEL_ICCG, nthread=8)
        dA = DeviceCSR.from_host(M)
        xo, ito, _ = Port.pcg(M, b, tol=1e-10)
        for _ in range(2):  # a second call reuses the workspace and a new flag epoch
            x = _t(np.zeros(M.n))
            it, rel = s.iccg(dA, _t(b), x, tol=1e-10)
            assert abs(it - ito) <= 1 and rel < 1e-10
