"""The level walk on the GPU (shallow group DAGs: a k-NN stiffness matrix, the 24^3 system under a
random symmetric permutation): its sweeps equal the oracle's bit for bit, and its ICCG matches the
oracle's PCG and the chunked walk's. (Systems this small fit the single-CTA walk, which the
automatic choice prefers; the level walk is asked for by name.)"""
import numpy as np
import pytest

from baas_b200 import KERNEL_ICCG, PREC_FP32_FACTORS, PREC_FP64, WALK_CHUNKED, WALK_LEVELS, DeviceCSR, Schedule, gen
from oracle.oracle import Port

pytestmark = pytest.mark.gpu


def _t(a):
    import torch

    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _ic_lu(A):
    lu, _ = Port.ic0(A)
    Lo = gen.CSR(A.n, A.rowptr, A.colidx, lu).lower()
    return Lo, Lo.transpose()


def _cases():
    return {"knn": gen.knn_stiffness(nodes=4000, k=12, seed=3),
            "permuted24": gen.laplace3d(24, 1e-3).permuted(gen.random_symmetric_permutation(24 ** 3, 7))}


@pytest.mark.parametrize("name", ["knn", "permuted24"])
def test_level_walk_sweeps_bitexact(name):
    A = _cases()[name]
    Lo, Up = _ic_lu(A)
    r = gen.uniform_rhs(A.n, 1)
    s = Schedule(A, kind=KERNEL_ICCG, nthread=8, walk=WALK_LEVELS)
    y, z = _t(np.zeros(A.n)), _t(np.zeros(A.n))
    s.forward(DeviceCSR.from_host(Lo), _t(r), y)
    assert s.last_walk == WALK_LEVELS
    s.backward(DeviceCSR.from_host(Up), _t(r), z)
    assert np.array_equal(y.cpu().numpy(), Port.lower_solve(Lo, r))
    assert np.array_equal(z.cpu().numpy(), Port.upper_solve(Up, r, descending=True))


@pytest.mark.parametrize("precision", [PREC_FP64, PREC_FP32_FACTORS])
@pytest.mark.parametrize("name", ["knn", "permuted24"])
def test_level_walk_iccg(name, precision):
    A = _cases()[name]
    b = gen.uniform_rhs(A.n, 1)
    xo, ito, _ = Port.pcg(A, b, tol=1e-10)
    dA = DeviceCSR.from_host(A)
    got = {}
    for walk in (WALK_LEVELS, WALK_CHUNKED):
        s = Schedule(A, kind=KERNEL_ICCG, nthread=8, walk=walk)
        x = _t(np.zeros(A.n))
        it, rel = s.iccg(dA, _t(b), x, tol=1e-10, maxiter=2000, precision=precision)
        assert s.last_walk == walk
        assert rel < 1e-10
        got[walk] = (it, x.cpu().numpy())
    it, xg = got[WALK_LEVELS]
    tol = 1e-12 if precision == PREC_FP64 else 1e-9
    assert abs(it - ito) <= (1 if precision == PREC_FP64 else max(3, ito // 10))
    assert np.linalg.norm(xg - xo) / np.linalg.norm(xo) <= tol
    # the walks agree to the last bits of the dot products' summation order
    assert np.linalg.norm(xg - got[WALK_CHUNKED][1]) / np.linalg.norm(xo) <= tol


@pytest.mark.parametrize("k", [14, 40])
def test_level_walk_ilu0_bitexact(k):
    """ILU0 by the level walk's plan (k_ilu0_levels: grid barrier per group level, no flags) gives
    the oracle's factor bit for bit (merge/ILU.cpp:350-386)."""
    from baas_b200 import KERNEL_ILU0

    A = gen.convdiff3d(k)
    s = Schedule(A, kind=KERNEL_ILU0, nthread=8, walk=WALK_LEVELS)
    dA = DeviceCSR.from_host(A)
    lu = dA.values.clone()
    s.ilu0(dA, lu)
    want, bad = Port.ilu0(A)
    assert bad == 0
    assert np.array_equal(lu.cpu().numpy(), want)
