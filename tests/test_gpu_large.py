"""GPU parity at full configuration sizes and with the plan streamed through shared memory.

* ILU0 of the 96^3 upwind convection-diffusion operator (n = 884,736) and the preconditioner
  apply on 8 right-hand sides (forward sweep on the unit lower factor, backward sweep on U),
  bit-exact against the oracle.
* A small shared-memory budget forces every CTA to stream its plan window by window (two
  buffers fed by bulk copies); sweeps and ICCG must stay bit-exact / iteration-exact.
"""
import numpy as np
import pytest
import scipy.sparse as sp

from baas_b200 import KERNEL_ICCG, KERNEL_ILU0, KERNEL_SPTRSV, DeviceCSR, Schedule, gen
from oracle.oracle import Port

pytestmark = pytest.mark.gpu


def _t(a):
    import torch

    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _ilu_factors(C, lu):
    """Unit lower L (strict lower part of lu, diagonal 1, diagonal last) and U (upper part of lu
    including the diagonal, diagonal first)."""
    M = gen.CSR(C.n, C.rowptr, C.colidx, lu).to_scipy()
    Lo = gen.from_scipy(sp.tril(M, k=-1) + sp.identity(C.n, format="csr"))
    Up = gen.from_scipy(sp.triu(M))
    return Lo, Up


def test_c3_ilu0_96_and_apply_8rhs():
    C = gen.convdiff3d(96)
    assert C.n == 884_736 and C.nnz == 6_137_856
    s = Schedule(C, kind=KERNEL_ILU0, nthread=8)
    dC = DeviceCSR.from_host(C)
    lu = dC.values.clone()
    s.ilu0(dC, lu)
    want, bad = Port.ilu0(C)
    assert bad == 0
    got = lu.cpu().numpy()
    assert np.array_equal(got, want)

    Lo, Up = _ilu_factors(C, want)
    B = gen.normal_rhs(C.n, 2, nrhs=8)
    Y = _t(np.zeros_like(B))
    Z = _t(np.zeros_like(B))
    s.forward(DeviceCSR.from_host(Lo), _t(B), Y)
    s.backward(DeviceCSR.from_host(Up), Y, Z)
    y = Y.cpu().numpy()
    z = Z.cpu().numpy()
    for r in (0, 3, 7):
        yw = Port.lower_solve(Lo, B[r])
        assert np.array_equal(y[r], yw)
        assert np.array_equal(z[r], Port.upper_solve(Up, yw, descending=True))


@pytest.mark.parametrize("budget", [24 * 1024, 40 * 1024])
def test_streamed_windows_sweeps_bitexact(budget):
    A = gen.laplace3d(24, 1e-3)
    lu, _ = Port.ic0(A)
    Lo = gen.CSR(A.n, A.rowptr, A.colidx, lu).lower()
    Up = Lo.transpose()
    s = Schedule(A, kind=KERNEL_ICCG, nthread=8, parts=8, smem_budget=budget)
    r = gen.uniform_rhs(A.n, 1)
    y = _t(np.zeros(A.n))
    z = _t(np.zeros(A.n))
    s.forward(DeviceCSR.from_host(Lo), _t(r), y)
    s.backward(DeviceCSR.from_host(Up), y, z)
    yw = Port.lower_solve(Lo, r)
    assert np.array_equal(y.cpu().numpy(), yw)
    assert np.array_equal(z.cpu().numpy(), Port.upper_solve(Up, yw, descending=True))
    # multi-right-hand-side walk, also streamed
    B = gen.normal_rhs(A.n, 2, nrhs=5)
    X = _t(np.zeros_like(B))
    s.forward(DeviceCSR.from_host(Lo), _t(B), X)
    got = X.cpu().numpy()
    for k in range(5):
        assert np.array_equal(got[k], Port.lower_solve(Lo, B[k]))


def test_streamed_windows_iccg():
    A = gen.laplace3d(24, 1e-3)
    b = gen.uniform_rhs(A.n, 1)
    xw, itw, relw = Port.pcg(A, b, tol=1e-10)
    dA = DeviceCSR.from_host(A)
    for budget in (24 * 1024, 0):
        s = Schedule(A, kind=KERNEL_ICCG, nthread=8, parts=8, smem_budget=budget)
        for prec in (0, 1):
            x = _t(np.zeros(A.n))
            it, rel = s.iccg(dA, _t(b), x, tol=1e-10, precision=prec)
            assert abs(it - itw) <= 1
            assert rel < 1e-10
            err = np.linalg.norm(x.cpu().numpy() - xw) / np.linalg.norm(xw)
            assert err <= (1e-12 if prec == 0 else 1e-9)


def test_c1_single_cta_and_wide_steps():
    """One CTA owns all rows; the first levels are wider than a chunk may hold."""
    L, x_true, b = gen.sptrsv_case(128, 0)
    s = Schedule(L, kind=KERNEL_SPTRSV, nthread=8, parts=1)
    x = _t(np.zeros(L.n))
    s.forward(DeviceCSR.from_host(L), _t(b), x)
    assert np.array_equal(x.cpu().numpy(), Port.lower_solve(L, b))
