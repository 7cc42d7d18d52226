"""GPU parity at the full sizes the benchmark runs: configuration 2 (IC0 + ICCG on the 64^3
7-point Laplacian with shift 1e-3, in natural order and under the seeded random symmetric
permutation) and its third input, the 3-dof k-NN stiffness matrix at n = 12,000.

Against the oracle (oracle/baas_oracle.c, pinned to the reference's own outputs):
  * the IC0 factor bit for bit (spic0_csr_uL_serial, merge/IC.cpp:32-89);
  * one forward and one backward sweep of that factor bit for bit (merge/SpTRSV.cpp:24-39,
    601-660);
  * ICCG in FP64: iterations within +-1 of the pcg loop's (test/iccg_level_merge.cpp:698-807,
    break at 1e-10) and the solution within 1e-12 relative. The iterates differ only in the
    summation order of the dot products (the oracle sums sequentially, the kernel in a fixed
    tree), so the bound is a few hundred ulps of accumulated CG rounding;
  * ICCG with FP32 factors: the solution against the FP64 oracle's, within 1e-9 relative.
"""
import numpy as np
import pytest

from baas_b200 import KERNEL_ICCG, PREC_FP32_FACTORS, PREC_FP64, DeviceCSR, Schedule, gen
from oracle.oracle import Port

pytestmark = pytest.mark.gpu

CASES = {
    "c2_natural": lambda: gen.c2_system(False),
    "c2_permuted": lambda: gen.c2_system(True),
    "c2_knn_12000": lambda: gen.knn_stiffness(nodes=4000),
}
FP64_TOL = 1e-12   # x vs the oracle's x, relative 2-norm
FP32_TOL = 1e-9    # FP32-factor x vs the FP64 oracle's x


_cache = {}


def _case(name):
    if name not in _cache:
        A = CASES[name]()
        b = gen.uniform_rhs(A.n, gen.C2_RHS_SEED)
        lu, bad = Port.ic0(A)
        xo, ito, relo = Port.pcg(A, b, tol=1e-10, maxiter=2000)
        _cache[name] = (A, b, lu, bad, xo, ito, relo)
    return _cache[name]


def _t(a):
    import torch

    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.mark.parametrize("name", list(CASES))
def test_ic0_and_sweeps_bitexact(name):
    A, b, lu_want, bad, *_ = _case(name)
    assert bad == 0
    s = Schedule(A, kind=KERNEL_ICCG, nthread=8)
    dA = DeviceCSR.from_host(A)
    lu = dA.values.clone()
    s.ic0(dA, lu)
    assert np.array_equal(lu.cpu().numpy(), lu_want)
    Lo = gen.CSR(A.n, A.rowptr, A.colidx, lu_want).lower()
    Up = Lo.transpose()
    y = _t(np.zeros(A.n))
    z = _t(np.zeros(A.n))
    s.forward(DeviceCSR.from_host(Lo), _t(b), y)
    s.backward(DeviceCSR.from_host(Up), y, z)
    yw = Port.lower_solve(Lo, b)
    assert np.array_equal(y.cpu().numpy(), yw)
    assert np.array_equal(z.cpu().numpy(), Port.upper_solve(Up, yw, descending=True))


@pytest.mark.parametrize("name", list(CASES))
def test_iccg_fp64_vs_oracle(name):
    A, b, _, _, xo, ito, relo = _case(name)
    assert relo < 1e-10
    s = Schedule(A, kind=KERNEL_ICCG, nthread=8)
    x = _t(np.zeros(A.n))
    it, rel = s.iccg(DeviceCSR.from_host(A), _t(b), x, tol=1e-10, maxiter=2000, precision=PREC_FP64)
    err = _rel(x.cpu().numpy(), xo)
    print(f"{name}: iterations {it} (oracle {ito}), relres {rel:.3e}, x rel err vs oracle {err:.3e}")
    assert abs(it - ito) <= 1
    assert rel < 1e-10
    assert err <= FP64_TOL


@pytest.mark.parametrize("name", list(CASES))
def test_iccg_fp32_factors_vs_fp64_oracle(name):
    A, b, _, _, xo, ito, _ = _case(name)
    s = Schedule(A, kind=KERNEL_ICCG, nthread=8)
    x = _t(np.zeros(A.n))
    it, rel = s.iccg(DeviceCSR.from_host(A), _t(b), x, tol=1e-10, maxiter=2000, precision=PREC_FP32_FACTORS)
    err = _rel(x.cpu().numpy(), xo)
    print(f"{name} FP32 factors: iterations {it} (FP64 oracle {ito}), relres {rel:.3e}, x rel err {err:.3e}")
    assert rel < 1e-10
    assert it <= ito + max(3, ito // 10)
    assert err <= FP32_TOL
