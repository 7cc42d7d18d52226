"""The single-CTA walk (BAAS_WALK_SMALL, baas_b200/csrc/small.cuh) on the GPU: one CTA, or one
thread-block cluster whose CTAs each hold the sweep's full solution in shared memory, walks the row
levels with a barrier per level.

  * forward and backward sweeps bit for bit against the oracle (merge/SpTRSV.cpp:24-39, 642-652),
    on a stencil's lower triangle, its transpose, and a k-NN stiffness matrix's IC0 factor;
  * IC0 bit for bit against the oracle (merge/IC.cpp:32-89);
  * ICCG against the oracle's PCG: iterations within one, the solution within 1e-12 relative
    (FP64) / 1e-9 (FP32 factors); the walk is the one the library picks for the k-NN system;
  * the adjoint solve and its gradient against the chunked walk's;
  * a system too large for one CTA's shared memory is refused when the walk is forced;
  * every cluster size (1, 2, 4, 8, 16) gives the same factor and sweeps; the walk autotuner
    (autotune.tune_walk) leaves the schedule on its fastest candidate.
"""
import numpy as np
import pytest

from baas_b200 import (KERNEL_ICCG, KERNEL_SPTRSV, PREC_FP32_FACTORS, PREC_FP64, WALK_CHUNKED, WALK_SMALL, BaasError,
                       DeviceCSR, Schedule, gen)
from oracle.oracle import Port

pytestmark = pytest.mark.gpu


def _t(a):
    import torch

    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def test_stencil_sweeps_bitexact():
    L, _, b = gen.sptrsv_case(128, 0)
    s = Schedule(L, kind=KERNEL_SPTRSV, nthread=8, walk=WALK_SMALL)
    x = _t(np.zeros(L.n))
    s.sptrsv(DeviceCSR.from_host(L), _t(b), x, upper=False)
    assert s.last_walk == WALK_SMALL
    assert np.array_equal(x.cpu().numpy(), Port.lower_solve(L, b))
    U = L.transpose()
    s.sptrsv(DeviceCSR.from_host(U), _t(b), x, upper=True)
    assert np.array_equal(x.cpu().numpy(), Port.upper_solve(U, b, descending=True))


@pytest.mark.parametrize("nodes", [800, 4000])
def test_knn_ic0_and_sweeps_bitexact(nodes):
    A = gen.knn_stiffness(nodes=nodes, k=12, seed=3)
    s = Schedule(A, kind=KERNEL_ICCG, nthread=8, walk=WALK_SMALL)
    dA = DeviceCSR.from_host(A)
    lu = dA.values.clone()
    s.ic0(dA, lu)
    want, bad = Port.ic0(A)
    assert bad == 0
    assert np.array_equal(lu.cpu().numpy(), want)
    Lo = gen.CSR(A.n, A.rowptr, A.colidx, want).lower()
    Up = Lo.transpose()
    r = gen.uniform_rhs(A.n, 2)
    y, z = _t(np.zeros(A.n)), _t(np.zeros(A.n))
    s.forward(DeviceCSR.from_host(Lo), _t(r), y)
    s.backward(DeviceCSR.from_host(Up), y, z)
    yw = Port.lower_solve(Lo, r)
    assert np.array_equal(y.cpu().numpy(), yw)
    assert np.array_equal(z.cpu().numpy(), Port.upper_solve(Up, yw, descending=True))


@pytest.mark.parametrize("precision", [PREC_FP64, PREC_FP32_FACTORS])
def test_knn_iccg_against_the_oracle(precision):
    A = gen.knn_stiffness(nodes=4000)
    b = gen.uniform_rhs(A.n, gen.C2_RHS_SEED)
    xo, ito, _ = Port.pcg(A, b, tol=1e-10, maxiter=2000)
    s = Schedule(A, kind=KERNEL_ICCG, nthread=8)  # automatic choice
    dA = DeviceCSR.from_host(A)
    x = _t(np.zeros(A.n))
    it, rel = s.iccg(dA, _t(b), x, tol=1e-10, maxiter=2000, precision=precision)
    assert s.last_walk == WALK_SMALL
    assert rel < 1e-10
    xg = x.cpu().numpy()
    if precision == PREC_FP64:
        assert abs(it - ito) <= 1
        assert np.linalg.norm(xg - xo) / np.linalg.norm(xo) <= 1e-12
    else:
        assert abs(it - ito) <= max(3, ito // 10)
        assert np.linalg.norm(xg - xo) / np.linalg.norm(xo) <= 1e-9
    # a second solve reuses nothing it should not: same iterations, same solution
    x2 = _t(np.zeros(A.n))
    it2, _ = s.iccg(dA, _t(b), x2, tol=1e-10, maxiter=2000, precision=precision)
    assert it2 == it and np.array_equal(x2.cpu().numpy(), xg)


def test_adjoint_small_walk_against_chunked():
    import torch

    A = gen.knn_stiffness(nodes=1000, k=12, seed=3)
    dA = DeviceCSR.from_host(A)
    b = gen.uniform_rhs(A.n, 4)
    g = gen.uniform_rhs(A.n, 5)
    out = {}
    for walk in (WALK_SMALL, WALK_CHUNKED):
        s = Schedule(A, kind=KERNEL_ICCG, nthread=8, walk=walk)
        x = _t(np.zeros(A.n))
        s.iccg(dA, _t(b), x, tol=1e-12, maxiter=2000)
        lam = _t(np.zeros(A.n))
        ga = torch.zeros(A.nnz, dtype=torch.float64, device="cuda")
        s.iccg_adjoint(dA, _t(g), lam, x=x, grad_a=ga, tol=1e-12, maxiter=2000)
        assert s.last_walk == walk
        out[walk] = (lam.cpu().numpy(), ga.cpu().numpy())
    for k in range(2):
        a, c = out[WALK_SMALL][k], out[WALK_CHUNKED][k]
        assert np.linalg.norm(a - c) / np.linalg.norm(c) <= 1e-10


def test_forced_small_walk_refuses_a_large_system():
    A = gen.laplace3d(32, 1e-3)  # 32,768 rows: more than one CTA's shared memory holds
    s = Schedule(A, kind=KERNEL_ICCG, nthread=8, walk=WALK_SMALL)
    x = _t(np.zeros(A.n))
    with pytest.raises(BaasError, match="single-CTA"):
        s.iccg(DeviceCSR.from_host(A), _t(gen.uniform_rhs(A.n, 1)), x)


@pytest.mark.parametrize("cs", [1, 2, 4, 8, 16])
def test_every_cluster_size_gives_the_same_factor_and_sweeps(cs):
    A = gen.knn_stiffness(nodes=1500, k=12, seed=6)
    s = Schedule(A, kind=KERNEL_ICCG, nthread=8, walk=WALK_SMALL, small_cluster=cs)
    dA = DeviceCSR.from_host(A)
    lu = dA.values.clone()
    s.ic0(dA, lu)
    want, _ = Port.ic0(A)
    assert np.array_equal(lu.cpu().numpy(), want)
    Lo = gen.CSR(A.n, A.rowptr, A.colidx, want).lower()
    r = gen.uniform_rhs(A.n, 8)
    y = _t(np.zeros(A.n))
    s.forward(DeviceCSR.from_host(Lo), _t(r), y)
    assert np.array_equal(y.cpu().numpy(), Port.lower_solve(Lo, r))
    b = gen.uniform_rhs(A.n, 9)
    xo, ito, _ = Port.pcg(A, b, tol=1e-10)
    x = _t(np.zeros(A.n))
    it, rel = s.iccg(dA, _t(b), x, tol=1e-10)
    assert abs(it - ito) <= 1 and np.linalg.norm(x.cpu().numpy() - xo) / np.linalg.norm(xo) <= 1e-12


def test_walk_autotuner_leaves_the_fastest_walk():
    from baas_b200 import autotune

    A = gen.knn_stiffness(nodes=1000, k=12, seed=3)
    s = Schedule(A, kind=KERNEL_ICCG, nthread=8)
    dA = DeviceCSR.from_host(A)
    b = _t(gen.uniform_rhs(A.n, 1))
    x = _t(np.zeros(A.n))

    def run():
        x.zero_()
        s.iccg(dA, b, x, tol=1e-10)

    out = autotune.tune_walk(s, run)
    ran = [r for r in out["table"] if r["ms"] is not None]
    assert min(r["ms"] for r in ran) == out["best"]["ms"]
    assert any(r["ms"] is None for r in out["table"])  # the fetch walk refuses the k-NN rows
    run()
    assert s.last_walk == out["best"]["walk"]
