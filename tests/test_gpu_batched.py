"""Batched ICCG (baas_analyze_batch + baas_iccg_batched): many independent SPD systems with several
right-hand sides each, in one persistent launch, checked per instance against the oracle's PCG
(iterations within +-1 for FP64 factors, solutions within 1e-12 relative for FP64 factors and
1e-9 for FP32 factors) and by independent residuals."""
import numpy as np
import pytest

from baas_b200 import PREC_FP32_FACTORS, PREC_FP64, BatchSchedule, DeviceCSR, gen
from oracle.oracle import Port

pytestmark = pytest.mark.gpu


def _t(a):
    import torch

    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _solve(systems, nrhs, precision, tol=1e-10, parts=0, seed=2):
    import torch

    s = BatchSchedule(systems, nthread=8, parts=parts)
    A = s.combined
    B = gen.uniform_rhs(A.n, seed, nrhs=nrhs).reshape(nrhs, A.n)
    dA = DeviceCSR.from_host(A)
    X = torch.zeros((nrhs, A.n), dtype=torch.float64, device="cuda")
    it, rel = s.iccg_batched(dA, _t(B), X, tol=tol, maxiter=5000, precision=precision)
    return s, B, X.cpu().numpy(), it, rel


@pytest.mark.parametrize("precision", [PREC_FP64, PREC_FP32_FACTORS])
@pytest.mark.parametrize("nrhs", [1, 4])
def test_batched_small_matches_oracle(precision, nrhs):
    rng = np.random.default_rng(3)
    systems = [gen.vardiff2d(int(k), seed=10 + j) for j, k in enumerate(rng.integers(6, 40, size=7))]
    s, B, X, it, rel = _solve(systems, nrhs, precision, parts=5)
    assert np.all(rel < 1e-10)
    off = s.sys_off
    for q, m in enumerate(systems):
        for r in range(nrhs):
            b = B[r, off[q]:off[q + 1]]
            xw, itw, _ = Port.pcg(m, b, tol=1e-10, maxiter=5000)
            x = X[r, off[q]:off[q + 1]]
            assert np.linalg.norm(x - xw) / np.linalg.norm(xw) <= (1e-12 if precision == PREC_FP64 else 1e-9)
            if precision == PREC_FP64:
                assert abs(int(it[q, r]) - itw) <= 1


def test_batched_zero_rhs_and_one_system():
    import torch

    systems = [gen.laplace2d(10), gen.vardiff2d(12, seed=1)]
    s = BatchSchedule(systems, parts=3)
    A = s.combined
    B = gen.uniform_rhs(A.n, 5, nrhs=2).reshape(2, A.n)
    B[1, s.sys_off[0]:s.sys_off[1]] = 0.0  # system 0, right-hand side 1: already solved
    X = torch.zeros((2, A.n), dtype=torch.float64, device="cuda")
    it, rel = s.iccg_batched(DeviceCSR.from_host(A), _t(B), X, tol=1e-10)
    assert it[0, 1] == 0 and rel[0, 1] == 0.0
    assert np.all(X[1, :100].cpu().numpy() == 0.0)
    assert np.all(rel[:, 0] < 1e-10) and rel[1, 1] < 1e-10


def test_batched_full_configuration():
    """64 systems, k ~ U[64, 512], 4 right-hand sides, FP32 factors; residuals recomputed on the
    CPU, and every system against the FP64 oracle's PCG at the same tolerance (system q with
    right-hand side q % 4; the oracle solves run in a pool of spawned processes)."""
    from oracle.oracle import pcg_many

    systems = gen.batch_vardiff2d()
    s, B, X, it, rel = _solve(systems, 4, PREC_FP32_FACTORS)
    assert np.all(rel < 1e-10)
    off = s.sys_off
    Asp = s.combined.to_scipy()
    for r in range(4):
        res = B[r] - Asp @ X[r]
        for q in range(len(systems)):
            sl = slice(off[q], off[q + 1])
            assert np.linalg.norm(res[sl]) / np.linalg.norm(B[r, sl]) < 1e-9
    jobs = [(m, B[q % 4, off[q]:off[q + 1]], 1e-10, 20000) for q, m in enumerate(systems)]
    errs = []
    for q, (xw, itw, relw) in enumerate(pcg_many(jobs)):
        assert relw < 1e-10
        x = X[q % 4, off[q]:off[q + 1]]
        errs.append(np.linalg.norm(x - xw) / np.linalg.norm(xw))
    print(f"FP32-factor batch vs FP64 oracle: max {max(errs):.3e}, median {np.median(errs):.3e}")
    assert max(errs) <= 1e-8


@pytest.mark.parametrize("nrhs", [2, 4])
def test_row_wide_sweeps_match_pair_sweeps(monkeypatch, nrhs):
    """FP32 factors with 2 or 4 right-hand sides sweep one row per thread for all of them; the
    one-pair-per-thread sweeps (BAAS_BATCH_PAIRS=1) must give the same bits, iterations and
    residuals, on systems wide enough that a level spans several passes of the pair mapping."""
    systems = [gen.vardiff2d(int(k), seed=30 + j) for j, k in enumerate((90, 40, 120, 7))]
    out = []
    for pairs in ("1", "0"):
        monkeypatch.setenv("BAAS_BATCH_PAIRS", pairs)
        s, B, X, it, rel = _solve(systems, nrhs, PREC_FP32_FACTORS, parts=6)
        out.append((X, it, rel))
    assert np.array_equal(out[0][0].view(np.int64), out[1][0].view(np.int64))
    assert np.array_equal(out[0][1], out[1][1]) and np.array_equal(out[0][2], out[1][2])
    assert np.all(out[1][2] < 1e-10)


def test_rank_share_of_a_batch_matches_the_oracle():
    """baas_b200.distributed.batched_solve (one rank's share of a batch split across GPUs) on one
    GPU: every system of the share solved to tol, solutions within 1e-9 of the oracle's FP64 PCG
    (FP32 factors) and the split a partition of the batch."""
    from baas_b200.distributed import batched_solve, split_systems
    from oracle.oracle import Port

    systems = gen.batch_vardiff2d(nsys=6, kmin=16, kmax=40, seed=9)
    parts = split_systems([S.n for S in systems], 2)
    rhs = lambda q: gen.uniform_rhs(systems[q].n, 500 + q, nrhs=2)  # noqa: E731
    for idx in parts:
        got = batched_solve(systems, idx, rhs, tol=1e-10, precision=1)
        assert got[-1] > 0.0
        for q in idx:
            B = rhs(q)
            for r in range(2):
                xo, _, _ = Port.pcg(systems[q], B[r], tol=1e-10)
                x = got[q]["x"][r]
                assert got[q]["relres"][r] < 1e-10
                assert np.linalg.norm(x - xo) / np.linalg.norm(xo) <= 1e-9
