"""Custom row-to-CTA maps (baas_replan_custom) on the GPU: blocks of grid columns, so cross-CTA
dependencies run both ways between CTAs. Sweeps and IC0 stay bit-exact with the oracle and ICCG
takes the oracle's iteration count (+-1), exactly as with the default contiguous ranges."""
import numpy as np
import pytest

from baas_b200 import KERNEL_IC0, KERNEL_ICCG, DeviceCSR, Schedule, gen
from oracle.oracle import Port

pytestmark = pytest.mark.gpu


def _t(a):
    import torch

    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _column_blocks(k, bi, bj):
    r = np.arange(k ** 3)
    i, j = r % k, (r // k) % k
    return (i // bi + ((k + bi - 1) // bi) * (j // bj)).astype(np.int32)


@pytest.mark.parametrize("blocks", [(4, 4), (3, 7)])
def test_custom_partition_sweeps_ic0_iccg(blocks):
    import torch

    k = 24
    A = gen.laplace3d(k, 1e-3)
    b = gen.uniform_rhs(A.n, 1)
    rp = _column_blocks(k, *blocks)
    dA = DeviceCSR.from_host(A)

    s = Schedule(A, kind=KERNEL_ICCG, nthread=8)
    s.replan_custom(rp)
    x = _t(np.zeros(A.n))
    it, rel = s.iccg(dA, _t(b), x, tol=1e-10, maxiter=2000)
    xo, ito, _ = Port.pcg(A, b, tol=1e-10)
    assert abs(it - ito) <= 1 and rel < 1e-10
    assert np.linalg.norm(x.cpu().numpy() - xo) / np.linalg.norm(xo) <= 1e-12

    lu_o, _ = Port.ic0(A)
    Lo = gen.CSR(A.n, A.rowptr, A.colidx, lu_o).lower()
    Up = Lo.transpose()
    y = torch.zeros(A.n, dtype=torch.float64, device="cuda")
    s.forward(DeviceCSR.from_host(Lo), _t(b), y)
    assert np.array_equal(y.cpu().numpy(), Port.lower_solve(Lo, b))
    z = torch.zeros_like(y)
    s.backward(DeviceCSR.from_host(Up), _t(b), z)
    assert np.array_equal(z.cpu().numpy(), Port.upper_solve(Up, b, descending=True))

    f = Schedule(A, kind=KERNEL_IC0, nthread=8)
    f.replan_custom(rp)
    lu = dA.values.clone()
    f.ic0(dA, lu)
    assert np.array_equal(lu.cpu().numpy(), lu_o)


@pytest.mark.parametrize("mapping", [1, 2, 3, 4])
def test_scheduler_mapping_on_gpu(mapping):
    """ICCG and the sweeps with CTA t running virtual thread t of the Scheduler's P2P, P2P_TIME or
    P2P_MAPPING mapping."""
    import torch

    from baas_b200 import PARTITION_BAAS_THREADS

    A = gen.laplace3d(16, 1e-3)
    b = gen.uniform_rhs(A.n, 1)
    s = Schedule(A, kind=KERNEL_ICCG, nthread=16, partition=PARTITION_BAAS_THREADS, mapping=mapping)
    dA = DeviceCSR.from_host(A)
    x = _t(np.zeros(A.n))
    it, rel = s.iccg(dA, _t(b), x, tol=1e-10, maxiter=2000)
    xo, ito, _ = Port.pcg(A, b, tol=1e-10)
    assert abs(it - ito) <= 1 and rel < 1e-10
    lu_o, _ = Port.ic0(A)
    Lo = gen.CSR(A.n, A.rowptr, A.colidx, lu_o).lower()
    y = torch.zeros(A.n, dtype=torch.float64, device="cuda")
    s.forward(DeviceCSR.from_host(Lo), _t(b), y)
    assert np.array_equal(y.cpu().numpy(), Port.lower_solve(Lo, b))


@pytest.mark.parametrize("k", [32, 72])
def test_default_range_count(k):
    """Automatic row ranges: one CTA per 2,048 rows, rounded up, and never more CTAs than SMs
    (32^3: 16 CTAs; 72^3 = 373,248 rows: capped at the SM count). The sweep on that plan solves
    L y = b, with L = I + tril(C, -1) diag(C)^-1 (columns scaled as in an ILU0 factor, so that
    forward substitution stays bounded)."""
    import scipy.sparse as sp
    import torch

    from baas_b200 import KERNEL_ILU0, PARTITION_RANGES

    C = gen.convdiff3d(k)
    Cs = C.to_scipy()
    Lo = gen.from_scipy(sp.tril(Cs, k=-1) @ sp.diags(1.0 / Cs.diagonal()) + sp.identity(C.n))
    s = Schedule(C, kind=KERNEL_ILU0, nthread=8, partition=PARTITION_RANGES)
    b = gen.normal_rhs(C.n, 5)
    y = _t(np.zeros(C.n))
    s.forward(DeviceCSR.from_host(Lo), _t(b), y)
    torch.cuda.synchronize()
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    P, box, _ = s.plan_parts()
    assert box is None
    assert P == min((C.n + 2047) // 2048, sms)
    r = Lo.to_scipy() @ y.cpu().numpy() - b
    assert np.linalg.norm(r) <= 1e-12 * np.linalg.norm(b)
