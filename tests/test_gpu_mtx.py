"""A matrix that arrives as a MatrixMarket file (baas_csr_read_mtx) through the GPU path: a k-NN
stiffness-like SPD system written to a symmetric .mtx, read back, then IC0 bit-exact against the
oracle and ICCG within +-1 iteration of the oracle's PCG."""
import numpy as np
import pytest

from baas_b200 import KERNEL_ICCG, KERNEL_IC0, DeviceCSR, Schedule, gen
from oracle.oracle import Port

pytestmark = pytest.mark.gpu


def test_mtx_file_to_gpu_solve(tmp_path):
    import torch

    p = tmp_path / "stiff.mtx"
    gen.write_mtx(gen.knn_stiffness(nodes=3000, k=12, seed=5), p, symmetric=True)
    A = gen.read_mtx(p)
    dA = DeviceCSR.from_host(A)

    f = Schedule(A, kind=KERNEL_IC0, nthread=8)
    lu = dA.values.clone()
    f.ic0(dA, lu)
    want, _ = Port.ic0(A)
    assert np.array_equal(lu.cpu().numpy(), want)

    s = Schedule(A, kind=KERNEL_ICCG, nthread=8)
    b = gen.uniform_rhs(A.n, 3)
    x = torch.zeros(A.n, dtype=torch.float64, device="cuda")
    it, rel = s.iccg(dA, torch.from_numpy(b).cuda(), x, tol=1e-10, maxiter=5000)
    xo, ito, _ = Port.pcg(A, b, tol=1e-10, maxiter=5000)
    assert abs(it - ito) <= 1 and rel < 1e-10
    assert np.linalg.norm(x.cpu().numpy() - xo) / np.linalg.norm(xo) < 1e-8
