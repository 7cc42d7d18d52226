"""Failure detection on the GPU without faulting it: a dependency that nothing will ever
satisfy makes a bounded device wait give up, the call returns BAAS_ERR_TIMEOUT, and the CUDA
context stays usable for the next call."""
import numpy as np
import pytest

from baas_b200 import KERNEL_SPTRSV, BaasError, DeviceCSR, Schedule, gen
from oracle.oracle import Port

pytestmark = pytest.mark.gpu


def _t(a):
    import torch

    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


@pytest.mark.parametrize("parts", [1, 4])
def test_unsatisfiable_dependency_times_out_and_context_survives(parts):
    L, x_true, b = gen.sptrsv_case(16, 0)
    dL = DeviceCSR.from_host(L)
    # ~1e4 polls (well under a second) before a wait gives up
    s = Schedule(L, kind=KERNEL_SPTRSV, nthread=2, spin_limit=1 << 14, parts=parts)
    # row 37 then waits on its own output slot, which only it would write; every index stays
    # inside [0, n)
    s.inject_unsatisfiable_wait(37)
    x = _t(np.zeros(L.n))
    with pytest.raises(BaasError) as e:
        s.forward(dL, _t(b), x)
    assert e.value.status_name == "BAAS_ERR_TIMEOUT"
    # a fresh schedule on the same device and context works and is exact
    s2 = Schedule(L, kind=KERNEL_SPTRSV, nthread=2, parts=parts)
    x2 = _t(np.zeros(L.n))
    s2.forward(dL, _t(b), x2)
    assert np.array_equal(x2.cpu().numpy(), Port.lower_solve(L, b))
