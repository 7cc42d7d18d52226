"""baas_ic0_noalloc: the IC0 entry point that allocates nothing, for callers that cannot call
cudaMalloc when they factor (pre-reserved real-time loops, plug-ins whose host forbids device
allocation after start-up, hosts whose device memory belongs to another allocator). Its scratch is a static
device array inside the library, shared by every call.

This file is collected last on purpose: if it fails, a run that stops at the first failure has
already run every other test. It passes alone in a fresh process (the schedule's plan is made
resident by the ordinary call below) and after the other tests (each call clears the shared
scratch it needs)."""
import numpy as np
import pytest

from baas_b200 import KERNEL_ICCG, BaasError, DeviceCSR, Schedule, gen

pytestmark = pytest.mark.gpu


def test_ic0_noalloc_matches_ic0_on_two_calls_in_a_row():
    import torch

    A = gen.laplace3d(20, 1e-3)
    s = Schedule(A, kind=KERNEL_ICCG, nthread=8)
    dA = DeviceCSR.from_host(A)
    ref = dA.values.clone()
    s.ic0(dA, ref)  # ordinary entry point; also makes the schedule's device plan resident
    want = ref.cpu().numpy()
    lus = [dA.values.clone() for _ in range(3)]
    s.ic0_noalloc(dA, lus[0])  # a first call (it looks the static array's address up)
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    for lu in lus[1:]:  # two calls in a row
        s.ic0_noalloc(dA, lu)
        torch.cuda.synchronize()
        # the property the entry point exists for: the device's free memory does not move
        assert torch.cuda.mem_get_info()[0] == free0
    for lu in lus:
        # same tolerance as the other IC0 tests: the factors are bit-identical
        assert np.array_equal(lu.cpu().numpy(), want)


def test_ic0_noalloc_needs_a_resident_plan():
    A = gen.laplace3d(6, 1e-3)
    s = Schedule(A, kind=KERNEL_ICCG, nthread=2)
    dA = DeviceCSR.from_host(A)
    lu = dA.values.clone()
    with pytest.raises(BaasError) as e:
        s.ic0_noalloc(dA, lu)
    assert e.value.status_name == "BAAS_ERR_STATE"
