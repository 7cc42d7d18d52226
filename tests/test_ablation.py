"""The SpTRSV runtime's ablation schedules (test/SpTRSV_level_merge.cpp:156-299) against the
reference compiled from its sources (oracle/_ref): BAASWOS (coarsening, TRSV level merge,
cost-balanced split), BAASWOA (no coarsening, four-rule mapping) and BAASWOAS (no coarsening,
min(rows, nthread) threads per level, cost-balanced split). Every exported array, bit for bit,
on a stencil, a k-NN stiffness matrix and a variable-coefficient grid at several thread counts;
the sweep plan of each, run on the host, against the oracle's serial sweep."""
import numpy as np
import pytest

from baas_b200 import (ABLATION_NONE, ABLATION_WOA, ABLATION_WOAS, ABLATION_WOS, KERNEL_ICCG, KERNEL_SPTRSV,
                       BaasError, Schedule, gen)
from baas_b200._native import FIELDS
from oracle.oracle import Ref, ref_available

CASES = [
    ("laplace2d_40", lambda: gen.laplace2d(40).lower()),
    ("laplace3d_12", lambda: gen.laplace3d(12, 1e-3).lower()),
    ("knn_600", lambda: gen.knn_stiffness(nodes=600, k=12, seed=3).lower()),
    ("vardiff2d_48", lambda: gen.vardiff2d(48, seed=5).lower()),
]


@pytest.mark.skipif(not ref_available(), reason="the reference library (oracle/_ref) is not built")
@pytest.mark.parametrize("ablation", [ABLATION_NONE, ABLATION_WOS, ABLATION_WOA, ABLATION_WOAS])
@pytest.mark.parametrize("case", [c[0] for c in CASES])
def test_ablation_schedules_match_live_reference(case, ablation):
    L = next(mk for name, mk in CASES if name == case)()
    for nt in (1, 3, 8, 16):
        ours = Schedule(L, kind=KERNEL_SPTRSV, nthread=nt, ablation=ablation).arrays()
        ref = Ref.Schedule(KERNEL_SPTRSV, L, nt, ablation=ablation).arrays()
        for f in FIELDS:
            assert np.array_equal(ours[f], ref[f]), f"{case} ablation={ablation} nthread={nt} field {f}"


@pytest.mark.parametrize("ablation", [ABLATION_WOS, ABLATION_WOA, ABLATION_WOAS])
def test_ablation_sweep_plans_solve(ablation):
    """The chunked plan of an ablation schedule, run on the host, equals the serial sweep."""
    from oracle.oracle import Port

    L = gen.laplace3d(10, 1e-3).lower()
    s = Schedule(L, kind=KERNEL_SPTRSV, nthread=8, ablation=ablation)
    b = gen.uniform_rhs(L.n, 3)
    x = s.emulate_sweep(L, b)
    assert np.array_equal(x, Port.lower_solve(L, b))


def test_ablation_needs_sptrsv_and_the_four_rule_mapping():
    with pytest.raises(BaasError):
        Schedule(gen.laplace2d(6), kind=KERNEL_ICCG, nthread=2, ablation=ABLATION_WOS)
    with pytest.raises(BaasError):
        Schedule(gen.laplace2d(6).lower(), kind=KERNEL_SPTRSV, nthread=2, ablation=9)


@pytest.mark.gpu
@pytest.mark.parametrize("ablation", [ABLATION_WOS, ABLATION_WOA, ABLATION_WOAS])
def test_gpu_sweep_on_ablation_schedules(ablation):
    """The GPU forward sweep on each ablation's schedule, bit-exact against the oracle's serial
    sweep (the device plan runs any grouping and mapping)."""
    import torch

    from baas_b200 import DeviceCSR
    from oracle.oracle import Port

    L = gen.laplace2d(128).lower()
    s = Schedule(L, kind=KERNEL_SPTRSV, nthread=8, ablation=ablation)
    dL = DeviceCSR.from_host(L)
    b = gen.uniform_rhs(L.n, 5)
    x = torch.zeros(L.n, dtype=torch.float64, device="cuda")
    s.sptrsv(dL, torch.from_numpy(b).cuda(), x, upper=False)
    assert np.array_equal(x.cpu().numpy(), Port.lower_solve(L, b))
