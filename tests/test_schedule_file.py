"""Schedule files (baas_schedule_save / baas_schedule_load): a saved schedule loads back with every
array of the analysis intact, so a later process skips the analysis; foreign, truncated or
inconsistent files are refused; on the GPU the loaded schedule solves bit for bit as the original."""
import numpy as np
import pytest

from baas_b200 import KERNEL_ICCG, KERNEL_ILU0, KERNEL_SPTRSV, BaasError, Schedule, gen
from baas_b200._native import FIELDS, GROUP_DAG_FIELDS

ALL = list(FIELDS) + list(GROUP_DAG_FIELDS)


@pytest.mark.parametrize("kind,mk", [(KERNEL_ICCG, lambda: gen.knn_stiffness(nodes=300, k=8, seed=1)),
                                     (KERNEL_ILU0, lambda: gen.convdiff3d(8)),
                                     (KERNEL_SPTRSV, lambda: gen.laplace2d(20).lower())])
def test_saved_schedule_loads_back(tmp_path, kind, mk):
    A = mk()
    s = Schedule(A, kind=kind, nthread=8, mapping=0)
    p = tmp_path / "sched.bin"
    s.save(p)
    t = Schedule.load(p)
    assert (t.n, t.nnz, t.kind, t.nthread) == (A.n, A.nnz, kind, 8)
    for f in ALL:
        assert np.array_equal(s.export(f), t.export(f)), f
    # the emulated sweep plan of the loaded schedule solves as the original's
    if kind == KERNEL_SPTRSV:
        b = gen.uniform_rhs(A.n, 2)
        assert np.array_equal(s.emulate_sweep(A, b), t.emulate_sweep(A, b))


def test_bad_files_are_refused(tmp_path):
    A = gen.laplace2d(12)
    s = Schedule(A, kind=KERNEL_ICCG, nthread=4)
    p = tmp_path / "s.bin"
    s.save(p)
    data = p.read_bytes()
    (tmp_path / "trunc.bin").write_bytes(data[: len(data) // 2])
    (tmp_path / "junk.bin").write_bytes(b"not a schedule at all" * 10)
    for name in ("trunc.bin", "junk.bin", "missing.bin"):
        with pytest.raises(BaasError) as e:
            Schedule.load(tmp_path / name)
        assert e.value.status_name == "BAAS_ERR_BAD_ARG"


@pytest.mark.gpu
def test_loaded_schedule_solves_like_the_original(tmp_path):
    import torch

    from baas_b200 import DeviceCSR

    A = gen.laplace3d(20, 1e-3)
    s = Schedule(A, kind=KERNEL_ICCG, nthread=8)
    p = tmp_path / "s.bin"
    s.save(p)
    t = Schedule.load(p)
    dA = DeviceCSR.from_host(A)
    b = torch.from_numpy(gen.uniform_rhs(A.n, 1)).cuda()
    out = []
    for sch in (s, t):
        x = torch.zeros_like(b)
        it, rel = sch.iccg(dA, b, x, tol=1e-10)
        out.append((it, x.cpu().numpy()))
    assert out[0][0] == out[1][0] and np.array_equal(out[0][1], out[1][1])
