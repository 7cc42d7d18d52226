"""The host-side BAAS schedule (baas_b200/csrc/schedule.cpp) against the reference.

Pinned two ways: against golden arrays the reference produced (tests/golden/make_golden.py; runs
anywhere) and against the reference compiled from its sources (oracle/_ref; runs where it was
built). Bit-exact equality of every exported array: level sets, groups, thread/task boundaries,
the four-rule mapping and both task DAGs.
"""
import hashlib
from pathlib import Path

import numpy as np
import pytest

from baas_b200 import KERNEL_ICCG, KERNEL_IC0, KERNEL_ILU0, KERNEL_SPTRSV, Schedule, gen
from baas_b200._native import FIELDS

GOLD = Path(__file__).resolve().parent / "golden" / "schedules.npz"


def _golden():
    return np.load(GOLD)


def _cases(z):
    names = sorted({k.split("__")[0] for k in z.files if k.endswith("__kind")})
    for name in names:
        threads = sorted({int(k.split("__")[1][1:]) for k in z.files if k.startswith(name + "__t")})
        for nt in threads:
            yield name, nt


@pytest.mark.parametrize("name,nt", list(_cases(np.load(GOLD))))
def test_schedule_matches_reference_golden(name, nt):
    z = _golden()
    A = gen.CSR(int(len(z[f"{name}__rowptr"]) - 1), z[f"{name}__rowptr"], z[f"{name}__colidx"],
                np.ones(len(z[f"{name}__colidx"])))
    kind = int(z[f"{name}__kind"][0])
    mapping = int(z[f"{name}__mapping"][0]) if f"{name}__mapping" in z.files else 0
    s = Schedule(A, kind=kind, nthread=nt, mapping=mapping)
    for f in FIELDS:
        want = z[f"{name}__t{nt}__{f}"]
        got = s.export(f)
        assert np.array_equal(got, want), f"{name} nthread={nt} field {f}"


def _digest(arrs):
    h = hashlib.sha256()
    for k in sorted(arrs):
        h.update(k.encode())
        h.update(np.ascontiguousarray(arrs[k], dtype=np.int32).tobytes())
    return h.digest()


@pytest.mark.parametrize("nt", [1, 4, 8])
def test_c1_full_size_schedule_digest(nt):
    z = _golden()
    L = gen.laplace2d(128).lower()
    s = Schedule(L, kind=KERNEL_SPTRSV, nthread=nt)
    arrs = s.arrays()
    assert int(arrs["ntasks"][0]) == int(z[f"c1_128__t{nt}__ntasks"][0])
    assert _digest(arrs) == bytes(z[f"c1_128__t{nt}__digest"])


LIVE = [
    (KERNEL_SPTRSV, lambda: gen.laplace2d(40).lower(), (1, 2, 5, 8, 16)),
    (KERNEL_ICCG, lambda: gen.laplace3d(12, 1e-3), (3, 8, 13)),
    (KERNEL_IC0, lambda: gen.laplace3d(10, 1e-3), (4, 7)),
    (KERNEL_ILU0, lambda: gen.convdiff3d(9), (2, 6)),
    (KERNEL_ICCG, lambda: gen.knn_stiffness(nodes=600, k=12, seed=3), (4, 8)),
    (KERNEL_ICCG, lambda: gen.vardiff2d(48, seed=5), (8,)),
    (KERNEL_ICCG, lambda: gen.laplace3d(10, 1e-3).permuted(gen.random_symmetric_permutation(1000, 7)), (8,)),
]


@pytest.mark.parametrize("case", range(len(LIVE)))
def test_schedule_matches_live_reference(case, ref_lib):
    kind, mk, threads = LIVE[case]
    A = mk()
    for nt in threads:
        ours = Schedule(A, kind=kind, nthread=nt).arrays()
        ref = ref_lib.Schedule(kind, A, nt).arrays()
        for f in FIELDS:
            assert np.array_equal(ours[f], ref[f]), f"kind={kind} nthread={nt} field {f}"


MAPPED = [
    lambda: gen.laplace3d(12, 1e-3),
    lambda: gen.knn_stiffness(nodes=600, k=12, seed=3),
    lambda: gen.vardiff2d(48, seed=5),
]


@pytest.mark.parametrize("mapping", [1, 2, 3, 4])
@pytest.mark.parametrize("case", range(len(MAPPED)))
def test_scheduler_mappings_match_live_reference(case, mapping, ref_lib):
    """The Scheduler's P2P algorithm (level merge + Task::constructTask), its barrier-mode task
    layout, P2P_TIME (Task::constructMappingByFinishTime) and P2P_MAPPING
    (Task::constructMappingMergeSerial), every exported array against the reference's."""
    A = MAPPED[case]()
    for nt in (3, 8, 16):
        ours = Schedule(A, kind=KERNEL_ICCG, nthread=nt, mapping=mapping).arrays()
        ref = ref_lib.Schedule(KERNEL_ICCG, A, nt, mapping=mapping).arrays()
        for f in FIELDS:
            assert np.array_equal(ours[f], ref[f]), f"mapping={mapping} nthread={nt} field {f}"


def test_mapping_checks():
    from baas_b200 import BaasError

    with pytest.raises(BaasError):
        Schedule(gen.laplace2d(8).lower(), kind=KERNEL_SPTRSV, mapping=1)  # the Scheduler's (ICCG) only
    with pytest.raises(BaasError):
        Schedule(gen.laplace3d(4, 1e-3), kind=KERNEL_ICCG, mapping=5)
    s = Schedule(gen.laplace3d(4, 1e-3), kind=KERNEL_ICCG, mapping=1)
    s.replan(parts=2)  # keeps the analysed mapping


def test_schedule_invariants():
    """Structural properties the executors rely on: groups partition the rows, levels partition
    the groups, every task DAG edge points to an earlier-level task on another thread."""
    A = gen.laplace3d(10, 1e-3)
    s = Schedule(A, kind=KERNEL_ICCG, nthread=6)
    a = s.arrays()
    n = A.n
    assert sorted(a["group_set"].tolist()) == list(range(n))
    ng = int(a["ngroups"][0])
    assert sorted(a["perm_to_orig"].tolist()) == list(range(ng))
    assert a["level_ptr"][-1] == ng
    assert a["thread_boundaries"][-1] == int(a["ntasks"][0])
    assert sorted(a["thread_cont_to_orig"].tolist()) == list(range(ng))
    tb = a["thread_boundaries"]
    owner = np.searchsorted(tb, np.arange(int(a["ntasks"][0])), side="right") - 1
    tp, ts = a["task_ptr"], a["task_set"]
    for t in range(int(a["ntasks"][0])):
        for q in ts[tp[t]:tp[t + 1]]:
            assert owner[q] != owner[t]


# The schedules the benchmark runs, at full size: configuration 2 (64^3, natural and permuted,
# and the k-NN stiffness matrix at n = 12,000) and configuration 3 (96^3 ILU0).
FULL = [
    ("c2_natural", KERNEL_ICCG, lambda: gen.c2_system(False), (8, 16)),
    ("c2_permuted", KERNEL_ICCG, lambda: gen.c2_system(True), (8,)),
    ("c2_knn_12000", KERNEL_ICCG, lambda: gen.knn_stiffness(nodes=4000), (8,)),
    ("c3_ilu0_96", KERNEL_ILU0, lambda: gen.convdiff3d(96), (8,)),
]


@pytest.mark.parametrize("case", [c[0] for c in FULL])
def test_full_size_schedules_match_live_reference(case, ref_lib):
    _, kind, mk, threads = next(c for c in FULL if c[0] == case)
    A = mk()
    for nt in threads:
        ours = Schedule(A, kind=kind, nthread=nt).arrays()
        ref = ref_lib.Schedule(kind, A, nt).arrays()
        for f in FIELDS:
            assert np.array_equal(ours[f], ref[f]), f"{case} nthread={nt} field {f}"
