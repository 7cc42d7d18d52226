"""Why the permuted (thread-contiguous) variant is not built: evidence from the reference's own
schedule. Scheduler::permPreprocessing (test/Schedule.hpp:298-314) orders the groups by the
mapping's thread-contiguous permutation (groupPerm, :81-112), and the perm routines
(sptrsv_p2p_csr_group_merge_perm_alloc, merge/SpTRSV.cpp:480-542; spic0_csr_uL_p2p_group_merge_perm,
merge/IC.cpp:409-508) then run on the lower part of the matrix permuted into that order. That lower
part is a different triangle whenever the permutation reverses the order of two coupled rows: row
i then reads row j although j comes after i in the dependency order (the task schedule never waits
for it), and the entry it should read instead lies in the dropped upper part. This test rebuilds
the permutation from the reference's exported schedule (oracle/_ref, the reference compiled from
its sources) and counts those reversed couplings: none with one thread, hundreds with eight."""
import numpy as np
import pytest

from baas_b200 import gen
from oracle.oracle import Ref, ref_available

pytestmark = pytest.mark.skipif(not ref_available(), reason="the reference library (oracle/_ref) is not built")


def _orig_to_perm(rs):
    """origToPermByThread of groupPerm: groups in thread-contiguous order, rows in group order."""
    gp, gs, tc = rs.export("group_ptr"), rs.export("group_set"), rs.export("thread_cont_to_orig")
    perm_to_orig = np.concatenate([gs[gp[g]:gp[g + 1]] for g in tc])
    o2p = np.empty_like(perm_to_orig)
    o2p[perm_to_orig] = np.arange(perm_to_orig.size)
    return o2p


def _reversed_couplings(A, nthread):
    rs = Ref.Schedule(1, A, nthread)  # kind ICCG: Scheduler(A, true, false, P2P_RULE, nthread)
    o2p = _orig_to_perm(rs)
    rows = np.repeat(np.arange(A.n), np.diff(A.rowptr))
    lower = A.colidx < rows  # entry (i, j), j < i: row j precedes row i in the dependency order
    i, j = rows[lower], A.colidx[lower]
    return int(np.count_nonzero(o2p[j] > o2p[i])), int(lower.sum())


def test_one_thread_keeps_every_coupling():
    flips, total = _reversed_couplings(gen.laplace3d(12, 1e-3), 1)
    assert total == 4752 and flips == 0


@pytest.mark.parametrize("nthread", [8, 16])
def test_several_threads_reverse_couplings(nthread):
    flips, total = _reversed_couplings(gen.laplace3d(12, 1e-3), nthread)
    assert total == 4752
    assert flips > 0  # the permuted lower part then reads rows its task schedule has not finished
    if nthread == 8:
        assert flips == 780
