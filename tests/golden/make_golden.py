"""Generates tests/golden/*.npz from the reference itself (oracle/_ref/libbaas_ref.so, the
reference's spm/, merge/ and blas/ sources compiled by oracle/Makefile).

The reference ships no golden vectors or known-answer tests (its drivers compare against its own
serial routines), so these fixtures pin our oracle and our schedule to outputs the reference
produced here:
  * schedule arrays (LevelSet, groups, thread/task boundaries, task DAGs) for small matrices
    of every schedule kind and several thread counts, plus SHA-256 digests of the full-size
    128x128 SpTRSV schedule at 1/4/8 threads;
  * results of the reference's serial and p2p numeric routines on small matrices: forward
    sweep, backward p2p sweep, IC0, ILU0, and the pcg_opt iteration count / solution.

Run from the repository root:  python tests/golden/make_golden.py
"""
from __future__ import annotations

import hashlib
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from baas_b200 import gen  # noqa: E402
from oracle.oracle import FIELDS, Ref  # noqa: E402

OUT = Path(__file__).resolve().parent

# (name, kind, matrix factory, thread counts[, mapping: BAAS_MAPPING_*, default the four-rule one])
SCHEDULE_CASES = [
    ("lap2d_12_lower", 0, lambda: gen.laplace2d(12).lower(), (1, 3, 4)),
    ("lap3d_6", 1, lambda: gen.laplace3d(6, 1e-3), (2, 4)),
    ("lap3d_6_ic0", 2, lambda: gen.laplace3d(6, 1e-3), (3,)),
    ("convdiff_5_ilu0", 3, lambda: gen.convdiff3d(5), (3,)),
    ("knn_200", 1, lambda: gen.knn_stiffness(nodes=200, k=12, seed=3), (4,)),
    ("lap3d_6_perm", 1, lambda: gen.laplace3d(6, 1e-3).permuted(gen.random_symmetric_permutation(216, 5)), (4,)),
    # the Scheduler's P2P algorithm: level merge + cost split, and its barrier-mode task layout
    ("lap3d_8_p2p", 1, lambda: gen.laplace3d(8, 1e-3), (3, 8), 1),
    ("knn_200_p2p_barrier", 1, lambda: gen.knn_stiffness(nodes=200, k=12, seed=3), (4,), 2),
    # P2P_TIME: earliest-finishing threads take the earliest-startable groups
    ("lap3d_8_p2p_time", 1, lambda: gen.laplace3d(8, 1e-3), (3, 8), 3),
    ("vardiff_30_p2p_time", 1, lambda: gen.vardiff2d(30, seed=2), (6,), 3),
    # P2P_MAPPING: parent-thread affinity with load rebalancing
    ("lap3d_8_p2p_mapping", 1, lambda: gen.laplace3d(8, 1e-3), (3, 8), 4),
    ("knn_200_p2p_mapping", 1, lambda: gen.knn_stiffness(nodes=200, k=12, seed=3), (5,), 4),
]


def schedule_digest(arrs: dict) -> str:
    h = hashlib.sha256()
    for k in sorted(arrs):
        h.update(k.encode())
        h.update(np.ascontiguousarray(arrs[k], dtype=np.int32).tobytes())
    return h.hexdigest()


def main() -> None:
    sched = {}
    for case in SCHEDULE_CASES:
        name, kind, mk, threads = case[:4]
        mapping = case[4] if len(case) > 4 else 0
        A = mk()
        sched[f"{name}__rowptr"] = A.rowptr
        sched[f"{name}__colidx"] = A.colidx
        sched[f"{name}__kind"] = np.array([kind], dtype=np.int32)
        sched[f"{name}__mapping"] = np.array([mapping], dtype=np.int32)
        for nt in threads:
            s = Ref.Schedule(kind, A, nt, mapping=mapping)
            for f in FIELDS:
                sched[f"{name}__t{nt}__{f}"] = s.export(f)
    # full-size C1 schedule digests
    L = gen.laplace2d(128).lower()
    for nt in (1, 4, 8):
        arrs = Ref.Schedule(0, L, nt).arrays()
        sched[f"c1_128__t{nt}__digest"] = np.frombuffer(bytes.fromhex(schedule_digest(arrs)), dtype=np.uint8)
        sched[f"c1_128__t{nt}__ntasks"] = arrs["ntasks"]
    np.savez_compressed(OUT / "schedules.npz", **sched)

    num = {}
    # forward sweep on tril(5-pt 16x16), x_true ~ U(-1,1) seed 0
    Lo, xt, b = gen.sptrsv_case(16, 0)
    num["lower_rowptr"], num["lower_colidx"], num["lower_values"], num["lower_b"] = Lo.rowptr, Lo.colidx, Lo.values, b
    num["lower_x_serial"] = Ref.sptrsv_serial(Lo, b)
    num["lower_x_p2p"] = Ref.Schedule(0, Lo, 4).forward(Lo, b)
    # IC0 (serial and p2p) and the p2p backward sweep on U = L^T, 7-pt 6^3 + 1e-3 I
    A = gen.laplace3d(6, 1e-3)
    num["ic_rowptr"], num["ic_colidx"], num["ic_values"] = A.rowptr, A.colidx, A.values
    lu = Ref.ic0_serial(A)
    num["ic_lu_serial"] = lu
    num["ic_lu_p2p"] = Ref.Schedule(1, A, 4).ic0(A)
    Lf = gen.CSR(A.n, A.rowptr, A.colidx, lu).lower()
    Uf = gen.from_scipy(Lf.to_scipy().T.tocsr())
    r = gen.uniform_rhs(A.n, 1)
    num["ic_r"] = r
    y = Ref.Schedule(1, A, 4).forward(Lf, r)
    num["ic_y"] = y
    num["ic_z_p2p"] = Ref.Schedule(1, A, 4).backward(Uf, y)
    # ILU0 on the 5^3 convection-diffusion operator
    C = gen.convdiff3d(5)
    num["ilu_rowptr"], num["ilu_colidx"], num["ilu_values"] = C.rowptr, C.colidx, C.values
    num["ilu_lu_serial"] = Ref.ilu0_serial(C)
    num["ilu_lu_p2p"] = Ref.Schedule(3, C, 3).ilu0(C)
    # pcg_opt structure on 7-pt 10^3 + 1e-3 I, b ~ U(-1,1) seed 1
    P = gen.laplace3d(10, 1e-3)
    pb = gen.uniform_rhs(P.n, 1)
    x, it, rel, _ = Ref.pcg(P, pb, maxiter=2000, tol=1e-10, mode=1, nthread=4)
    num["pcg_b"], num["pcg_x"] = pb, x
    num["pcg_iters"] = np.array([it], dtype=np.int32)
    num["pcg_relres"] = np.array([rel])
    np.savez_compressed(OUT / "numeric.npz", **num)
    print("wrote", OUT / "schedules.npz", OUT / "numeric.npz")


if __name__ == "__main__":
    main()
