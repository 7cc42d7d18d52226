"""MatrixMarket ingestion (baas_csr_read_mtx): the reader against files this test writes, its
error handling, and -- where the reference tree is present -- against the reference's own reader
(SPM::CSR(fileName), spm/CSR.cpp:90-112) on the two real SPD stiffness matrices it ships
(data/bcsstk18.mtx, data/bcsstk38.mtx), followed by the BAAS schedule, IC0 and the plan's sweeps
on them, each bit for bit against the reference or the oracle."""
import os
from pathlib import Path

import numpy as np
import pytest

from baas_b200 import KERNEL_ICCG, BaasError, Schedule, gen
from oracle.oracle import Port

# the reference's shipped fixtures: $BAAS_REFERENCE/data, else beside this repository
REF_DATA = Path(os.environ.get("BAAS_REFERENCE") or Path(__file__).resolve().parents[2] / "reference") / "data"


def _same(a, b):
    return (a.n == b.n and np.array_equal(a.rowptr, b.rowptr) and np.array_equal(a.colidx, b.colidx)
            and np.array_equal(np.asarray(a.values).view(np.int64), np.asarray(b.values).view(np.int64)))


@pytest.mark.parametrize("symmetric", [False, True])
def test_roundtrip_real(tmp_path, symmetric):
    A = gen.knn_stiffness(nodes=250, k=8, seed=2)
    p = tmp_path / "a.mtx"
    gen.write_mtx(A, p, symmetric=symmetric)
    assert _same(gen.read_mtx(p), A)


def test_pattern_and_integer_fields(tmp_path):
    A = gen.laplace2d(9)
    p = tmp_path / "p.mtx"
    gen.write_mtx(A, p, symmetric=True, field="pattern")
    B = gen.read_mtx(p)
    assert np.array_equal(B.rowptr, A.rowptr) and np.array_equal(B.colidx, A.colidx)
    assert np.all(B.values == 1.0)
    q = tmp_path / "i.mtx"
    gen.write_mtx(gen.CSR(A.n, A.rowptr, A.colidx, np.round(A.values)), q, field="real")
    text = q.read_text().replace(" real ", " integer ").splitlines()
    body = [f"{l.split()[0]} {l.split()[1]} {int(float(l.split()[2]))}" for l in text[3:]]
    q.write_text("\n".join(text[:3] + body) + "\n")
    C = gen.read_mtx(q)
    assert np.array_equal(C.values, np.round(A.values))


def test_symmetric_expansion_order(tmp_path):
    """Stored entries first, then the mirrors of the off-diagonal ones, rows sorted by column."""
    p = tmp_path / "s.mtx"
    p.write_text("%%MatrixMarket matrix coordinate real symmetric\n% c\n3 3 4\n1 1 4\n3 1 -1.5\n2 2 5\n3 3 6\n")
    A = gen.read_mtx(p)
    assert A.rowptr.tolist() == [0, 2, 3, 5]
    assert A.colidx.tolist() == [0, 2, 1, 0, 2]
    assert A.values.tolist() == [4.0, -1.5, 5.0, -1.5, 6.0]


@pytest.mark.parametrize("text,why", [
    ("%%MatrixMarket matrix array real general\n2 2\n1\n2\n3\n4\n", "coordinate"),
    ("%%MatrixMarket matrix coordinate complex general\n1 1 1\n1 1 1 0\n", "field"),
    ("%%NotMatrixMarket\n1 1 1\n1 1 1\n", "banner"),
    ("%%MatrixMarket matrix coordinate real general\n2 3 1\n1 1 1\n", "square"),
    ("%%MatrixMarket matrix coordinate real general\n2 2 2\n1 1 1\n", "fewer"),
    ("%%MatrixMarket matrix coordinate real general\n2 2 1\n3 1 1\n", "range"),
    ("%%MatrixMarket matrix coordinate real general\n2 2 2\n1 1 1\n1 1 2\n", "repeated"),
    ("%%MatrixMarket matrix coordinate real skew-symmetric\n2 2 1\n2 1 1\n", "symmetry"),
])
def test_reader_errors(tmp_path, text, why):
    p = tmp_path / "bad.mtx"
    p.write_text(text)
    with pytest.raises(BaasError, match=why):
        gen.read_mtx(p)
    with pytest.raises(BaasError, match="cannot open"):
        gen.read_mtx(tmp_path / "missing.mtx")


@pytest.mark.parametrize("name", ["bcsstk18", "bcsstk38"])
def test_reference_fixtures(name, ref_lib):
    path = REF_DATA / f"{name}.mtx"
    if not path.exists():
        pytest.skip("the reference's data/ fixtures are not present")
    A = gen.read_mtx(path)
    assert _same(A, ref_lib.read_mtx(path))
    # the BAAS schedule of the real matrix, every exported array
    from baas_b200._native import FIELDS

    ours = Schedule(A, kind=KERNEL_ICCG, nthread=8)
    ref = ref_lib.Schedule(KERNEL_ICCG, A, 8).arrays()
    mine = ours.arrays()
    for f in FIELDS:
        assert np.array_equal(mine[f], ref[f]), f"{name} field {f}"
    # IC0: the oracle's restatement and the reference's serial routine agree bit for bit
    lu, _ = Port.ic0(A)
    assert np.array_equal(lu.view(np.int64), ref_lib.ic0_serial(A).view(np.int64))
    # the chunked sweep plan of the real matrix, run on the host, against the oracle
    L = gen.CSR(A.n, A.rowptr, A.colidx, lu).lower()
    U = L.transpose()
    b = gen.uniform_rhs(A.n, 1)
    assert np.array_equal(ours.emulate_sweep(L, b), Port.lower_solve(L, b))
    assert np.array_equal(ours.emulate_sweep(U, b, upper=True), Port.upper_solve(U, b, descending=True))
