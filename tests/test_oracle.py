"""The oracle (oracle/baas_oracle.c, our C restatement of the reference's serial numeric
routines) pinned against the golden vectors the reference produced (tests/golden/numeric.npz)
and, where it was built here, against the reference library itself (oracle/_ref)."""
from pathlib import Path

import numpy as np
import pytest

from baas_b200 import gen
from oracle.oracle import Port

GOLD = Path(__file__).resolve().parent / "golden" / "numeric.npz"


def _csr(z, pre):
    rp = z[f"{pre}_rowptr"]
    return gen.CSR(len(rp) - 1, rp, z[f"{pre}_colidx"], z[f"{pre}_values"])


def test_lower_sweep_bitexact_vs_golden():
    z = np.load(GOLD)
    L = _csr(z, "lower")
    x = Port.lower_solve(L, z["lower_b"])
    assert np.array_equal(x, z["lower_x_serial"])
    assert np.array_equal(x, z["lower_x_p2p"])  # the reference's p2p sweep equals its serial one


def test_ic0_and_sweeps_bitexact_vs_golden():
    z = np.load(GOLD)
    A = _csr(z, "ic")
    lu, bad = Port.ic0(A)
    assert bad == 0
    assert np.array_equal(lu, z["ic_lu_serial"])
    assert np.array_equal(lu, z["ic_lu_p2p"])
    Lf = gen.CSR(A.n, A.rowptr, A.colidx, lu).lower()
    Uf = gen.from_scipy(Lf.to_scipy().T.tocsr())
    y = Port.lower_solve(Lf, z["ic_r"])
    assert np.array_equal(y, z["ic_y"])
    zz = Port.upper_solve(Uf, y, descending=True)
    assert np.array_equal(zz, z["ic_z_p2p"])


def test_ilu0_bitexact_vs_golden():
    z = np.load(GOLD)
    C = _csr(z, "ilu")
    lu, bad = Port.ilu0(C)
    assert bad == 0
    assert np.array_equal(lu, z["ilu_lu_serial"])
    assert np.array_equal(lu, z["ilu_lu_p2p"])


def test_pcg_vs_golden():
    z = np.load(GOLD)
    P = gen.laplace3d(10, 1e-3)
    x, it, rel = Port.pcg(P, z["pcg_b"], tol=1e-10)
    assert abs(it - int(z["pcg_iters"][0])) <= 1
    assert rel < 1e-10
    assert np.linalg.norm(x - z["pcg_x"]) / np.linalg.norm(z["pcg_x"]) < 1e-9


def test_spmv_matches_scipy():
    A = gen.laplace3d(8, 1e-3)
    x = gen.uniform_rhs(A.n, 3)
    y = Port.spmv(A, x)
    assert np.allclose(y, A.to_scipy() @ x, rtol=1e-14, atol=1e-14)


@pytest.mark.parametrize("k", [20, 64])
def test_oracle_vs_live_reference(k, ref_lib):
    """Port and reference agree bit for bit on bigger inputs (sweep, IC0, ILU0)."""
    L, xt, b = gen.sptrsv_case(k, 0)
    assert np.array_equal(Port.lower_solve(L, b), ref_lib.sptrsv_serial(L, b))
    A = gen.laplace3d(k // 4, 1e-3)
    assert np.array_equal(Port.ic0(A)[0], ref_lib.ic0_serial(A))
    C = gen.convdiff3d(k // 4)
    assert np.array_equal(Port.ilu0(C)[0], ref_lib.ilu0_serial(C))
    U = L.to_scipy().T.tocsr()
    Uc = gen.from_scipy(U)
    assert np.array_equal(Port.upper_solve(Uc, b, descending=False), ref_lib.upper_serial(Uc, b))


def test_ic0_flags_nonpositive_pivots():
    # an indefinite matrix: IC0 leaves those diagonals unchanged (merge/IC.cpp:371-378)
    A = gen.laplace2d(6, diag=1.0)
    lu, bad = Port.ic0(A)
    assert bad > 0
    assert np.all(np.isfinite(lu))


def test_empty_offdiagonal_rows():
    # a diagonal matrix: every row has only its pivot
    import scipy.sparse as sp

    D = gen.from_scipy(sp.diags(np.arange(1.0, 11.0)).tocsr())
    b = np.arange(10.0)
    assert np.array_equal(Port.lower_solve(D, b), b / np.arange(1.0, 11.0))
    lu, bad = Port.ic0(D)
    assert bad == 0 and np.allclose(lu, np.sqrt(np.arange(1.0, 11.0)))
