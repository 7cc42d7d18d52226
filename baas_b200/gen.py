"""Seeded synthetic matrices for the five workloads of the sparse hot path.

The reference ships no generators for these shapes (spm/Laplacian.cpp only has an unused
27-point Laplacian), so these are this project's own. Every generator is deterministic for a
given seed (numpy PCG64 via ``default_rng``) and returns a :class:`CSR` with int32 indices,
float64 values and strictly ascending column indices in every row -- the layout of the
reference's ``SPM::CSR`` (spm/include/CSR.hpp:16-31), whose diagonal pointer is "first
column >= row" (spm/CSR.cpp:853-870).
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np
import scipy.sparse as sp


@dataclass
class CSR:
    n: int
    rowptr: np.ndarray  # int32 [n+1]
    colidx: np.ndarray  # int32 [nnz]
    values: np.ndarray  # float64 [nnz]

    @property
    def nnz(self) -> int:
        return int(self.rowptr[-1])

    def diagptr(self) -> np.ndarray:
        """Index of the first entry with column >= row (spm/CSR.cpp:853-870)."""
        rows = np.repeat(np.arange(self.n, dtype=np.int64), np.diff(self.rowptr))
        ge = self.colidx >= rows
        first = np.full(self.n, -1, dtype=np.int64)
        idx = np.nonzero(ge)[0]
        r = rows[idx]
        # first index per row among entries with col >= row
        keep = np.ones(len(idx), dtype=bool)
        keep[1:] = r[1:] != r[:-1]
        first[r[keep]] = idx[keep]
        return first.astype(np.int32)

    def to_scipy(self) -> sp.csr_matrix:
        return sp.csr_matrix((self.values, self.colidx, self.rowptr), shape=(self.n, self.n))

    def lower(self) -> "CSR":
        """Lower triangle incl. diagonal, diagonal last in each row."""
        return from_scipy(sp.tril(self.to_scipy(), format="csr"))

    def upper(self) -> "CSR":
        """Upper triangle incl. diagonal, diagonal first in each row."""
        return from_scipy(sp.triu(self.to_scipy(), format="csr"))

    def transpose(self) -> "CSR":
        """A^T in CSR (for an IC0 factor L: U = L^T, diagonal first in each row)."""
        return from_scipy(self.to_scipy().T.tocsr())

    def permuted(self, perm: np.ndarray) -> "CSR":
        """Symmetric permutation P A P^T with new row i = old row perm[i]."""
        m = self.to_scipy()[perm][:, perm]
        return from_scipy(m)


def from_scipy(m) -> CSR:
    m = sp.csr_matrix(m)
    m.sum_duplicates()
    m.sort_indices()
    return CSR(
        n=m.shape[0],
        rowptr=np.ascontiguousarray(m.indptr, dtype=np.int32),
        colidx=np.ascontiguousarray(m.indices, dtype=np.int32),
        values=np.ascontiguousarray(m.data, dtype=np.float64),
    )


def _lap1d(k: int) -> sp.csr_matrix:
    return sp.diags([-np.ones(k - 1), -np.ones(k - 1)], [-1, 1], shape=(k, k), format="csr")


def laplace2d(k: int, diag: float = 4.0) -> CSR:
    """5-point Laplacian on a k x k grid, natural (row-major) order, -1 off-diagonals."""
    e = sp.identity(k, format="csr")
    off = sp.kron(e, _lap1d(k)) + sp.kron(_lap1d(k), e)
    return from_scipy(off + diag * sp.identity(k * k, format="csr"))


def laplace3d(k: int, shift: float = 0.0) -> CSR:
    """7-point Laplacian on a k^3 grid, natural order, diagonal 6 + shift."""
    e = sp.identity(k, format="csr")
    off = (sp.kron(sp.kron(e, e), _lap1d(k)) + sp.kron(sp.kron(e, _lap1d(k)), e)
           + sp.kron(sp.kron(_lap1d(k), e), e))
    return from_scipy(off + (6.0 + shift) * sp.identity(k ** 3, format="csr"))


def sptrsv_case(k: int = 128, seed: int = 0):
    """Lower triangle of the 2-D 5-point Laplacian (k x k), x_true ~ U(-1,1), b = L x_true."""
    L = laplace2d(k).lower()
    rng = np.random.default_rng(seed)
    x_true = rng.uniform(-1.0, 1.0, L.n)
    b = L.to_scipy() @ x_true
    return L, x_true, b


def random_symmetric_permutation(n: int, seed: int) -> np.ndarray:
    return np.random.default_rng(seed).permutation(n).astype(np.int32)


# Configuration 2: the 64^3 7-point Laplacian with diagonal shift 1e-3, in natural order and under
# a seeded random symmetric permutation; right-hand side b ~ U(-1, 1) with seed 1.
C2_GRID = 64
C2_SHIFT = 1e-3
C2_PERMUTATION_SEED = 1
C2_RHS_SEED = 1


def c2_system(permuted: bool = False, k: int = C2_GRID) -> CSR:
    """The configuration-2 matrix, natural order or P A P^T with the seeded permutation."""
    A = laplace3d(k, C2_SHIFT)
    return A.permuted(random_symmetric_permutation(A.n, C2_PERMUTATION_SEED)) if permuted else A


def convdiff3d(k: int, velocity=(1.0, 0.5, 0.25), peclet: float = 10.0) -> CSR:
    """Nonsymmetric 7-point convection-diffusion on a k^3 grid (Dirichlet boundary).

    Unit diffusion, first-order upwind convection; the cell Peclet number of the fastest
    direction is `peclet` (c_d = peclet * v_d / max|v| in units of D/h). Scaled by h^2/D:
    diagonal 6 + sum|c_d|, upwind neighbour -(1 + |c_d|), downwind neighbour -1.
    """
    v = np.asarray(velocity, dtype=np.float64)
    c = peclet * v / np.max(np.abs(v))
    e = sp.identity(k, format="csr")
    ones = np.ones(k - 1)

    def axis_op(cd):
        # upwind for cd > 0: the (i-1) neighbour carries the convective flux
        lo = -(1.0 + max(cd, 0.0)) * ones
        hi = -(1.0 + max(-cd, 0.0)) * ones
        return sp.diags([lo, hi], [-1, 1], shape=(k, k), format="csr")

    ax, ay, az = (axis_op(c[0]), axis_op(c[1]), axis_op(c[2]))
    off = (sp.kron(sp.kron(e, e), ax) + sp.kron(sp.kron(e, ay), e) + sp.kron(sp.kron(az, e), e))
    diag = 6.0 + np.sum(np.abs(c))
    return from_scipy(off + diag * sp.identity(k ** 3, format="csr"))


def gaussian_field(shape, sigma: float, corr_len: float, seed: int) -> np.ndarray:
    """Stationary Gaussian random field: white noise filtered by a Gaussian kernel of
    standard deviation `corr_len` cells (FFT, periodic), rescaled to std `sigma`."""
    rng = np.random.default_rng(seed)
    w = rng.standard_normal(shape)
    freqs = [np.fft.fftfreq(s) for s in shape]
    grids = np.meshgrid(*freqs, indexing="ij")
    k2 = sum(g * g for g in grids)
    filt = np.exp(-2.0 * (np.pi ** 2) * (corr_len ** 2) * k2)
    f = np.real(np.fft.ifftn(np.fft.fftn(w) * filt))
    f -= f.mean()
    std = f.std()
    return f * (sigma / std if std > 0 else 0.0)


def vardiff2d(k: int, seed: int, sigma: float = 1.0, corr_len: float = 8.0) -> CSR:
    """SPD 5-point variable-coefficient diffusion on a k x k grid, kappa = exp(g) per cell,
    face coefficient = harmonic mean of the two cells, Dirichlet boundary (boundary faces use
    the cell's own kappa)."""
    g = gaussian_field((k, k), sigma, corr_len, seed)
    kap = np.exp(g)
    n = k * k
    idx = np.arange(n).reshape(k, k)
    rows, cols, vals = [], [], []
    diag = np.zeros(n)
    for axis in (0, 1):
        a = kap.take(np.arange(k - 1), axis=axis)
        b = kap.take(np.arange(1, k), axis=axis)
        face = 2.0 * a * b / (a + b)
        i0 = idx.take(np.arange(k - 1), axis=axis).ravel()
        i1 = idx.take(np.arange(1, k), axis=axis).ravel()
        f = face.ravel()
        rows += [i0, i1]
        cols += [i1, i0]
        vals += [-f, -f]
        np.add.at(diag, i0, f)
        np.add.at(diag, i1, f)
        # Dirichlet faces on both ends of this axis
        first = idx.take([0], axis=axis).ravel()
        last = idx.take([k - 1], axis=axis).ravel()
        np.add.at(diag, first, kap.take([0], axis=axis).ravel())
        np.add.at(diag, last, kap.take([k - 1], axis=axis).ravel())
    rows.append(np.arange(n))
    cols.append(np.arange(n))
    vals.append(diag)
    m = sp.coo_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))), shape=(n, n))
    return from_scipy(m)


def vardiff3d_faces(k: int, theta_faces) -> CSR:
    """SPD 7-point diffusion on k^3 with face coefficients kappa = exp(theta); theta_faces is a
    tuple of three arrays of interior-face parameters, shapes (k,k,k-1), (k,k-1,k), (k-1,k,k)
    for the x, y, z faces (axis order z, y, x), plus unit Dirichlet boundary faces."""
    n = k ** 3
    idx = np.arange(n).reshape(k, k, k)
    rows, cols, vals = [], [], []
    diag = np.full(n, 0.0)
    for axis, th in zip((2, 1, 0), theta_faces):
        f = np.exp(th).ravel()
        i0 = idx.take(np.arange(k - 1), axis=axis).ravel()
        i1 = idx.take(np.arange(1, k), axis=axis).ravel()
        rows += [i0, i1]
        cols += [i1, i0]
        vals += [-f, -f]
        np.add.at(diag, i0, f)
        np.add.at(diag, i1, f)
        np.add.at(diag, idx.take([0], axis=axis).ravel(), 1.0)
        np.add.at(diag, idx.take([k - 1], axis=axis).ravel(), 1.0)
    rows.append(np.arange(n))
    cols.append(np.arange(n))
    vals.append(diag)
    m = sp.coo_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))), shape=(n, n))
    return from_scipy(m)


def knn_stiffness(nodes: int = 4000, k: int = 12, seed: int = 3) -> CSR:
    """SPD stiffness-like matrix, 3 dof per node on a random 3-D mutual-k-NN graph.

    Nodes uniform in the unit cube; nodes i, j are coupled when each is among the other's k
    nearest neighbours. Each coupling adds -w_ij to the (i,d),(j,d) entries (same dof) and
    +w_ij to both diagonals; each node carries a random SPD 3x3 diagonal block; a diagonal
    shift keeps the matrix strictly diagonally dominant. n = 3 * nodes.
    """
    from scipy.spatial import cKDTree

    rng = np.random.default_rng(seed)
    pts = rng.uniform(0.0, 1.0, (nodes, 3))
    tree = cKDTree(pts)
    _, nb = tree.query(pts, k=k + 1)
    nb = nb[:, 1:]
    pairs = set()
    nbset = [set(r.tolist()) for r in nb]
    for i in range(nodes):
        for j in nb[i]:
            j = int(j)
            if i in nbset[j] and i < j:
                pairs.add((i, j))
    pairs = np.array(sorted(pairs), dtype=np.int64).reshape(-1, 2)
    w = rng.uniform(0.5, 1.5, len(pairs))
    n = 3 * nodes
    rows, cols, vals = [], [], []
    diag = np.zeros(n)
    for d in range(3):
        a = 3 * pairs[:, 0] + d
        b = 3 * pairs[:, 1] + d
        rows += [a, b]
        cols += [b, a]
        vals += [-w, -w]
        np.add.at(diag, a, w)
        np.add.at(diag, b, w)
    # random SPD 3x3 blocks
    blk = rng.standard_normal((nodes, 3, 3))
    blk = np.einsum("nij,nkj->nik", blk, blk) / 3.0
    base = 3 * np.arange(nodes)
    for r in range(3):
        for c in range(3):
            rows.append(base + r)
            cols.append(base + c)
            vals.append(blk[:, r, c] + (diag[base + r] + 1.0 if r == c else 0.0))
    m = sp.coo_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))), shape=(n, n)).tocsr()
    # strict diagonal dominance
    absrow = np.asarray(abs(m).sum(axis=1)).ravel() - np.abs(m.diagonal())
    shift = np.maximum(absrow - m.diagonal(), 0.0) + 1e-2
    m = m + sp.diags(shift)
    return from_scipy(m)


def uniform_rhs(n: int, seed: int, nrhs: int = 1) -> np.ndarray:
    rng = np.random.default_rng(seed)
    out = rng.uniform(-1.0, 1.0, (nrhs, n))
    return out[0] if nrhs == 1 else out


def normal_rhs(n: int, seed: int, nrhs: int = 1) -> np.ndarray:
    rng = np.random.default_rng(seed)
    out = rng.standard_normal((nrhs, n))
    return out[0] if nrhs == 1 else out


def batch_vardiff2d(nsys: int = 64, kmin: int = 64, kmax: int = 512, seed: int = 4) -> list:
    """Batched configuration: nsys SPD 2-D 5-point variable-coefficient diffusion systems with grid
    sizes k ~ U[kmin, kmax] (seeded), kappa = exp(g), g a Gaussian field (sigma 1, correlation
    length 8 cells), each with its own field seed."""
    rng = np.random.default_rng(seed)
    ks = rng.integers(kmin, kmax + 1, size=nsys)
    return [vardiff2d(int(k), seed=seed * 1000 + j) for j, k in enumerate(ks)]


def read_mtx(path) -> CSR:
    """A coordinate MatrixMarket file as a CSR, through the library's reader
    (baas_csr_read_mtx: symmetric storage expanded, each row sorted by column)."""
    import ctypes as C

    from . import _native

    m = _native.BaasCsr()
    _native.check(_native.lib().baas_csr_read_mtx(str(path).encode(), C.byref(m)), "baas_csr_read_mtx")
    try:
        n, nnz = m.n, m.nnz
        rowptr = np.ctypeslib.as_array(C.cast(m.rowptr, C.POINTER(C.c_int32)), shape=(n + 1,)).copy()
        colidx = np.ctypeslib.as_array(C.cast(m.colidx, C.POINTER(C.c_int32)), shape=(max(nnz, 1),))[:nnz].copy()
        values = np.ctypeslib.as_array(C.cast(m.values, C.POINTER(C.c_double)), shape=(max(nnz, 1),))[:nnz].copy()
    finally:
        _native.lib().baas_csr_free(C.byref(m))
    return CSR(n, rowptr, colidx, values)


def write_mtx(A: CSR, path, symmetric: bool = False, field: str = "real") -> None:
    """Write A as a coordinate MatrixMarket file: every entry ('general'), or the lower triangle
    with 'symmetric' storage. Values are written with 17 significant digits, so a read gives back
    the same doubles."""
    rows = np.repeat(np.arange(A.n), np.diff(A.rowptr))
    keep = rows >= A.colidx if symmetric else np.ones(A.nnz, dtype=bool)
    r, c, v = rows[keep], A.colidx[keep], A.values[keep]
    with open(path, "w") as f:
        f.write(f"%%MatrixMarket matrix coordinate {field} {'symmetric' if symmetric else 'general'}\n")
        f.write("% written by baas_b200.gen.write_mtx\n")
        f.write(f"{A.n} {A.n} {len(r)}\n")
        if field == "pattern":
            for i, j in zip(r, c):
                f.write(f"{i + 1} {j + 1}\n")
        else:
            for i, j, x in zip(r, c, v):
                f.write(f"{i + 1} {j + 1} {x:.17g}\n")
