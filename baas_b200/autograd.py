"""Differentiated ICCG: x = A(theta)^-1 b as a torch.autograd.Function.

Used for gradient checks only. The forward pass is `baas_iccg`. The backward pass is
`baas_iccg_adjoint`: it solves A^T lambda = dL/dx with the forward solve's IC0 factors and
writes the gradient on A's sparsity pattern, -lambda_i x_j, in the same launch. This module adds
only the chain rule of the parametrisation (face coefficients kappa = exp(theta) of a 7-point
diffusion operator) and dL/db = lambda.
"""
from __future__ import annotations

import numpy as np

from . import KERNEL_ICCG, PREC_FP32_FACTORS, DeviceCSR, Schedule, gen


def face_shapes(k: int):
    """Interior-face parameter shapes of gen.vardiff3d_faces: x, y and z faces (axis order z, y, x)."""
    return ((k, k, k - 1), (k, k - 1, k), (k - 1, k, k))


class FaceDiffusion3D:
    """7-point diffusion on k^3 with interior-face coefficients kappa = exp(theta) and unit
    Dirichlet boundary faces (the operator of gen.vardiff3d_faces). Holds the CSR pattern and,
    for every interior face (p, q), the positions of its four entries pp, qq, pq, qp."""

    def __init__(self, k: int, device="cuda"):
        import torch

        self.k = k
        ones = tuple(np.zeros(s) for s in face_shapes(k))
        A1 = gen.vardiff3d_faces(k, ones)  # every interior face kappa = 1
        n = A1.n
        self.n = n
        idx = np.arange(n).reshape(k, k, k)
        ps, qs = [], []
        for axis in (2, 1, 0):
            ps.append(idx.take(np.arange(k - 1), axis=axis).ravel())
            qs.append(idx.take(np.arange(1, k), axis=axis).ravel())
        p = np.concatenate(ps).astype(np.int64)
        q = np.concatenate(qs).astype(np.int64)
        rows = np.repeat(np.arange(n, dtype=np.int64), np.diff(A1.rowptr))
        keys = rows * n + A1.colidx.astype(np.int64)

        def pos(r, c):
            at = np.searchsorted(keys, r * n + c)
            assert np.all(keys[at] == r * n + c)
            return at

        self.pp, self.qq, self.pq, self.qp = pos(p, p), pos(q, q), pos(p, q), pos(q, p)
        base = A1.values.copy()  # boundary contributions only: remove the unit interior faces
        np.add.at(base, self.pp, -1.0)
        np.add.at(base, self.qq, -1.0)
        np.add.at(base, self.pq, 1.0)
        np.add.at(base, self.qp, 1.0)
        self.pattern = A1
        self.nfaces = len(p)
        t = lambda a: torch.from_numpy(a).to(device)  # noqa: E731
        self.d_pp, self.d_qq, self.d_pq, self.d_qp = t(self.pp), t(self.qq), t(self.pq), t(self.qp)
        self.d_base = t(base)
        self.d_rowptr = t(A1.rowptr)
        self.d_colidx = t(A1.colidx)

    def values(self, kappa):
        """A's values for face coefficients kappa (torch, flattened x, y, z faces)."""
        v = self.d_base.clone()
        v.index_add_(0, self.d_pp, kappa)
        v.index_add_(0, self.d_qq, kappa)
        v.index_add_(0, self.d_pq, -kappa)
        v.index_add_(0, self.d_qp, -kappa)
        return v

    def device_csr(self, values) -> DeviceCSR:
        return DeviceCSR(self.n, self.d_rowptr, self.d_colidx, values)

    def theta_grad(self, grad_a, kappa):
        """dL/dtheta_f = kappa_f (gA_pp + gA_qq - gA_pq - gA_qp) = -kappa_f (lam_p - lam_q)(x_p - x_q)."""
        return kappa * (grad_a[self.d_pp] + grad_a[self.d_qq] - grad_a[self.d_pq] - grad_a[self.d_qp])


class DiffIccg:
    """Holds the operator and one ICCG schedule; `solve(theta, b)` is differentiable in theta and b."""

    def __init__(self, op: FaceDiffusion3D, tol: float = 1e-10, maxiter: int = 4000,
                 precision: int = PREC_FP32_FACTORS, nthread: int = 8):
        self.op = op
        self.sched = Schedule(op.pattern, kind=KERNEL_ICCG, nthread=nthread)
        self.tol = tol
        self.maxiter = maxiter
        self.precision = precision
        self._solves = 0
        self._factored = -1  # number of the solve whose IC0 factors the schedule holds
        self.last_iters = (0, 0)

    def _solve(self, values, b):
        import torch

        x = torch.zeros_like(b)
        it, _ = self.sched.iccg(self.op.device_csr(values), b, x, tol=self.tol, maxiter=self.maxiter,
                                precision=self.precision)
        self._solves += 1
        self._factored = self._solves
        return x, it

    def solve(self, theta, b):
        return _IccgFn.apply(theta, b, self)


try:
    import torch

    class _IccgFn(torch.autograd.Function):
        @staticmethod
        def forward(ctx, theta, b, solver: DiffIccg):
            kappa = torch.exp(theta)
            values = solver.op.values(kappa)
            x, it = solver._solve(values, b)
            ctx.solver = solver
            ctx.token = solver._factored
            ctx.save_for_backward(kappa, values, x, b)
            ctx.fwd_iters = it
            return x

        @staticmethod
        def backward(ctx, gx):
            solver: DiffIccg = ctx.solver
            kappa, values, x, b = ctx.saved_tensors
            if solver._factored != ctx.token:
                # another solve ran on the schedule since: recompute this operator's factors
                solver._solve(values, b)
            lam = torch.empty_like(x)
            grad_a = torch.empty_like(values)
            it, _ = solver.sched.iccg_adjoint(solver.op.device_csr(values), gx.contiguous(), lam, x, grad_a,
                                              tol=solver.tol, maxiter=solver.maxiter, precision=solver.precision)
            solver.last_iters = (ctx.fwd_iters, it)
            return solver.op.theta_grad(grad_a, kappa), lam, None
except ImportError:  # torch is plumbing; the C ABI does not need it
    pass
