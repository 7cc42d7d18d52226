"""Differentiated ICCG: the adjoint kernel (baas_iccg_adjoint) against central finite differences
and against an FP64 CPU gradient built on the oracle's PCG.

Problem: 7-point diffusion on k^3 with interior-face coefficients kappa = exp(theta), theta a
seeded Gaussian field (sigma = 0.5); FP64 CG with FP32 IC0 factors; loss
L = 1/2 ||x - x_obs||^2 with x_obs the solution for a perturbed theta plus N(0, 1e-3) noise.
"""
import numpy as np
import pytest

from baas_b200 import PREC_FP32_FACTORS, PREC_FP64, gen

pytestmark = pytest.mark.gpu


def _theta(k, seed, sigma=0.5):
    from baas_b200.autograd import face_shapes

    parts = []
    for j, shp in enumerate(face_shapes(k)):
        parts.append(gen.gaussian_field(shp, sigma, 4.0, seed + j).ravel())
    return np.concatenate(parts)


def _problem(k, precision, tol):
    import torch

    from baas_b200.autograd import DiffIccg, FaceDiffusion3D

    op = FaceDiffusion3D(k)
    solver = DiffIccg(op, tol=tol, maxiter=20000, precision=precision)
    theta = torch.from_numpy(_theta(k, 11)).cuda()
    b = torch.from_numpy(gen.uniform_rhs(op.n, 4)).cuda()
    with torch.no_grad():
        x_pert = solver.solve(theta + torch.from_numpy(_theta(k, 23, 0.1)).cuda(), b)
    noise = torch.from_numpy(np.random.default_rng(5).normal(0.0, 1e-3, op.n)).cuda()
    x_obs = x_pert + noise
    return op, solver, theta, b, x_obs


def _loss(solver, theta, b, x_obs):
    x = solver.solve(theta, b)
    return 0.5 * ((x - x_obs) ** 2).sum()


def test_adjoint_matches_central_differences_64():
    """32 random directions in (theta, b), h = 1e-6, relative error of the directional
    derivatives below 1e-6."""
    import torch

    op, solver, theta, b, x_obs = _problem(64, PREC_FP32_FACTORS, 1e-14)
    th = theta.clone().requires_grad_(True)
    bb = b.clone().requires_grad_(True)
    L = _loss(solver, th, bb, x_obs)
    L.backward()
    gth, gb = th.grad.detach(), bb.grad.detach()
    rng = np.random.default_rng(7)
    h = 1e-6
    ad, fd = [], []
    with torch.no_grad():
        x0 = solver.solve(theta, b)

        def perturbed(sign, vt, vb):
            # warm start from the unperturbed solution: the initial residual is O(h), so the
            # solver's error (relative to it) stays far below the O(h) change being measured
            x = x0.clone()
            vals = op.values(torch.exp(theta + sign * h * vt))
            solver.sched.iccg(op.device_csr(vals), b + sign * h * vb, x, tol=1e-12, maxiter=20000,
                              precision=PREC_FP32_FACTORS)
            return x

        for _ in range(32):
            vt = torch.from_numpy(rng.standard_normal(theta.numel())).cuda()
            vb = torch.from_numpy(rng.standard_normal(b.numel())).cuda()
            vt /= vt.norm()
            vb /= vb.norm()
            xp, xm = perturbed(1.0, vt, vb), perturbed(-1.0, vt, vb)
            # L(+) - L(-) = 1/2 (x+ - x-) . (x+ + x- - 2 x_obs), without cancelling two large losses
            fd.append(float(0.5 * ((xp - xm) * (xp + xm - 2.0 * x_obs)).sum() / (2 * h)))
            ad.append(float((gth * vt).sum() + (gb * vb).sum()))
    ad, fd = np.array(ad), np.array(fd)
    rel = np.linalg.norm(ad - fd) / np.linalg.norm(ad)
    assert rel < 1e-6, (rel, ad[:4], fd[:4])


def test_adjoint_matches_fp64_cpu_gradient_16():
    import torch

    from oracle.oracle import Port

    for precision in (PREC_FP64, PREC_FP32_FACTORS):
        op, solver, theta, b, x_obs = _problem(16, precision, 1e-12)
        th = theta.clone().requires_grad_(True)
        bb = b.clone().requires_grad_(True)
        _loss(solver, th, bb, x_obs).backward()
        # FP64 CPU reference: forward and adjoint PCG with the oracle, gradient by formula
        kappa = np.exp(theta.cpu().numpy())
        A = gen.CSR(op.n, op.pattern.rowptr, op.pattern.colidx, op.values(torch.from_numpy(kappa).cuda()).cpu().numpy())
        x, _, _ = Port.pcg(A, b.cpu().numpy(), tol=1e-14, maxiter=20000)
        g = x - x_obs.cpu().numpy()
        lam, _, _ = Port.pcg(A, g, tol=1e-14, maxiter=20000)
        Ak = A.to_scipy()
        # -kappa_f (lam_p - lam_q)(x_p - x_q) for each interior face
        rows = np.repeat(np.arange(op.n), np.diff(A.rowptr))
        p, q = rows[op.pq], A.colidx[op.pq]
        gth_ref = -kappa * (lam[p] - lam[q]) * (x[p] - x[q])
        e_th = np.linalg.norm(th.grad.cpu().numpy() - gth_ref) / np.linalg.norm(gth_ref)
        e_b = np.linalg.norm(bb.grad.cpu().numpy() - lam) / np.linalg.norm(lam)
        assert e_th < 1e-8 and e_b < 1e-8, (precision, e_th, e_b)
        assert Ak.shape == (op.n, op.n)


def test_adjoint_requires_factors():
    import torch

    from baas_b200 import BaasError, DeviceCSR, KERNEL_ICCG, Schedule

    A = gen.laplace3d(8, 1e-3)
    s = Schedule(A, kind=KERNEL_ICCG, nthread=4)
    dA = DeviceCSR.from_host(A)
    g = torch.ones(A.n, dtype=torch.float64, device="cuda")
    lam = torch.empty_like(g)
    with pytest.raises(BaasError) as e:
        s.iccg_adjoint(dA, g, lam)
    assert e.value.status_name == "BAAS_ERR_STATE"
    x = torch.zeros_like(g)
    s.iccg(dA, g, x, precision=PREC_FP64)
    with pytest.raises(BaasError):
        s.iccg_adjoint(dA, g, lam, precision=PREC_FP32_FACTORS)
    s.iccg_adjoint(dA, g, lam, precision=PREC_FP64)
    # A symmetric, g = b: the adjoint solution is the forward one
    assert torch.allclose(lam, x, rtol=1e-8, atol=1e-10)
