"""Adjoint gradient of a PDE-constrained misfit over the multigrid solver (no counterpart in
the reference).

Problem: -div(exp(m) grad u) = f on a box with homogeneous Dirichlet data, continuous FE_Q(p),
the log-coefficient m given at the (p+1)^3 Gauss points of every cell;
J(m) = 1/2 ||u(m) - u_d||^2_{L2} = 1/2 (u - u_d)^T M (u - u_d).
dJ/dm_q = -exp(m_q) grad lambda_q^T G_q grad u_q with A(m) lambda = M (u - u_d).

Everything runs in libpmg_b200.so (FP64 CG with the mixed-precision multigrid preconditioner,
the mass matrix, the per-point form); this module only wires it to torch.autograd:

    problem = AdjointPoisson(box, degree=4)
    m = fourier_field(problem.quadrature_points(), seed=1)        # [C, nq^3]
    u_d = problem.solve(fourier_field(problem.quadrature_points(), seed=2))
    m.requires_grad_(True)
    J = misfit(m, problem, u_d)
    J.backward()                                                   # m.grad = dJ/dm
"""
from __future__ import annotations

import math

import numpy as np

from . import (COEFF_VALUES, F32, F64, GEOMETRY_AUTO, Box, Hierarchy, MassOperator, adjoint_gradient,
               solve_cg)


def fourier_modes(seed: int, n_modes: int = 16, kmax: int = 4):
    """Wave vectors k_j in {1..kmax}^3, phases phi_j ~ U[0, 2 pi), amplitudes a_j ~ N(0, 1)
    (Box-Muller) from a seeded PCG64 stream."""
    rng = np.random.Generator(np.random.PCG64(seed))
    k = rng.integers(1, kmax + 1, size=(n_modes, 3)).astype(np.float64)
    phi = rng.random(n_modes) * 2.0 * math.pi
    u1, u2 = 1.0 - rng.random(n_modes), rng.random(n_modes)
    a = np.sqrt(-2.0 * np.log(u1)) * np.cos(2.0 * math.pi * u2)
    return k, phi, a


def fourier_field(xq, seed: int, n_modes: int = 16, kmax: int = 4, std: float = 0.5):
    """m(x) = sum_j a_j sin(pi k_j . x + phi_j) at the points xq [..., 3] (numpy array or torch
    tensor), rescaled so that its standard deviation over the given points is `std`."""
    k, phi, a = fourier_modes(seed, n_modes, kmax)
    if hasattr(xq, "is_cuda"):
        import torch
        kt = torch.as_tensor(k, dtype=xq.dtype, device=xq.device)
        arg = math.pi * torch.einsum("...d,jd->...j", xq, kt) + torch.as_tensor(phi, dtype=xq.dtype,
                                                                               device=xq.device)
        m = (torch.sin(arg) * torch.as_tensor(a, dtype=xq.dtype, device=xq.device)).sum(-1)
        return m * (std / m.std(unbiased=False))
    arg = math.pi * np.einsum("...d,jd->...j", xq, k) + phi
    m = (np.sin(arg) * a).sum(-1)
    return m * (std / m.std())


class AdjointPoisson:
    """-div(exp(m) grad u) = f with the ph-multigrid preconditioned FP64 CG of `Hierarchy`
    (coefficient values on every level, coarser levels interpolated) and the FP64 mass matrix
    for the misfit.  f_kind selects the right-hand side of pmg_operator_assemble_rhs."""

    def __init__(self, box: Box, degree: int = 4, pseq=None, mg_dtype=F32, cheb_degree=4,
                 f_kind: int = 0, reduce: float = 1e-13, max_iterations: int = 200, device: int = 0):
        pseq = pseq if pseq is not None else sorted({degree, max(1, degree // 2), 1}, reverse=True)
        self.degree = degree
        self.reduce = reduce
        self.max_iterations = max_iterations
        self.h = Hierarchy(box, pseq, mg_dtype=mg_dtype, cheb_degree=cheb_degree, geometry=GEOMETRY_AUTO,
                           coeff_kind=COEFF_VALUES, device=device)
        self.A = self.h.fine64
        self.M = MassOperator(self.A.mesh, degree, F64, device=device)
        self.b = self.A.assemble_rhs(f_kind)
        self.last_info = {}

    def quadrature_points(self):
        return self.A.quadrature_points()

    def set_parameter(self, m):
        """Load exp(m) into the CG matrix and every multigrid level."""
        import torch
        kappa = torch.exp(m.detach().to(torch.float64)).contiguous()
        self.h.set_coefficient(kappa)

    def solve(self, m, x0=None):
        """u(m), FP64 CUDA tensor."""
        self.set_parameter(m)
        u = self.A.initialize_dof_vector() if x0 is None else x0.clone()
        info = solve_cg(self.A, u, self.b, self.h.mg, self.reduce, 1e-300, self.max_iterations)
        self.last_info["forward"] = info
        return u

    def objective(self, m, u_d):
        """(J, u) for the log-coefficient m."""
        import torch
        u = self.solve(m)
        e = u - u_d
        r = torch.empty_like(e)
        self.M.vmult(r, e)
        return 0.5 * float(torch.dot(e, r)), u

    def gradient(self, m, u_d, u=None):
        """(J, dJ/dm [C, nq^3], u)."""
        if u is None:
            u = self.solve(m)
        else:
            self.set_parameter(m)
        J, g, _, info = adjoint_gradient(self.A, self.M, u, u_d, self.h.mg, self.reduce, 1e-300,
                                         self.max_iterations)
        self.last_info["adjoint"] = info
        return J, g, u


def _misfit_function():
    import torch

    class MisfitFunction(torch.autograd.Function):
        """J(m) forward (one solve), dJ/dm backward (one adjoint solve + the per-point kernel)."""

        @staticmethod
        def forward(ctx, m, problem, u_d):
            J, u = problem.objective(m, u_d)
            ctx.problem = problem
            ctx.save_for_backward(m, u, u_d)
            return torch.tensor(J, dtype=torch.float64, device=m.device)

        @staticmethod
        def backward(ctx, grad_out):
            m, u, u_d = ctx.saved_tensors
            _, g, _ = ctx.problem.gradient(m, u_d, u=u)
            return grad_out * g.to(m.dtype), None, None

    return MisfitFunction


_MISFIT = None


def misfit(m, problem: AdjointPoisson, u_d):
    """Differentiable J(m) = 1/2 ||u(m) - u_d||^2_{L2}."""
    global _MISFIT
    if _MISFIT is None:
        _MISFIT = _misfit_function()
    return _MISFIT.apply(m, problem, u_d)
