"""torch.autograd.Function over the B200 solver: the adjoint of x = A^{-1} b.

A is the HPL-AI matrix of a factored `hplai.Solver` context (generated from
its LCG seed; its FP32 LU factors live on the GPU).  The forward pass solves
A x = b through `hplai_solve_rhs`; the backward pass solves the adjoint
system A^T lambda = dL/dx through `hplai_solve_transpose` (U^T and L^T
solves, A^T regenerated in FP64), so dL/db = lambda and
dL/dA_ij = -lambda_i x_j.  The reference (RIKEN-RCCS/hpl-ai) has no
counterpart; this is the adjoint that its solve would need inside a
differentiable program.

    s = hplai.Solver(n, b); s.generate(42); s.factor()
    b = torch.tensor(..., dtype=torch.float64, requires_grad=True)
    x = hplai_torch.solve(b, s)
    loss = (xt * x).sum(); loss.backward()      # b.grad = A^{-T} xt
"""
from __future__ import annotations

import numpy as np
import torch

import hplai


def _to_host(t: torch.Tensor) -> np.ndarray:
    return np.ascontiguousarray(t.detach().to("cpu", torch.float64).numpy())


class SolveFunction(torch.autograd.Function):
    """x = A^{-1} b; backward: grad_b = A^{-T} grad_x."""

    @staticmethod
    def forward(ctx, b: torch.Tensor, solver: "hplai.Solver", maxit: int = 50):
        x, res = solver.solve_rhs(_to_host(b), maxit)
        if res.status != hplai.HPLAI_OK:
            raise hplai.HplaiError(res.status, "hplai_solve_rhs")
        ctx.solver = solver
        ctx.maxit = maxit
        out = torch.from_numpy(x).to(b.device)
        ctx.save_for_backward(out)
        return out

    @staticmethod
    def backward(ctx, grad_x: torch.Tensor):
        lam, res = ctx.solver.solve_transpose(_to_host(grad_x), ctx.maxit)
        if res.status != hplai.HPLAI_OK:
            raise hplai.HplaiError(res.status, "hplai_solve_transpose")
        return torch.from_numpy(lam).to(grad_x.device), None, None


def solve(b: torch.Tensor, solver: "hplai.Solver", maxit: int = 50) -> torch.Tensor:
    """Differentiable x = A^{-1} b with the context's matrix."""
    return SolveFunction.apply(b, solver, maxit)


def matrix_grad_entries(lam, x, rows, cols) -> np.ndarray:
    """dL/dA_ij = -lambda_i x_j at the sampled (rows[k], cols[k])."""
    lam = np.asarray(lam, dtype=np.float64)
    x = np.asarray(x, dtype=np.float64)
    return -lam[np.asarray(rows)] * x[np.asarray(cols)]
