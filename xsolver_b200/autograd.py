"""torch.autograd.Function over the hand-written adjoint (ctypes).

    x = SparseSolve.apply(values, b, solver)

solves A(values) x = b with a ``Solver`` (its matrix pattern is fixed; the
values tensor replaces A's stored values) and, in backward, returns
dL/dvalues (on A's sparsity pattern, CSR order) and dL/db from
xs_adjoint: A^T lambda = dL/dx, dL/db = lambda, dL/dA_ij = -lambda_i x_j.
Tensors are float64 CPU tensors (the data crosses the C ABI as host arrays).
"""
from __future__ import annotations

import numpy as np
import torch

from .api import Solver
from .stencils import CSRMatrix


class SparseSolve(torch.autograd.Function):
    @staticmethod
    def forward(ctx, values: torch.Tensor, b: torch.Tensor, solver: Solver):
        A = solver.A
        vals = values.detach().cpu().numpy().astype(np.float64)
        if not np.array_equal(vals, A.val):
            # same pattern, new values: rebuild the handle's matrix
            newA = CSRMatrix(A.n, A.rowptr, A.colidx, vals, A.name)
            solver.close()
            solver.__init__(newA)  # type: ignore[misc]
            for step in getattr(solver, "_config", []):
                step()
        x = solver.solve(b.detach().cpu().numpy())
        ctx.solver = solver
        ctx.save_for_backward(values, b)
        return torch.from_numpy(x)

    @staticmethod
    def backward(ctx, gx):
        solver = ctx.solver
        db, dA = solver.adjoint(gx.detach().cpu().numpy().astype(np.float64))
        return torch.from_numpy(dA), torch.from_numpy(db), None


def configured_solver(A: CSRMatrix, ksp="cg", pc="ilu0", tol=1e-12, maxiter=2000, restart=0) -> Solver:
    """A Solver whose configuration is replayed when SparseSolve swaps values."""
    s = Solver(A)

    def cfg():
        s.ksp_settype(ksp)
        s.ksp_setoption(tol, maxiter, restart)
        s.pc_settype(pc)

    cfg()
    s._config = [cfg]
    return s
