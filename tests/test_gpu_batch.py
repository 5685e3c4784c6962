"""Several right-hand sides in one iteration (xs_solve_batch, xs_adjoint_batch).

With PCG and an exact preconditioner solve, k right-hand sides iterate
together: one pass over the matrix and one triangular-solve dependency chain
serve all of them.  Row sums keep the single-column operations and order:
the batched LU solve equals xs_plan_lusolve column by column, bit for bit.
Dot products reduce in their own order, so a batched solve agrees with k
single solves (the reference's one-right-hand-side loop,
intel/mpisolver-C-v1.cpp:193-272 restated) to rounding: per column the
iteration count within +-1 and the solution within 1e-10 relative; the
residual history against the reference loop within the calibrated bound of
tests/parity.py (1e-10 wherever the reference's own dot order allows)."""
import numpy as np
import pytest

import oracle
from parity import history_ok, reference_with_bounds
from xsolver_b200 import stencils as st

pytestmark = pytest.mark.gpu


class batch_kernels:
    def __init__(self, enable):
        self.enable = enable

    def __enter__(self):
        from xsolver_b200 import _lib

        assert _lib.lib().xs_set_batch_kernels(self.enable) == 0

    def __exit__(self, *exc):
        from xsolver_b200 import _lib

        _lib.lib().xs_set_batch_kernels(1)


class tiles:
    def __init__(self, on, box=(8, 8, 8)):
        self.args = (1 if on else 0, *box, 8)

    def __enter__(self):
        from xsolver_b200 import _lib

        assert _lib.lib().xs_set_trsv_tiles(*self.args) == 0

    def __exit__(self, *exc):
        from xsolver_b200 import _lib

        _lib.lib().xs_set_trsv_tiles(1, 16, 16, 8, 65536)


@pytest.mark.parametrize("box_layout", [True, False])
@pytest.mark.parametrize("k", [3, 8])
def test_batched_lusolve_bitwise_per_column(cuda, k, box_layout):
    import torch
    from xsolver_b200.api import Plan

    A = st.varcoef3d_7pt(26, 1)
    with tiles(box_layout):
        P = Plan(A).factor("ilu0")
    X = np.stack([st.rhs_uniform(A.n, s) for s in range(k)], axis=1)  # (n, k)
    dX = torch.from_numpy(np.ascontiguousarray(X)).to(cuda)
    dZ = torch.zeros_like(dX)
    P.lusolve_batch(dX, dZ)
    P.sync()
    Z = dZ.cpu().numpy()
    z1 = torch.zeros(A.n, dtype=torch.float64, device=cuda)
    for c in range(k):
        xc = torch.from_numpy(np.ascontiguousarray(X[:, c])).to(cuda)
        P.lusolve(xc, z1)
        P.sync()
        assert np.array_equal(Z[:, c], z1.cpu().numpy()), c


def _pcg(A, pc="ilu0"):
    from xsolver_b200.api import Solver

    return Solver(A).ksp_settype("cgm").ksp_setoption(1e-12, 3000).pc_settype(pc)


@pytest.mark.parametrize("pc", ["ilu0", "jacobi", "ic0"])
@pytest.mark.parametrize("k", [2, 5, 8])
def test_batched_pcg_matches_single_solves(cuda, k, pc):
    A = st.varcoef3d_7pt(24, 3)
    B = np.stack([st.rhs_uniform(A.n, 10 + s) for s in range(k)])
    S = _pcg(A, pc)
    X = S.solve_batch(B)
    its = S.batch_iterations(k)
    with batch_kernels(0):
        for c in range(k):
            xs = S.solve(B[c])
            h1 = S.resvec()
            assert abs(int(its[c]) - S.usediter) <= 1, (c, its[c], S.usediter)
            assert np.linalg.norm(X[c] - xs) / np.linalg.norm(xs) < 1e-10, c
    # the handle's history is the last column's: against the reference loop
    # (the oracle's PCG with the same preconditioner) within the calibrated
    # bound of tests/parity.py, as the single solve is
    S2 = _pcg(A, pc)
    S2.solve_batch(B)
    hb = S2.resvec()
    F = {"ilu0": oracle.ilu0, "ic0": oracle.ic0}.get(pc)
    kw = dict(tol=1e-12, maxiter=3000, pc="lu", factors=F(A)) if F else dict(tol=1e-12, maxiter=3000, pc="jacobi")
    _, ho, uo, hbnd, _ = reference_with_bounds("cgm", A, B[k - 1], **kw)
    ok, worst = history_ok(hb[1:] / hb[0], ho, hbnd)
    assert ok, worst
    Asp = A.to_scipy()
    for c in range(k):
        assert np.linalg.norm(B[c] - Asp @ X[c]) / np.linalg.norm(B[c]) < 1e-11


def test_batched_pcg_with_box_layout_and_columns_converging_apart(cuda):
    """Box-scheduled triangular solves; one column has a zero right-hand
    side (done at iteration 0, stays zero) and one is a scaled copy of
    another: each column stops on its own, as its single solve does."""
    A = st.poisson3d_7pt(30)
    k = 4
    B = np.stack([st.rhs_uniform(A.n, s) for s in range(k)])
    B[2] = 1e-3 * B[0]
    B[3] = 0.0
    with tiles(True):
        S = _pcg(A)
        X = S.solve_batch(B)
    its = S.batch_iterations(k)
    assert its[3] == 0 and not X[3].any()
    with tiles(True), batch_kernels(0):
        S1 = _pcg(A)
        for c in range(3):
            xs = S1.solve(B[c])
            assert abs(int(its[c]) - S1.usediter) <= 1
            assert np.linalg.norm(X[c] - xs) / np.linalg.norm(xs) < 1e-10


def test_batched_adjoint_matches_single(cuda):
    A = st.varcoef3d_7pt(20, 5)
    n, k = A.n, 6
    rng = np.random.default_rng(1)
    B = np.stack([st.rhs_uniform(n, s) for s in range(k)])
    S = _pcg(A)
    X = S.solve_batch(B)
    G = X - rng.uniform(-1, 1, (k, n))
    DB, DA = S.adjoint_batch(X, G)
    with batch_kernels(0):
        DB1, DA1 = S.adjoint_batch(X, G)
    for c in range(k):
        assert np.linalg.norm(DB[c] - DB1[c]) / np.linalg.norm(DB1[c]) < 1e-10, c
        assert np.linalg.norm(DA[c] - DA1[c]) / np.linalg.norm(DA1[c]) < 1e-10, c
    rows = np.repeat(np.arange(n), np.diff(A.rowptr))
    for c in range(k):
        assert np.array_equal(DA[c], -DB[c][rows] * X[c][A.colidx])
