"""Mixed-precision iterative refinement and the adjoint.

Mixed: FP64 outer residual/update around an FP32 inner solve with FP32 /
BF16 / FP16 ILU factors; the refined solution must reach relative residual
1e-10 and agree with an FP64 solve converged to 1e-14.
Adjoint: dL/db and dL/dA from the transposed solve against central finite
differences (h = 1e-6, probe solves at 1e-14) and against the oracle's
transposed solve."""
import numpy as np
import pytest

import oracle
from xsolver_b200 import stencils as st

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("ksp,carry", [("bicgstab", True), ("bicgstab", False), ("gmres", False)])
@pytest.mark.parametrize("factor", ["fp32", "bf16", "fp16"])
def test_mixed_refinement_reaches_1e10(cuda, ksp, carry, factor):
    """carry: BiCGSTAB keeps one FP32 iteration across the refinement steps
    (residual replaced by the FP64 residual at each step) instead of
    restarting it."""
    from xsolver_b200.api import Solver

    A = st.poisson3d_7pt(40) if ksp == "bicgstab" else st.convdiff3d_27pt(20)
    b = st.rhs_uniform(A.n, 0, -1.0 if ksp == "bicgstab" else 0.0, 1.0)
    S = Solver(A).ksp_settype(ksp).ksp_setoption(1e-10, 2000, 30).pc_settype("ilu0")
    S.set_precision("fp64", "fp32", factor).set_inner(1e-4, 200).set_refinement_mode(carry)
    x = S.solve(b)
    r = b - A.to_scipy() @ x
    relres = np.linalg.norm(r) / np.linalg.norm(b)
    assert relres < 1e-10, relres
    assert S.outer_steps() >= 2
    ref = Solver(A).ksp_settype(ksp).ksp_setoption(1e-14, 4000, 30).pc_settype("ilu0").solve(b)
    err = np.linalg.norm(x - ref) / np.linalg.norm(ref)
    # the error is bounded by cond(A) * 1e-10; these systems are mildly conditioned
    assert err < 1e-7, err


def _loss_grad(x, xs):
    return x - xs


def test_adjoint_vs_finite_differences(cuda):
    """dL/dA and dL/db from the GPU adjoint against central finite
    differences with h = 1e-6.  The probe solves use a sparse direct LU on the
    host (deterministic, forward error far below an iterative 1e-14 solve),
    so the finite differences are not dominated by probe-solve noise."""
    import scipy.sparse as sp
    import scipy.sparse.linalg as sla
    from xsolver_b200.api import Solver

    A = st.varcoef3d_7pt(9, seed=4)
    n = A.n
    rng = np.random.default_rng(0)
    b = st.rhs_uniform(n, 1)
    xs = rng.uniform(-1, 1, n)
    S = Solver(A).ksp_settype("cg").ksp_setoption(1e-14, 4000).pc_settype("ilu0")
    x = S.solve(b)
    dLdb, dLdA = S.adjoint(_loss_grad(x, xs))

    def direct(vals, rhs):
        M = sp.csc_matrix(sp.csr_matrix((vals, A.colidx, A.rowptr), shape=(n, n)))
        return sla.splu(M).solve(rhs)

    # lambda itself against a direct transposed solve
    lam = direct(A.val, _loss_grad(direct(A.val, b), xs))  # A symmetric: A^T = A
    assert np.linalg.norm(dLdb - lam) / np.linalg.norm(lam) < 1e-9

    def dL(xp, xm):
        # L(x+) - L(x-) = 1/2 sum (x+ - x-)(x+ + x- - 2 x*)
        return 0.5 * np.sum((xp - xm) * (xp + xm - 2 * xs))

    def cd_A(k, h):
        vp = A.val.copy(); vp[k] += h
        vm = A.val.copy(); vm[k] -= h
        return dL(direct(vp, b), direct(vm, b)) / (2 * h)

    def cd_b(i, h):
        bp = b.copy(); bp[i] += h
        bm = b.copy(); bm[i] -= h
        return dL(direct(A.val, bp), direct(A.val, bm)) / (2 * h)

    # h = 1e-4: central differences are accurate to ~1e-8 here, so the
    # gradient must agree to 1e-6 relative.  h = 1e-6 (the target step): the
    # central difference itself carries ~1e-6 relative rounding noise on this
    # system (measured against the exact adjoint), so it is checked at 1e-5.
    for k in rng.choice(A.nnz, 48, replace=False):
        f4 = cd_A(k, 1e-4)
        assert abs(f4 - dLdA[k]) <= 1e-6 * max(abs(f4), 1e-3), (k, f4, dLdA[k])
        f6 = cd_A(k, 1e-6)
        assert abs(f6 - dLdA[k]) <= 1e-5 * max(abs(f6), 1e-3), (k, f6, dLdA[k])
    for i in rng.choice(n, 48, replace=False):
        f4 = cd_b(i, 1e-4)
        assert abs(f4 - dLdb[i]) <= 1e-6 * max(abs(f4), 1e-3), (i, f4, dLdb[i])
        f6 = cd_b(i, 1e-6)
        assert abs(f6 - dLdb[i]) <= 1e-5 * max(abs(f6), 1e-3), (i, f6, dLdb[i])


def test_adjoint_nonsymmetric_vs_oracle_transposed_solve(cuda):
    """On a nonsymmetric matrix, lambda must solve A^T lambda = g: compare
    with the oracle solving the explicitly transposed system."""
    from xsolver_b200.api import Solver

    A = st.convdiff3d_27pt(10)
    n = A.n
    b = st.rhs_uniform(n, 2, 0.0, 1.0)
    S = Solver(A).ksp_settype("gmres").ksp_setoption(1e-13, 2000, 30).pc_settype("ilu0")
    x = S.solve(b)
    g = st.rhs_uniform(n, 3)
    dLdb, dLdA = S.adjoint(g)
    At = A.to_scipy().T.tocsr()
    At.sort_indices()
    T = st.CSRMatrix(n, At.indptr, At.indices, At.data)
    lam, _, _ = oracle.solve("fgmres", T, g, tol=1e-13, maxiter=2000, restart=30, pc="lu", factors=oracle.ilu0(T),
                             quirk=0)
    assert np.linalg.norm(dLdb - lam) / np.linalg.norm(lam) < 1e-9
    rows = np.repeat(np.arange(n), np.diff(A.rowptr))
    assert np.allclose(dLdA, -dLdb[rows] * x[A.colidx], rtol=1e-12, atol=1e-14)


def test_adjoint_batch_matches_single(cuda):
    from xsolver_b200.api import Solver

    A = st.varcoef3d_7pt(8, seed=7)
    n = A.n
    S = Solver(A).ksp_settype("cg").ksp_setoption(1e-12, 2000).pc_settype("ilu0")
    B = np.stack([st.rhs_uniform(n, s) for s in range(3)])
    X = S.solve_batch(B)
    G = X - 0.5
    DB, DA = S.adjoint_batch(X, G)
    for k in range(3):
        S.solve(B[k])
        db, da = S.adjoint(G[k])
        assert np.allclose(DB[k], db, rtol=1e-12, atol=1e-15)
        assert np.allclose(DA[k], da, rtol=1e-12, atol=1e-15)


def test_adjoint_needs_a_valid_solution(cuda):
    """XS_ERR_ORDER (8) with no solution to differentiate through: before any
    solve, after a solve that ended with an error, and after new values
    replaced the ones the last solve used."""
    from xsolver_b200.api import Solver, XsError

    A = st.varcoef3d_7pt(6, seed=2)
    S = Solver(A).ksp_settype("cg").ksp_setoption(1e-12, 500).pc_settype("ilu0")
    g = st.rhs_uniform(A.n, 1)
    b = st.rhs_uniform(A.n, 2)
    with pytest.raises(XsError) as e:
        S.adjoint(g)
    assert e.value.code == 8
    b_nan = b.copy()
    b_nan[3] = np.nan
    with pytest.raises(XsError):
        S.solve(b_nan)
    with pytest.raises(XsError) as e:
        S.adjoint(g)
    assert e.value.code == 8
    S.solve(b)
    db, _ = S.adjoint(g)
    assert np.all(np.isfinite(db))
    S.mat_update(A.val * 2.0)
    with pytest.raises(XsError) as e:
        S.adjoint(g)
    assert e.value.code == 8
    S.solve(b)
    db2, _ = S.adjoint(g)  # A^T doubled: lambda halves
    assert np.allclose(db2, db / 2.0, rtol=1e-8, atol=1e-14)


def test_autograd_function(cuda):
    import torch
    from xsolver_b200.autograd import SparseSolve, configured_solver

    A = st.varcoef3d_7pt(6, seed=2)
    S = configured_solver(A, ksp="cg", pc="ilu0", tol=1e-14)
    vals = torch.tensor(A.val, dtype=torch.float64, requires_grad=True)
    b = torch.tensor(st.rhs_uniform(A.n, 0), dtype=torch.float64, requires_grad=True)
    x = SparseSolve.apply(vals, b, S)
    loss = 0.5 * (x ** 2).sum()
    loss.backward()
    # check against a dense solve
    Ad = torch.tensor(A.to_scipy().toarray(), dtype=torch.float64, requires_grad=True)
    bd = b.detach().clone().requires_grad_(True)
    xd = torch.linalg.solve(Ad, bd)
    (0.5 * (xd ** 2).sum()).backward()
    rows = np.repeat(np.arange(A.n), np.diff(A.rowptr))
    gA = Ad.grad.numpy()[rows, A.colidx]
    assert np.allclose(b.grad.numpy(), bd.grad.numpy(), rtol=1e-8, atol=1e-12)
    assert np.allclose(vals.grad.numpy(), gA, rtol=1e-8, atol=1e-12)


def test_unsorted_input_keeps_caller_entry_order(cuda):
    """Rows given with unsorted columns: the solve equals the sorted input's,
    dL/dA comes back in the caller's entry order, and xs_mat_update takes
    values in that order too."""
    from xsolver_b200.api import Solver

    A = st.convdiff3d_27pt(7)
    n = A.n
    rng = np.random.default_rng(5)
    perm = np.concatenate([A.rowptr[i] + rng.permutation(A.rowptr[i + 1] - A.rowptr[i]) for i in range(n)])
    U = st.CSRMatrix(n, A.rowptr.copy(), A.colidx[perm].copy(), A.val[perm].copy(), "unsorted")
    b = st.rhs_uniform(n, 4, 0.0, 1.0)
    g = st.rhs_uniform(n, 5)

    def run(M):
        S = Solver(M).ksp_settype("gmres").ksp_setoption(1e-12, 2000, 30).pc_settype("ilu0")
        x = S.solve(b)
        db, da = S.adjoint(g)
        v2 = M.val * 1.5  # scaled values in the matrix's own entry order
        S.mat_update(v2)
        x2 = S.solve(b)
        return x, db, da, x2

    xs, dbs, das, x2s = run(A)
    xu, dbu, dau, x2u = run(U)
    assert np.array_equal(xs, xu)
    assert np.array_equal(dbs, dbu)
    assert np.array_equal(das[perm], dau)
    assert np.array_equal(x2s, x2u)
    assert np.allclose(x2s, xs / 1.5, rtol=1e-9, atol=1e-12)
