"""The oracle (CPU restatement) is pinned to the reference's own CPU code:
bitwise against golden fixtures produced by the compiled reference
(tests/golden/make_golden.py) and, when present, against the compiled
reference itself."""
import os

import numpy as np
import pytest

import oracle
from xsolver_b200 import stencils as st

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def _load(name):
    return np.load(os.path.join(GOLD, name))


def _problems(z):
    names = sorted({k.split("/")[0] for k in z.files})
    for nm in names:
        A = st.CSRMatrix(len(z[f"{nm}/rowptr"]) - 1, z[f"{nm}/rowptr"], z[f"{nm}/colidx"], z[f"{nm}/val"], nm)
        yield nm, A


def _gmres_inner_view(glob_hist, used, m):
    """The intel GMRES writes resvec with the inner index (each restart cycle
    overwrites it); rebuild that view from the global-index history."""
    out = {}
    last_cycle = used // m
    for c in range(last_cycle + 1):
        for i in range(m):
            j = c * m + i
            if j < len(glob_hist):
                out[i] = glob_hist[j]
    return out


@pytest.mark.parametrize("method", ["cg", "cgm", "bicgstab", "gcr", "igcr", "gmres", "fgmres"])
def test_krylov_restatement_bitwise_vs_golden(method):
    z = _load("krylov_jacobi.npz")
    seen = 0
    for nm, A in _problems(z):
        key = f"{nm}/{method}/x"
        if key not in z.files:
            continue
        b = z[f"{nm}/rhs"]
        x, rv, used = oracle.solve(method, A, b, tol=1e-9, maxiter=400, restart=20, pc="jacobi")
        assert used == int(z[f"{nm}/{method}/usediter"]), (nm, method)
        assert np.array_equal(x, z[key]), (nm, method)
        ref_rv = z[f"{nm}/{method}/resvec"]
        if method in ("gmres", "fgmres"):
            view = _gmres_inner_view(rv, used, 20)
            for i, v in view.items():
                assert ref_rv[i] == v, (nm, method, i)
        else:
            assert np.array_equal(rv, ref_rv[: len(rv)]), (nm, method)
        seen += 1
    assert seen >= 1


def test_ilu0_restatement_bitwise_vs_golden():
    z = _load("ilu0.npz")
    for nm, A in _problems(z):
        assert np.array_equal(oracle.ilu0_values(A), z[f"{nm}/luv"]), nm


@pytest.mark.parametrize("method", ["icg", "icgm", "ibicgstab"])
def test_single_reduction_restatement_bitwise_vs_golden(method):
    """icg / icgm / ibicgstab with Jacobi against the compiled reference's
    recorded outputs (tests/golden/krylov_single_reduction.npz)."""
    z = _load("krylov_single_reduction.npz")
    seen = 0
    for nm, A in _problems(z):
        key = f"{nm}/{method}/x"
        if key not in z.files:
            continue
        x, rv, used = oracle.solve(method, A, z[f"{nm}/rhs"], tol=1e-9, maxiter=400, restart=20, pc="jacobi")
        assert used == int(z[f"{nm}/{method}/usediter"]), (nm, method)
        assert np.array_equal(x, z[key]), (nm, method)
        assert np.array_equal(rv, z[f"{nm}/{method}/resvec"][: len(rv)]), (nm, method)
        seen += 1
    assert seen >= 3


def test_ic0_restatement_bitwise_vs_golden():
    """IC(0) against the compiled reference's ic0_csr_A recorded in
    tests/golden/ic0.npz (Precond_ic0 defaults)."""
    z = _load("ic0.npz")
    seen = 0
    for nm, A in _problems(z):
        assert np.array_equal(oracle.ic0_values(A), z[f"{nm}/luv"]), nm
        seen += 1
    assert seen == 4


@pytest.mark.skipif(oracle.ref_intel() is None, reason="compiled reference not present")
@pytest.mark.parametrize("method", ["cg", "cgm", "icg", "icgm", "bicgstab", "ibicgstab", "gcr", "igcr", "gmres", "fgmres"])
def test_krylov_restatement_bitwise_vs_compiled_reference(method):
    A = st.poisson2d_5pt(20)
    b = st.rhs_uniform(A.n, 11)
    xr, rr, ur = oracle.ref_solve(method, A, b, tol=1e-8, maxiter=300, restart=25)
    xo, ro, uo = oracle.solve(method, A, b, tol=1e-8, maxiter=300, restart=25, pc="jacobi")
    assert ur == uo
    assert np.array_equal(xr, xo)
    if method not in ("gmres", "fgmres"):
        assert np.array_equal(rr[: len(ro)], ro)


EDGE_CASES = {
    # zero right-hand side (res0 = 0), a single iteration, a restart longer
    # than the iteration budget, and a non-zero initial guess
    "zero-b": (lambda n: np.zeros(n), None, dict(tol=1e-8, maxiter=50, restart=10)),
    "maxiter1": (lambda n: st.rhs_uniform(n, 1), None, dict(tol=1e-8, maxiter=1, restart=10)),
    "restart>maxiter": (lambda n: st.rhs_uniform(n, 2), None, dict(tol=1e-8, maxiter=7, restart=30)),
    "x0": (lambda n: st.rhs_uniform(n, 3), lambda n: st.rhs_uniform(n, 9), dict(tol=1e-8, maxiter=40, restart=5)),
}


@pytest.mark.skipif(oracle.ref_intel() is None, reason="compiled reference not present")
@pytest.mark.parametrize("case", sorted(EDGE_CASES))
@pytest.mark.parametrize("method", ["cg", "cgm", "icg", "icgm", "bicgstab", "ibicgstab", "gcr", "igcr", "gmres", "fgmres"])
def test_krylov_restatement_edge_cases_vs_compiled_reference(method, case):
    """The restated intel/ loops equal the compiled ones bitwise on the
    edge cases a caller can hit: count, solution and (outside GMRES's
    inner-index history) the residual history."""
    rhs, x0f, kw = EDGE_CASES[case]
    mats = [st.poisson2d_5pt(12)]
    if method not in ("cg", "cgm", "icg", "icgm"):
        mats.append(st.convdiff3d_27pt(5, pe=5.0))
    for A in mats:
        b = rhs(A.n)
        x0 = x0f(A.n) if x0f else None
        xr, rr, ur = oracle.ref_solve(method, A, b, x0=x0, **kw)
        xo, ro, uo = oracle.solve(method, A, b, x0=x0, pc="jacobi", **kw)
        assert ur == uo, (A.name, ur, uo)
        assert np.array_equal(xr, xo), A.name
        if method not in ("gmres", "fgmres"):
            assert np.array_equal(rr[: len(ro)], ro), A.name


@pytest.mark.skipif(oracle.ref_ilu0() is None, reason="compiled reference not present")
def test_ilu0_restatement_bitwise_vs_compiled_reference():
    for A in (st.convdiff3d_27pt(6, pe=5.0), st.varcoef3d_7pt(7, 9), st.poisson2d_5pt(13)):
        assert np.array_equal(oracle.ilu0_values(A), oracle.ref_ilu0_values(A))


def test_ilu0_is_exact_on_pattern():
    """ILU(0): (L U)_ij = a_ij for every (i, j) in A's pattern."""
    A = st.varcoef3d_7pt(6, 2)
    F = oracle.ilu0(A)
    import scipy.sparse as sp
    n = A.n
    L = sp.csr_matrix((F.lv, F.lci, F.lrp), shape=(n, n)) + sp.eye(n)
    U = sp.diags(1.0 / F.dinv) @ (sp.csr_matrix((F.uv, F.uci, F.urp), shape=(n, n)) + sp.eye(n))
    LU = (L @ U).tocsr()
    Asp = A.to_scipy()
    rows = np.repeat(np.arange(n), np.diff(A.rowptr))
    diff = np.asarray(LU[rows, A.colidx]).ravel() - A.val
    assert np.max(np.abs(diff)) < 1e-12 * np.max(np.abs(A.val))


def test_lusolve_matches_scipy():
    A = st.convdiff3d_27pt(6)
    F = oracle.ilu0(A)
    import scipy.sparse as sp
    import scipy.sparse.linalg as sla
    n = A.n
    L = (sp.csr_matrix((F.lv, F.lci, F.lrp), shape=(n, n)) + sp.eye(n)).tocsr()
    Up = (sp.csr_matrix((F.uv, F.uci, F.urp), shape=(n, n)) + sp.eye(n)).tocsr()
    x = st.rhs_uniform(n, 4)
    y = oracle.lusolve(F, x)
    ref = sla.spsolve_triangular(Up, F.dinv * sla.spsolve_triangular(L, x, lower=True), lower=False)
    assert np.allclose(y, ref, rtol=1e-12, atol=1e-12)
    yt = oracle.lusolve_t(F, x)
    reft = sla.spsolve_triangular(L.T.tocsr(), F.dinv * sla.spsolve_triangular(Up.T.tocsr(), x, lower=True),
                                  lower=False)
    assert np.allclose(yt, reft, rtol=1e-12, atol=1e-12)


def test_parilu_converges_to_ilu0():
    """Synchronous ParILU sweeps are Jacobi iterations for the ILU(0) fixed
    point; with enough sweeps they reach the exact factors."""
    A = st.poisson2d_5pt(12)
    exact = oracle.ilu0_values(A)
    few = oracle.parilu_values(A, sweeps=3)
    many = oracle.parilu_values(A, sweeps=60)
    assert np.max(np.abs(many - exact)) < 1e-12
    assert np.max(np.abs(few - exact)) > np.max(np.abs(many - exact))


def test_parilut_quality_and_fill():
    A = st.convdiff3d_27pt(6, pe=10.0)
    F = oracle.parilut(A, fill=2.0, sweeps=5)
    nnz_lu = len(F.lv) + len(F.uv) + A.n
    assert nnz_lu <= 2.0 * A.nnz + 2 * A.n  # budget rate*nnz0 per factor; diagonals are always kept
    # as a preconditioner it must beat no preconditioning and roughly match ILU(0)
    b = st.rhs_uniform(A.n, 0, 0.0, 1.0)
    _, _, it_lut = oracle.solve("fgmres", A, b, tol=1e-10, maxiter=300, restart=30, pc="lu", factors=F)
    _, _, it_ilu = oracle.solve("fgmres", A, b, tol=1e-10, maxiter=300, restart=30, pc="lu", factors=oracle.ilu0(A))
    _, _, it_none = oracle.solve("fgmres", A, b, tol=1e-10, maxiter=300, restart=30, pc="none")
    assert it_lut <= it_ilu + 2
    assert it_lut < it_none


def test_levels_lower():
    A = st.poisson3d_7pt(8)
    rows = np.repeat(np.arange(A.n), np.diff(A.rowptr))
    m = A.colidx < rows
    lrp = np.zeros(A.n + 1, np.int32)
    np.cumsum(np.bincount(rows[m], minlength=A.n), out=lrp[1:])
    lev, nlev = oracle.levels_lower(A.n, lrp, np.ascontiguousarray(A.colidx[m]))
    assert nlev == 3 * 8 - 2


@pytest.mark.skipif(oracle.ref_ic0_values(st.poisson2d_5pt(3)) is None, reason="compiled reference not present")
def test_ic0_restatement_bitwise_vs_compiled_reference():
    """IC(0) (hip/Precond/ic0.cpp, ic0_csr_A with the Precond_ic0 defaults)."""
    for A in (st.poisson2d_5pt(15), st.varcoef3d_7pt(7, 2), st.poisson3d_7pt(8), st.varcoef3d_7pt(5, 7)):
        assert np.array_equal(oracle.ic0_values(A), oracle.ref_ic0_values(A)), A.name


def test_threaded_timing_variant_tracks_the_oracle():
    """The CPU reference arm of the benchmark times a threaded variant of the
    restated BiCGSTAB + ILU(0) (SpMV and vector operations on host threads,
    triangular solves sequential, dot products in a fixed blocked order).
    It must solve the same system as the oracle: residual below the
    tolerance, iteration count within two of the oracle's, the same solution
    to the accuracy the tolerance allows, and identical results for any
    thread count."""
    A = st.varcoef3d_7pt(20, 3)
    b = st.rhs_uniform(A.n, 1)
    F = oracle.ilu0(A)
    xo, ho, uo = oracle.solve("bicgstab", A, b, tol=1e-10, maxiter=500, pc="lu", factors=F)
    runs = [oracle.bicgstab_threads(A, b, F, tol=1e-10, maxiter=500, threads=t) for t in (1, 3, 8)]
    x, it, rsm = runs[0]
    for xt, itt, rt in runs[1:]:
        assert np.array_equal(xt, x) and itt == it and rt == rsm
    rel = np.linalg.norm(b - A.to_scipy() @ x) / np.linalg.norm(b)
    assert rsm < 1e-10 and rel < 1e-9
    assert abs(it - (uo + 1)) <= 2, (it, uo + 1)
    assert np.linalg.norm(x - xo) / np.linalg.norm(xo) < 1e-7
