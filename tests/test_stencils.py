"""Synthetic stencil generators: sizes and nnz from the closed forms, sorted
columns, diagonal present, symmetry where expected."""
import numpy as np

from xsolver_b200 import stencils as st


def _check_csr(A):
    assert A.rowptr[0] == 0 and A.rowptr[-1] == len(A.colidx) == len(A.val)
    rows = np.repeat(np.arange(A.n), np.diff(A.rowptr))
    assert np.all(np.diff(A.colidx)[np.diff(rows) == 0] > 0)  # sorted, unique per row
    assert np.sum(A.colidx == rows) == A.n  # diagonal present


def test_poisson2d():
    A = st.poisson2d_5pt(128)
    assert A.n == 16384 and A.nnz == 5 * 16384 - 4 * 128 == 81408
    _check_csr(A)
    S = A.to_scipy()
    assert abs(S - S.T).max() == 0


def test_poisson3d():
    A = st.poisson3d_7pt(20)
    assert A.nnz == 7 * 20 ** 3 - 6 * 20 ** 2
    _check_csr(A)


def test_convdiff27_counts_and_nonsymmetry():
    A = st.convdiff3d_27pt(12)
    assert A.nnz == (3 * 12 - 2) ** 3
    _check_csr(A)
    S = A.to_scipy()
    assert abs(S - S.T).max() > 0
    # weakly diagonally dominant by construction
    d = S.diagonal()
    off = np.asarray(abs(S).sum(axis=1)).ravel() - np.abs(d)
    assert np.all(d >= off - 1e-12)


def test_varcoef_symmetric_positive():
    A = st.varcoef3d_7pt(10, seed=1)
    _check_csr(A)
    S = A.to_scipy()
    assert abs(S - S.T).max() < 1e-14
    assert np.all(S.diagonal() > 0)


def test_rhs_seeded():
    a = st.rhs_uniform(100, 3)
    b = st.rhs_uniform(100, 3)
    assert np.array_equal(a, b) and a.min() >= -1 and a.max() <= 1
