"""Saad ILUT and ICT factors: the oracle restatement and the library's host
factorization (xs_host_ilut / xs_host_ict, no device) bitwise against the
reference's own ilutp_final and ict_csr_A_l, recorded in
tests/golden/threshold_factors.npz and, where the compiled reference is
present, run directly on larger and nonsymmetric matrices."""
import os

import numpy as np
import pytest

import oracle
from xsolver_b200 import stencils as st
from xsolver_b200.api import host_ict, host_ilut
from xsolver_b200._lib import XsError

GOLD = os.path.join(os.path.dirname(__file__), "golden", "threshold_factors.npz")
KEYS = ("lrp", "lci", "lv", "dinv", "urp", "uci", "uv")


def _get(F, k):
    return F[k] if isinstance(F, dict) else getattr(F, k)


def _same(F, G):
    for k in KEYS:
        a, b = _get(F, k), _get(G, k)
        if a.shape != b.shape or not np.array_equal(a, b):
            return k
    return None


def _golden_cases():
    z = np.load(GOLD)
    names = sorted({k.split("/")[0] for k in z.files})
    for nm in names:
        A = st.CSRMatrix(len(z[f"{nm}/rowptr"]) - 1, z[f"{nm}/rowptr"], z[f"{nm}/colidx"], z[f"{nm}/val"], nm)
        tags = sorted({k.split("/")[1] for k in z.files if k.startswith(nm + "/") and k.count("/") == 2})
        for tag in tags:
            fill, tol = z[f"{nm}/{tag}/params"]
            yield nm, A, tag, int(fill), float(tol), {k: z[f"{nm}/{tag}/{k}"] for k in KEYS}


def test_golden_covers_both_methods_and_the_pivot_substitute():
    cases = list(_golden_cases())
    assert {c[2][:3] for c in cases} == {"ilu", "ict"}
    assert any(c[0] == "p2d_zero_pivot" for c in cases)
    assert len(cases) == 16


@pytest.mark.parametrize("who", ["oracle", "library"])
def test_threshold_factors_bitwise_vs_golden(who):
    for nm, A, tag, fill, tol, G in _golden_cases():
        if tag.startswith("ilut"):
            F = oracle.ilut_saad(A, fill, tol) if who == "oracle" else host_ilut(A, fill, tol)
        else:
            F = oracle.ict(A, fill, tol) if who == "oracle" else host_ict(A, fill, tol)
        assert _same(F, G) is None, (nm, tag, _same(F, G))


def test_zero_pivot_takes_the_substitute():
    """Row 0 with a zero diagonal: both factorizations replace the pivot by
    (1e-4/droptol + 1) * droptol * ||a_0|| (ILUT) or take 1/sqrt of it (ICT)."""
    A = st.poisson2d_5pt(12)
    v = A.val.copy()
    v[A.rowptr[0]] = 0.0
    A = st.CSRMatrix(A.n, A.rowptr, A.colidx, v)
    tol = 1e-4
    tn = np.sqrt(np.sum(v[A.rowptr[0]:A.rowptr[1]] ** 2)) * tol
    d = 1e-4 / tol * tn + tn
    assert host_ilut(A, 5, tol)["dinv"][0] == 1 / d
    d2 = 1e-4 * (1 / tol) * tn + tn
    assert host_ict(A, 5, tol)["dinv"][0] == (1 / np.sqrt(d2)) ** 2


def test_entry_limits_hold():
    A = st.poisson3d_7pt(9)
    for lfil in (1, 3, 8):
        F = host_ilut(A, lfil, 1e-6)
        assert np.diff(F["lrp"]).max() <= lfil and np.diff(F["urp"]).max() <= lfil
    for m in (1, 4):
        F = host_ict(A, m, 1e-6)
        assert np.diff(F["lrp"]).max() <= m
        # U' is L' transposed
        L = _csr(A.n, F["lrp"], F["lci"], F["lv"])
        U = _csr(A.n, F["urp"], F["uci"], F["uv"])
        assert (L.T != U).nnz == 0


def _csr(n, rp, ci, v):
    import scipy.sparse as sp

    return sp.csr_matrix((v, ci, rp), shape=(n, n))


def test_invalid_arguments_and_missing_diagonal():
    A = st.poisson2d_5pt(6)
    with pytest.raises(XsError):
        host_ilut(A, 0, 1e-4)  # lfil >= 1
    with pytest.raises(XsError):
        host_ict(A, 3, 0.0)  # ICT divides by droptol
    rows = np.repeat(np.arange(A.n), np.diff(A.rowptr))
    keep = (A.colidx != rows) | (rows != 3)  # row 3 without its diagonal
    nrp = np.concatenate([[0], np.cumsum(np.bincount(rows[keep], minlength=A.n))]).astype(np.int32)
    B = st.CSRMatrix(A.n, nrp, A.colidx[keep], A.val[keep])
    with pytest.raises(XsError) as e:
        host_ict(B, 3, 1e-4)
    assert e.value.code == 4  # XS_ERR_NO_DIAG
    with pytest.raises(ValueError):
        oracle.ict(B, 3, 1e-4)


def test_empty_matrix():
    A = st.CSRMatrix(0, np.zeros(1, np.int32), np.zeros(0, np.int32), np.zeros(0))
    for F in (host_ilut(A, 2, 1e-3), host_ict(A, 2, 1e-3)):
        assert F["lrp"].tolist() == [0] and F["lci"].size == 0 and F["uci"].size == 0


@pytest.mark.skipif(oracle.ref_ict(st.poisson2d_5pt(3), 1, 1e-2) is None, reason="compiled reference not present")
@pytest.mark.parametrize("case", ["p3d_16", "cd27_12", "vc3d_14", "p2d_64"])
def test_threshold_factors_bitwise_vs_compiled_reference(case):
    """Larger and nonsymmetric matrices (ILUT), symmetric ones (ICT), several
    parameter sets, straight against the compiled reference."""
    A = {"p3d_16": lambda: st.poisson3d_7pt(16), "cd27_12": lambda: st.convdiff3d_27pt(12),
         "vc3d_14": lambda: st.varcoef3d_7pt(14, 1), "p2d_64": lambda: st.poisson2d_5pt(64)}[case]()
    for lfil, tol in ((1, 0.0), (4, 1e-3), (10, 1e-5), (30, 1e-8)):
        R = oracle.ref_ilut_saad(A, lfil, tol)
        assert _same(oracle.ilut_saad(A, lfil, tol), R) is None, (case, lfil, tol)
        assert _same(host_ilut(A, lfil, tol), R) is None, (case, lfil, tol)
    if case == "cd27_12":
        return  # ICT is for symmetric matrices
    for m, tol in ((2, 1e-2), (8, 1e-5), (40, 1e-8)):
        R = oracle.ref_ict(A, m, tol)
        assert _same(oracle.ict(A, m, tol), R) is None, (case, m, tol)
        assert _same(host_ict(A, m, tol), R) is None, (case, m, tol)
