"""GPU kernel parity: SpMV, ILU(0)/ParILU factorisation and sync-free LU
solves against the oracle (and the reference's own ILU(0) output).

FP64 SpMV (CSR and ELL), ILU(0), ParILU and the FP64 LU solve run in the
same operation order as the CPU code, so they are compared bit for bit."""
import os

import numpy as np
import pytest

import oracle
from xsolver_b200 import stencils as st

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")


def _dev(a, cuda):
    import torch

    return torch.from_numpy(np.ascontiguousarray(a)).to(cuda)


def _matrices():
    yield st.poisson2d_5pt(37)
    yield st.poisson3d_7pt(17)
    yield st.convdiff3d_27pt(11)
    yield st.varcoef3d_7pt(13, 5)


def _long_row_matrix():
    """A matrix with one dense row longer than the SpMV staging capacity,
    an empty row, and ragged row lengths."""
    rng = np.random.default_rng(0)
    n = 9000
    rows = []
    for i in range(n):
        if i == 7:
            cols = np.arange(n)  # dense row
        elif i == 11:
            cols = np.array([], dtype=np.int64)  # empty row
        else:
            k = int(rng.integers(1, 12))
            cols = np.unique(np.concatenate([[i], rng.integers(0, n, k)]))
        rows.append(np.sort(cols))
    rp = np.zeros(n + 1, np.int32)
    rp[1:] = np.cumsum([len(c) for c in rows])
    ci = np.concatenate(rows).astype(np.int32)
    v = rng.standard_normal(len(ci))
    return st.CSRMatrix(n, rp, ci, v, "ragged")


@pytest.fixture(params=[0, 16, 32], ids=["diag", "idx16", "idx32"])
def ell_columns(request):
    """ELL column storage for copies built inside the test: diagonal slots
    (where the pattern allows), 16-bit row offsets, 32-bit columns."""
    from xsolver_b200 import _lib

    L = _lib.lib()
    assert L.xs_set_ell_index_bits(request.param) == 0
    yield request.param
    L.xs_set_ell_index_bits(0)


@pytest.mark.parametrize("fmt", ["csr", "ell"])
def test_spmv_fp64_bitwise(cuda, fmt, ell_columns):
    import torch
    from xsolver_b200.api import Plan

    if fmt == "csr" and ell_columns != 0:
        pytest.skip("column storage only affects the ELL copy")
    for A in list(_matrices()) + ([_long_row_matrix()] if fmt == "csr" else []):
        P = Plan(A)
        if fmt == "ell":
            w = P.build_ell()
            # diagonal slots: one slot per diagonal; otherwise the longest row
            offs = np.unique(A.colidx - np.repeat(np.arange(A.n), np.diff(A.rowptr)))
            assert w == (len(offs) if ell_columns == 0 else int(np.max(np.diff(A.rowptr))))
        x = st.rhs_uniform(A.n, 1)
        y = torch.zeros(A.n, dtype=torch.float64, device=cuda)
        P.spmv(_dev(x, cuda), y, fmt=fmt)
        P.sync()
        ref = oracle.spmv(A, x)
        got = y.cpu().numpy()
        if A.name == "ragged":
            # a row longer than the staging capacity is reduced by the whole
            # block (parallel order): equal to rounding; every other row bitwise
            long_row = 7
            assert abs(got[long_row] - ref[long_row]) <= 1e-12 * np.sum(np.abs(A.val[A.rowptr[7]:A.rowptr[8]]))
            got[long_row] = ref[long_row]
            assert got[11] == 0.0  # empty row
        assert np.array_equal(got, ref), A.name


def test_spmv_fp32(cuda):
    import torch
    from xsolver_b200.api import Plan

    A = st.convdiff3d_27pt(13)
    P = Plan(A)
    x = st.rhs_uniform(A.n, 2)
    y = torch.zeros(A.n, dtype=torch.float32, device=cuda)
    P.spmv(_dev(x.astype(np.float32), cuda), y, precision="fp32")
    P.sync()
    ref = oracle.spmv(A, x)
    err = np.abs(y.cpu().numpy() - ref).max() / np.abs(ref).max()
    assert err < 1e-5


def test_spmv_transposed(cuda):
    import torch
    from xsolver_b200.api import Plan

    A = st.convdiff3d_27pt(9)
    P = Plan(A)
    x = st.rhs_uniform(A.n, 3)
    y = torch.zeros(A.n, dtype=torch.float64, device=cuda)
    P.spmv_t(_dev(x, cuda), y)
    P.sync()
    ref = oracle.spmv_t(A, x)
    assert np.allclose(y.cpu().numpy(), ref, rtol=1e-13, atol=1e-13)


def test_ilu0_bitwise_vs_reference_golden(cuda):
    """Exact GPU ILU(0) equals the reference's own ilu0_simple output."""
    from xsolver_b200.api import Plan

    z = np.load(os.path.join(GOLD, "ilu0.npz"))
    for nm in sorted({k.split("/")[0] for k in z.files}):
        A = st.CSRMatrix(len(z[f"{nm}/rowptr"]) - 1, z[f"{nm}/rowptr"], z[f"{nm}/colidx"], z[f"{nm}/val"], nm)
        P = Plan(A).factor("ilu0")
        assert np.array_equal(P.lu_values(), z[f"{nm}/luv"]), nm


def test_ilu0_bitwise_vs_oracle_large(cuda):
    from xsolver_b200.api import Plan

    for A in (st.poisson3d_7pt(48), st.convdiff3d_27pt(24)):
        P = Plan(A).factor("ilu0")
        assert np.array_equal(P.lu_values(), oracle.ilu0_values(A)), A.name
        F = oracle.ilu0(A)
        G = P.factors()
        for k in ("lrp", "lci", "lv", "dinv", "urp", "uci", "uv"):
            assert np.array_equal(G[k], getattr(F, k)), (A.name, k)


def test_ilu0_box_schedule_bitwise(cuda):
    """The box-scheduled ILU(0) (systems whose L solve has boxes: at least
    65536 rows on a grid) and the level-ordered lane groups give the oracle's
    factors bit for bit: 7- and 27-point patterns, variable coefficients."""
    from xsolver_b200 import _lib
    from xsolver_b200.api import Plan

    L = _lib.lib()
    for A in (st.poisson3d_7pt(64), st.convdiff3d_27pt(48), st.varcoef3d_7pt(56, 2)):
        ref = oracle.ilu0_values(A)
        for on in (1, 0):
            assert L.xs_set_ilu_tiles(on) == 0
            try:
                P = Plan(A).factor("ilu0")
                assert np.array_equal(P.lu_values(), ref), (A.name, on)
            finally:
                L.xs_set_ilu_tiles(0)


def _wide_rows_matrix():
    """2D 5-point Poisson 40x40 plus 5 rows coupled to 40-60 random columns
    (weakly, so the pivots stay away from zero): rows wider than 32 entries,
    the row-width class the lane-group ILU(0) kernel leaves to the
    thread-per-row kernel, next to ordinary rows."""
    A = st.poisson2d_5pt(40)
    n = A.n
    rng = np.random.default_rng(3)
    S = A.to_scipy().tolil()
    for i in (100, 555, 800, 1201, 1599):
        for j in rng.choice(n, int(rng.integers(40, 61)), replace=False):
            if j != i:
                S[i, j] = -0.01 * rng.random()
                S[j, i] = -0.01 * rng.random()
    S = S.tocsr()
    S.sort_indices()
    return st.CSRMatrix(n, S.indptr.astype(np.int32), S.indices.astype(np.int32), S.data.copy(), "wide-rows")


def test_ilu0_bitwise_vs_oracle_wide_and_narrow_rows(cuda):
    """Both ILU(0) row kernels against the oracle: lane groups of 4, 8 and 32
    (5-, 7- and 27-point rows) and the thread-per-row kernel (rows over 32
    entries)."""
    from xsolver_b200.api import Plan

    for A in (st.poisson2d_5pt(64), st.poisson3d_7pt(20), st.convdiff3d_27pt(14), _wide_rows_matrix()):
        P = Plan(A).factor("ilu0")
        assert np.array_equal(P.lu_values(), oracle.ilu0_values(A)), A.name


def test_ic0_bitwise_vs_oracle(cuda):
    """GPU IC(0) (the reference's ic0_csr_A order, bitwise vs the restatement
    that is pinned to the compiled reference) and its conversion into the
    LU solve's factors (HostMatrixCSR::seqic0)."""
    from xsolver_b200.api import Plan

    for A in (st.poisson2d_5pt(30), st.varcoef3d_7pt(11, 4), st.poisson3d_7pt(16)):
        P = Plan(A).factor("ic0")
        assert np.array_equal(P.lu_values()[_lower_mask(A)], oracle.ic0_values(A)[_lower_mask(A)]), A.name
        G = P.factors()
        F = oracle.ic0(A)
        for k in ("lrp", "lci", "lv", "dinv", "urp", "uci", "uv"):
            assert np.array_equal(G[k], getattr(F, k)), (A.name, k)


def _lower_mask(A):
    return A.colidx <= np.repeat(np.arange(A.n), np.diff(A.rowptr))


def test_ic0_refuses_unsymmetric_pattern(cuda):
    from xsolver_b200.api import Plan, XsError

    A = st.convdiff3d_27pt(5)
    rows = np.repeat(np.arange(A.n), np.diff(A.rowptr))
    keep = ~((rows == 3) & (A.colidx == 4))  # drop one upper entry, keep its lower twin (4, 3)
    rp = np.zeros(A.n + 1, np.int32)
    np.cumsum(np.bincount(rows[keep], minlength=A.n), out=rp[1:])
    B = st.CSRMatrix(A.n, rp, A.colidx[keep], A.val[keep], "unsym")
    keep2 = ~((rows == 4) & (A.colidx == 3))  # drop one lower entry, keep its upper twin (3, 4)
    rp2 = np.zeros(A.n + 1, np.int32)
    np.cumsum(np.bincount(rows[keep2], minlength=A.n), out=rp2[1:])
    C2 = st.CSRMatrix(A.n, rp2, A.colidx[keep2], A.val[keep2], "unsym2")
    # U is L's transpose (seqic0): either missing twin makes A's upper pattern differ from it
    for M in (B, C2):
        with pytest.raises(XsError) as e:
            Plan(M).factor("ic0")
        assert e.value.code == 10, M.name


def test_parilu_bitwise_vs_oracle(cuda):
    from xsolver_b200.api import Plan

    for A in (st.poisson3d_7pt(14), st.convdiff3d_27pt(9)):
        for sweeps in (1, 5, 20):
            P = Plan(A).factor("parilu", sweeps=sweeps)
            assert np.array_equal(P.lu_values(), oracle.parilu_values(A, sweeps)), (A.name, sweeps)


def test_lusolve_fp64_bitwise(cuda):
    import torch
    from xsolver_b200.api import Plan

    for A in (st.poisson3d_7pt(33), st.convdiff3d_27pt(17), st.varcoef3d_7pt(15, 2)):
        P = Plan(A).factor("ilu0")
        F = oracle.ilu0(A)
        x = st.rhs_uniform(A.n, 7)
        z = torch.zeros(A.n, dtype=torch.float64, device=cuda)
        for rep in range(3):  # repeated solves reuse the re-armed buffers
            P.lusolve(_dev(x, cuda), z)
            P.sync()
            assert np.array_equal(z.cpu().numpy(), oracle.lusolve(F, x)), (A.name, rep)


@pytest.mark.parametrize("prec,tol", [("fp32", 2e-5), ("bf16", 5e-2), ("fp16", 5e-3)])
def test_lusolve_reduced_precision(cuda, prec, tol):
    import torch
    from xsolver_b200.api import Plan

    A = st.poisson3d_7pt(31)
    P = Plan(A).factor("ilu0").set_factor_precision(prec)
    F = oracle.ilu0(A)
    x = st.rhs_uniform(A.n, 8)
    z = torch.zeros(A.n, dtype=torch.float32, device=cuda)
    P.lusolve(_dev(x.astype(np.float32), cuda), z)
    P.sync()
    ref = oracle.lusolve(F, x)
    err = np.linalg.norm(z.cpu().numpy() - ref) / np.linalg.norm(ref)
    assert err < tol, err


def test_lusolve_transposed(cuda):
    import torch
    from xsolver_b200.api import Plan

    A = st.convdiff3d_27pt(10)
    P = Plan(A).factor("ilu0")
    F = oracle.ilu0(A)
    x = st.rhs_uniform(A.n, 9)
    z = torch.zeros(A.n, dtype=torch.float64, device=cuda)
    P.lusolve_t(_dev(x, cuda), z)
    P.sync()
    ref = oracle.lusolve_t(F, x)
    assert np.allclose(z.cpu().numpy(), ref, rtol=1e-12, atol=1e-12)


def test_levels_match_oracle(cuda):
    from xsolver_b200.api import Plan

    A = st.poisson3d_7pt(20)
    P = Plan(A).factor("ilu0")
    assert P.levels() == (3 * 20 - 2, 3 * 20 - 2)


def test_parilut_bitwise_vs_oracle(cuda):
    """GPU ParILUT (synchronous sweeps, radix-select thresholds) equals the
    CPU restatement entry for entry."""
    from xsolver_b200.api import Plan

    for A, fill, sweeps, droptol in ((st.convdiff3d_27pt(9), 2.0, 5, 0.0), (st.poisson3d_7pt(12), 3.0, 4, 0.0),
                                     (st.convdiff3d_27pt(8, pe=10.0), 2.0, 3, 1e-4)):
        P = Plan(A).factor("parilut", sweeps=sweeps, fill=fill, droptol=droptol)
        G = P.factors()
        F = oracle.parilut(A, fill=fill, sweeps=sweeps, droptol=droptol)
        for k in ("lrp", "lci", "lv", "dinv", "urp", "uci", "uv"):
            assert np.array_equal(G[k], getattr(F, k)), (A.name, k)


def _parilut_fallback_matrix():
    """2D 5-point Poisson 280x280 (n = 78,400) with (a) five long-range
    couplings (i, i + 70000 mod n) and their transposes, so some rows'
    candidate columns span more than the 65,536-column bitmap window, and (b)
    one row and column coupled to 600 columns within +-30,000, so one row has
    over 512 candidates and over 256 pattern entries in the sweeps: the
    sort-based candidate path and the per-entry value and sweep paths next
    to the bitmap and row-wise paths."""
    A = st.poisson2d_5pt(280)
    n = A.n
    rng = np.random.default_rng(7)
    S = A.to_scipy().tolil()
    for i in (10, 20, 30, 77000, 78390):
        j = (i + 70000) % n
        S[i, j] = -0.05
        S[j, i] = -0.05
    r = 39000
    for j in r - 30000 + rng.choice(60000, 600, replace=False):
        if j != r:
            S[r, j] = -0.001
            S[j, r] = -0.001
    S = S.tocsr()
    S.sort_indices()
    return st.CSRMatrix(n, S.indptr.astype(np.int32), S.indices.astype(np.int32), S.data.copy(), "parilut-fallbacks")


def test_parilut_fallback_paths_bitwise(cuda):
    from xsolver_b200.api import Plan

    A = _parilut_fallback_matrix()
    for fill, sweeps, droptol in ((2.0, 3, 0.0), (1.5, 2, 1e-4)):
        G = Plan(A).factor("parilut", sweeps=sweeps, fill=fill, droptol=droptol).factors()
        F = oracle.parilut(A, fill=fill, sweeps=sweeps, droptol=droptol)
        for k in ("lrp", "lci", "lv", "dinv", "urp", "uci", "uv"):
            assert np.array_equal(G[k], getattr(F, k)), (fill, k)


def test_block_and_syncfree_lusolve_bitwise(cuda):
    """The single-CTA solve (small systems; staged level batches and
    per-level loads) and the sync-free multi-CTA solve give the same bits,
    FP64 and FP32/BF16 factors."""
    import torch
    from xsolver_b200 import _lib
    from xsolver_b200.api import Plan

    L = _lib.lib()
    for A in (st.poisson2d_5pt(128), st.convdiff3d_27pt(14), st.convdiff3d_27pt(24)):
        x = st.rhs_uniform(A.n, 11)
        outs = []
        for rows, staged in ((1 << 30, 1), (1 << 30, 0), (0, 1)):
            assert L.xs_set_trsv_block_rows(rows) == 0
            assert L.xs_set_trsv_block_staging(staged) == 0
            try:
                P = Plan(A).factor("ilu0")
                # device inputs stay referenced until the plan's stream is synchronised
                # (the solves run on the plan's own stream, not torch's)
                dx, dx32 = _dev(x, cuda), _dev(x.astype(np.float32), cuda)
                z = torch.zeros(A.n, dtype=torch.float64, device=cuda)
                z32 = torch.zeros(A.n, dtype=torch.float32, device=cuda)
                P.lusolve(dx, z)
                P.sync()
                P.set_factor_precision("bf16")
                P.lusolve(dx32, z32)
                P.sync()
                outs.append((z.cpu().numpy(), z32.cpu().numpy()))
            finally:
                L.xs_set_trsv_block_rows(1 << 30)
                L.xs_set_trsv_block_staging(1)
        for o in outs[1:]:
            assert np.array_equal(outs[0][0], o[0]), A.name
            assert np.array_equal(outs[0][1], o[1]), A.name
        assert np.array_equal(outs[0][0], oracle.lusolve(oracle.ilu0(A), x)), A.name


def test_syncfree_wait_times_out_and_recovers(cuda):
    """A dependency nothing publishes: the bounded wait gives up (about 1 s),
    the error is reported, and the plan works again after the dependency is
    restored.  (Sync-free solve forced: the single-CTA solve has no waits.)"""
    import torch
    from xsolver_b200 import _lib
    from xsolver_b200.api import Plan, XsError

    _lib.lib().xs_set_trsv_block_rows(0)
    try:
        _timeout_case(cuda, torch, Plan, XsError)
    finally:
        _lib.lib().xs_set_trsv_block_rows(1 << 30)


def _timeout_case(cuda, torch, Plan, XsError):
    A = st.poisson3d_7pt(16)
    P = Plan(A).factor("ilu0")
    F = oracle.ilu0(A)
    x = st.rhs_uniform(A.n, 1)
    z = torch.zeros(A.n, dtype=torch.float64, device=cuda)
    P.debug_break_dependency(A.n - 1, True)
    P.lusolve(_dev(x, cuda), z)
    with pytest.raises(XsError) as e:
        P.sync()
    assert e.value.code == 5  # XS_ERR_TRSV_TIMEOUT
    P.debug_break_dependency(A.n - 1, False)
    P.lusolve(_dev(x, cuda), z)
    P.sync()
    assert np.array_equal(z.cpu().numpy(), oracle.lusolve(F, x))


@pytest.mark.parametrize("k", [1, 2, 3, 5])
def test_jacobi_sweep_lusolve_matches_emulation(cuda, k, ell_columns):
    """The approximate solve of the reference GPU path (k Jacobi sweeps per
    triangle, DeviceMatrixCSR.cpp:281-304), ELL layout on the device, against
    a numpy emulation of the same sweeps on the oracle's factors."""
    import scipy.sparse as sp
    import torch
    from xsolver_b200.api import Plan

    for A in (st.poisson3d_7pt(20), st.convdiff3d_27pt(12)):
        n = A.n
        P = Plan(A).factor("ilu0").set_trsv(k)
        F = oracle.ilu0(A)
        L = sp.csr_matrix((F.lv, F.lci, F.lrp), shape=(n, n))
        U = sp.csr_matrix((F.uv, F.uci, F.urp), shape=(n, n))
        x = st.rhs_uniform(n, k)
        y = x.copy()
        for _ in range(k - 1):
            y = x - L @ y
        d = F.dinv * y
        w = d.copy()
        for _ in range(k - 1):
            w = d - U @ w
        from xsolver_b200 import _lib

        got = []
        for fuse in (1, 0):  # sweeps 2 and 3 in one pass, or in two
            _lib.lib().xs_set_sweep_fusion(fuse)
            z = torch.zeros(n, dtype=torch.float64, device=cuda)
            P.lusolve(_dev(x, cuda), z)
            P.sync()
            got.append(z.cpu().numpy())
        _lib.lib().xs_set_sweep_fusion(0)
        assert np.array_equal(got[0], got[1]), (A.name, k)
        assert np.allclose(got[0], w, rtol=1e-12, atol=1e-13), (A.name, k)
