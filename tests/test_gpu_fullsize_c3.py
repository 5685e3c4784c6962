"""Parity at the full size of the 27-point convection-diffusion configuration.

27-point convection-diffusion on a 160^3 grid (n = 4,096,000, nnz =
109,215,352), velocity (1, 0.5, 0.25) * Pe at Pe = 50 (h^2-scaled upwind),
b ~ U(0, 1) from seed 0, x0 = 0, ParILUT (fill factor 2, 5 sweeps, drop
tolerance 1e-4):

  * the GPU ParILUT factors equal the oracle's (hip/Precond/parilut.cpp:
    621-1206, restated with synchronous sweeps) bit for bit;
  * FP64 GMRES(30) and GCR(30) with those factors and the exact triangular
    solves, rtol 1e-10 (intel/mpisolver-C-v1.cpp:685-1087 restated; the
    handle API's GMRES is right-preconditioned, the oracle's FGMRES with a
    fixed preconditioner is the same method, and its GCR is the reference's
    hip/Solver/xsolver_igcr.cpp:29-108): the per-iteration residual history
    within the strict 1e-10 relative bound at every iteration, the
    iteration count within +-1 and the solution within 1e-10 relative of the
    oracle run on the same factors;
  * the mixed-precision form (FP64 outer refinement around an FP32
    GMRES(30), BF16 and FP16 factors, exact and Jacobi-sweep triangular
    solves): true relative residual below 1e-10 and the error against the
    oracle's FP64 solve converged to 1e-14 within cond(A) times the
    residual.  cond_2(A) of this operator grows about linearly with the grid
    (dense SVD: 9.8, 14.1, 23.2, 32.6 at 6^3, 8^3, 12^3, 16^3), about 330 at
    160^3; the bound uses 1e3.

The oracle's ParILUT runs on all host threads (its per-row loops write
disjoint outputs, so the factors do not depend on the thread count); at this
size it takes a few minutes of the test time.
"""
import numpy as np
import pytest

import oracle
from parity import strict_report
from xsolver_b200 import stencils as st

pytestmark = pytest.mark.gpu

FILL, SWEEPS, DROPTOL = 2.0, 5, 1e-4
COND_BOUND = 1e3


@pytest.fixture(scope="module")
def c3():
    A = st.convdiff3d_27pt(160)
    assert A.n == 4096000 and A.nnz == 109215352
    b = st.rhs_uniform(A.n, 0, 0.0, 1.0)
    F = oracle.parilut(A, fill=FILL, sweeps=SWEEPS, droptol=DROPTOL)
    return A, b, F


def _solver(A, ksp, trsv=0):
    from xsolver_b200.api import Solver

    S = Solver(A).ksp_settype(ksp).ksp_setoption(1e-10, 3000, 30).pc_settype("parilut")
    S.pc_setparilut(FILL, SWEEPS, DROPTOL).pc_set_trsv(trsv)
    return S


def test_c3_parilut_factors_bitwise(cuda, c3):
    from xsolver_b200.api import Plan

    A, b, F = c3
    G = Plan(A).factor("parilut", sweeps=SWEEPS, fill=FILL, droptol=DROPTOL).factors()
    for k in ("lrp", "lci", "lv", "dinv", "urp", "uci", "uv"):
        assert np.array_equal(G[k], getattr(F, k)), k


@pytest.mark.parametrize("ksp,oracle_method", [("gmres", "fgmres"), ("gcr", "hip_igcr")])
def test_c3_fp64_vs_reference(cuda, c3, ksp, oracle_method):
    A, b, F = c3
    S = _solver(A, ksp)
    x = S.solve(b)
    hist = S.resvec()
    xo, ho, uo = oracle.solve(oracle_method, A, b, tol=1e-10, maxiter=3000, restart=30, pc="lu", factors=F, quirk=0)
    if oracle_method == "hip_igcr":  # absolute residuals, [0] = ||r0||, count = last index
        frac, worst = strict_report(hist, ho, scale=ho[0])
        assert abs(S.usediter - uo) <= 1, (S.usediter, uo)
    else:
        frac, worst = strict_report(hist[1:] / hist[0], ho)
        assert abs(S.usediter - (uo + 1)) <= 1, (S.usediter, uo + 1)
    print(f"C3 {ksp}: {S.usediter} iterations, history within 1e-10 at {frac:.0%} of iterations, "
          f"worst |diff|/1e-10 = {worst:.3g}")
    assert frac == 1.0, (frac, worst)
    assert np.linalg.norm(x - xo) / np.linalg.norm(xo) < 1e-10
    r = b - A.to_scipy() @ x
    assert np.linalg.norm(r) / np.linalg.norm(b) < 1e-10


@pytest.fixture(scope="module")
def c3_x14(c3):
    A, b, F = c3
    x14, _, _ = oracle.solve("fgmres", A, b, tol=1e-14, maxiter=3000, restart=30, pc="lu", factors=F, quirk=0)
    return x14


@pytest.mark.parametrize("factor", ["bf16", "fp16"])
@pytest.mark.parametrize("trsv", [0, 3])
def test_c4_mixed_gmres_parilut_vs_fp64_1e14(cuda, c3, c3_x14, factor, trsv):
    A, b, _ = c3
    S = _solver(A, "gmres", trsv)
    S.set_precision("fp64", "fp32", factor).set_inner(1e-4, 300)
    x = S.solve(b)
    relres = np.linalg.norm(b - A.to_scipy() @ x) / np.linalg.norm(b)
    assert relres < 1e-10, relres
    assert S.outer_steps() >= 2
    err = np.linalg.norm(x - c3_x14) / np.linalg.norm(c3_x14)
    print(f"C4 {factor} trsv={trsv}: relres {relres:.2e}, error vs FP64 1e-14 solve {err:.2e}")
    assert err < COND_BOUND * max(relres, 1e-14) + 1e-12, (err, relres)
