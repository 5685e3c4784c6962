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
    hip/Solver/xsolver_igcr.cpp:29-108), against the oracle run on the same
    factors: the per-iteration residual history within 1e-10 relative
    wherever the reference's own summation-order spread allows it and
    within 10 times that spread elsewhere (tests/parity.py; the spread comes
    from tests/golden/c3_orders.npz — GMRES's last iterations move by up to
    1e-5 between two valid dot orders of the reference itself), the
    iteration count within the reference's own range over the orders +-1,
    and the solution within max(1e-10, 10 x the orders' spread);
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
import os

import numpy as np
import pytest

import oracle
from parity import history_bound, history_ok
from xsolver_b200 import stencils as st

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")

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
    z = np.load(os.path.join(GOLD, "c3_orders.npz"))
    orders = [str(o) for o in z["orders"]]
    assert np.array_equal(z[f"{oracle_method}/sequential/hist"], ho)  # the fixture is this oracle run
    hb = history_bound(ho, [z[f"{oracle_method}/{o}/hist"] for o in orders if o != "sequential"])
    its = [int(z[f"{oracle_method}/{o}/usediter"]) for o in orders]
    xb = max(1e-10, 10.0 * float(z[f"{oracle_method}/xsens"]))
    if oracle_method == "hip_igcr":  # absolute residuals, [0] = ||r0||, count = last index
        ok, worst = history_ok(hist, ho, hb, scale=ho[0])
        count, lo, hi = S.usediter, min(its), max(its)
    else:
        ok, worst = history_ok(hist[1:] / hist[0], ho, hb)
        count, lo, hi = S.usediter, min(its) + 1, max(its) + 1
    print(f"C3 {ksp}: {S.usediter} iterations (reference over orders {lo}-{hi})")
    assert ok, worst
    assert lo - 1 <= count <= hi + 1, (count, lo, hi)
    assert np.linalg.norm(x - xo) / np.linalg.norm(xo) < xb
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
