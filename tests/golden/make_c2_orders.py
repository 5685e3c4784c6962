"""Order-sensitivity fixture for the 128^3 7-point BiCGSTAB + ILU(0) solve
(rtol 1e-10, b ~ U(-1,1) seed 0, x0 = 0).

The restated reference loop (oracle/, bitwise equal to the reference's CPU
code where both exist) is run once per valid dot-product summation order
(oracle.DOT_MODES).  At this size the BiCGSTAB residual history is very
sensitive to rounding: the reference itself ends anywhere in a range of
iterations depending on the order of its own dot products.  The fixture
records, per order, the relative residual history and the iteration count,
and the largest relative distance of each order's solution from the
sequential one; tests/test_gpu_fullsize.py derives its bounds from it.

    python tests/golden/make_c2_orders.py      (about 3 minutes, one core)
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import oracle  # noqa: E402
from xsolver_b200 import stencils as st  # noqa: E402


def main():
    A = st.poisson3d_7pt(128)
    b = st.rhs_uniform(A.n, 0)
    F = oracle.ilu0(A)
    out = {}
    xs = None
    xsens = 0.0
    try:
        for name in oracle.DOT_MODES:
            oracle.set_dot_mode(name)
            x, h, u = oracle.solve("bicgstab", A, b, tol=1e-10, maxiter=1000, pc="lu", factors=F)
            out[f"{name}/hist"] = h
            out[f"{name}/usediter"] = np.int64(u)
            if name == "sequential":
                xs = x
            else:
                xsens = max(xsens, float(np.linalg.norm(x - xs) / np.linalg.norm(xs)))
            print(name, u, flush=True)
    finally:
        oracle.set_dot_mode("sequential")
    out["xsens"] = np.float64(xsens)
    out["orders"] = np.array(list(oracle.DOT_MODES))
    np.savez_compressed(os.path.join(HERE, "c2_orders.npz"), **out)


if __name__ == "__main__":
    main()
