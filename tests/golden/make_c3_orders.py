"""Order-sensitivity fixture for the 160^3 27-point convection-diffusion
solves (Pe = 50, b ~ U(0,1) seed 0, x0 = 0, ParILUT fill 2 / 5 sweeps /
drop tolerance 1e-4, rtol 1e-10, restart 30): right-preconditioned GMRES
(the oracle's FGMRES with a fixed preconditioner) and the reference's GCR
(hip/Solver/xsolver_igcr.cpp:29-108, oracle "hip_igcr").

The restated reference loops are run once per valid dot-product summation
order (oracle.DOT_MODES) with the same ParILUT factors.  GMRES's residual
history at this size is sensitive to rounding in its last iterations: with
pairwise instead of sequential dots it moves by 1.5e-10 at iteration 18 and
1e-5 at iteration 21, where Gram-Schmidt works on nearly dependent vectors.
The fixture records, per method and order, the residual history and the
iteration count, and the largest relative distance of each order's solution
from the sequential one; tests/test_gpu_fullsize_c3.py derives its bounds
from it, and pins the sequential history to its own oracle run.

    python tests/golden/make_c3_orders.py      (about 20 minutes: the ParILUT
                                                restatement on all host
                                                threads, then 18 solves)
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import oracle  # noqa: E402
from xsolver_b200 import stencils as st  # noqa: E402


def main():
    A = st.convdiff3d_27pt(160)
    b = st.rhs_uniform(A.n, 0, 0.0, 1.0)
    F = oracle.parilut(A, fill=2.0, sweeps=5, droptol=1e-4)
    out = {}
    for method in ("fgmres", "hip_igcr"):
        xs = None
        xsens = 0.0
        try:
            for name in oracle.DOT_MODES:
                oracle.set_dot_mode(name)
                x, h, u = oracle.solve(method, A, b, tol=1e-10, maxiter=3000, restart=30, pc="lu", factors=F,
                                       quirk=0)
                out[f"{method}/{name}/hist"] = h
                out[f"{method}/{name}/usediter"] = np.int64(u)
                if name == "sequential":
                    xs = x
                else:
                    xsens = max(xsens, float(np.linalg.norm(x - xs) / np.linalg.norm(xs)))
                print(method, name, u, flush=True)
        finally:
            oracle.set_dot_mode("sequential")
        out[f"{method}/xsens"] = np.float64(xsens)
    out["orders"] = np.array(list(oracle.DOT_MODES))
    np.savez_compressed(os.path.join(HERE, "c3_orders.npz"), **out)


if __name__ == "__main__":
    main()
