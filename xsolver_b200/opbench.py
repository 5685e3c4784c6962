"""Run and time single kernels of the solve path on a synthetic stencil.

    python -m xsolver_b200.opbench --grid 128 --ops csr64,lsolve,usolve
    python -m xsolver_b200.opbench --stencil convdiff27 --grid 64 --factor parilut --solve gmres

Each op in --ops is timed with CUDA events over --reps launches (L2 flushed
between launches) and printed with its algorithmic bytes and GB/s; --solve
runs whole solves of that Krylov method instead (its iteration kernels:
vector updates, SpMV epilogues, GMRES orthogonalisation).  This is the
command the kernel profiles are taken with: it launches each kernel a known,
small number of times on a fixed, seeded system.
"""
from __future__ import annotations

import argparse
import json

from . import stencils as st
from .api import Plan, Solver

STENCILS = {
    "poisson7": lambda g: st.poisson3d_7pt(g),
    "poisson5": lambda g: st.poisson2d_5pt(g),
    "convdiff27": lambda g: st.convdiff3d_27pt(g),
    "varcoef7": lambda g: st.varcoef3d_7pt(g, 0),
}


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--stencil", default="poisson7", choices=sorted(STENCILS))
    ap.add_argument("--grid", type=int, default=128)
    ap.add_argument("--factor", default="ilu0", choices=["ilu0", "parilu", "parilut", "ic0", "ilup", "ict"],
                    help="ilup: Saad ILUT (lfil 5, 1e-4), ict: ICT (5, 1e-4), factored on the host")
    ap.add_argument("--ops", default="", help="comma-separated: " + ",".join(Plan.OPS))
    ap.add_argument("--prec", default="fp64", choices=list(Plan.PREC), help="factor storage precision")
    ap.add_argument("--trsv", type=int, default=0, help="0 exact triangular solves, k>0 k Jacobi sweeps")
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--solve", default="", help="Krylov method for whole solves (bicgstab, cg, gmres, gcr, ...)")
    ap.add_argument("--mixed", action="store_true", help="whole solves by mixed-precision refinement")
    ap.add_argument("--solves", type=int, default=1)
    ap.add_argument("--batch", type=int, default=0,
                    help="k: PCG on k right-hand sides (seeds 0..k-1) with xs_solve_batch and xs_adjoint_batch, "
                         "timed against k single solves")
    ap.add_argument("--rtol", type=float, default=1e-10)
    a = ap.parse_args(argv)
    A = STENCILS[a.stencil](a.grid)
    out = {"stencil": a.stencil, "grid": a.grid, "n": A.n, "nnz": A.nnz}
    if a.ops:
        P = Plan(A).factor(a.factor, fill=2.0, sweeps=5 if a.factor == "parilut" else 20,
                           droptol=1e-4 if a.factor == "parilut" else 0.0)
        P.build_ell()
        P.set_factor_precision(a.prec).set_trsv(a.trsv)
        for op in a.ops.split(","):
            ms = P.time_op(op, reps=a.reps, flush_l2=True)
            by = P.op_bytes(op)
            out[op] = {"ms": ms, "bytes": by, "GBs": by / ms / 1e6}
        out["levels"] = P.levels()
    if a.batch:
        import time

        import numpy as np

        from . import _lib

        k = a.batch
        B = np.stack([st.rhs_uniform(A.n, c) for c in range(k)])
        L = _lib.lib()
        S = Solver(A).ksp_settype("cgm").ksp_setoption(a.rtol, 5000).pc_settype(a.factor).pc_set_trsv(a.trsv)
        res = {}
        for mode, on in (("batched", 1), ("one_by_one", 0)):
            L.xs_set_batch_kernels(on)
            Xw = S.solve_batch(B)  # setup and graph capture outside the timing
            S.adjoint_batch(Xw, Xw - 0.5)
            t0 = time.perf_counter()
            X = S.solve_batch(B)
            t1 = time.perf_counter()
            its = S.batch_iterations(k).tolist() if on else None
            G = X - 0.5
            t2 = time.perf_counter()
            S.adjoint_batch(X, G)
            t3 = time.perf_counter()
            res[mode] = {"forward_ms": (t1 - t0) * 1e3, "adjoint_ms": (t3 - t2) * 1e3, "iterations": its}
        L.xs_set_batch_kernels(1)
        out["batch"] = {"k": k, "rtol": a.rtol, **res}
    if a.solve:
        b = st.rhs_uniform(A.n, 0, 0.0 if a.stencil == "convdiff27" else -1.0, 1.0)
        S = Solver(A, fmt="ell").ksp_settype(a.solve).ksp_setoption(a.rtol, 3000, 30).pc_settype(a.factor)
        if a.factor == "parilut":
            S.pc_setparilut(2.0, 5, 1e-4)
        elif a.factor == "ilup":
            S.pc_setilut(1e-4, 5)
        elif a.factor == "ict":
            S.pc_setict(1e-4, 5)
        S.pc_set_trsv(a.trsv)
        if a.mixed:
            S.set_precision("fp64", "fp32", a.prec).set_inner(1e-4, 300)
        for _ in range(a.solves):
            S.solve(b)
        out["solve"] = S.timing()
    print(json.dumps(out))


if __name__ == "__main__":
    main()
