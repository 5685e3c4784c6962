"""Generate the golden fixtures in this directory from the reference's own
CPU code, compiled from its sources by oracle/Makefile into oracle/_ref:

  krylov_jacobi.npz   intel/ cpu_{cg,cgm,bicgstab,gcr,igcr,gmres,fgmres}_solve
                      (Jacobi, the only preconditioner intel/ has) on small
                      seeded stencil systems: matrix, rhs, solution, resvec,
                      usediter.
  ilu0.npz            hip ilu0_simple (hip/Precond/ilut_diag_in_csr.cpp:347)
                      combined LU values on small stencil matrices.
  krylov_single_reduction.npz
                      intel/ cpu_{icg,icgm,ibicgstab}_solve
                      (intel/mpisolver-C-v1.cpp:104-191, 273-363, 484-683)
                      with Jacobi on the same systems (icg/icgm on the
                      symmetric ones); same fields as krylov_jacobi.npz.
  ic0.npz             hip ic0_csr_A (hip/Precond/ic0.cpp:72-81) with the
                      Precond_ic0 defaults, in A's layout, on small
                      symmetric stencil matrices.
  threshold_factors.npz
                      hip ilutp_final (hip/Precond/ilut_diag_in_csr.cpp:20-251)
                      split as seqilut, and ict_csr_A_l (hip/Precond/
                      ict_l.cpp:196-201) converted as seqict, in the
                      L / dinv / U' layout, for two parameter sets each on
                      small matrices (one with a zero pivot, which takes the
                      pivot substitute).

Run here (where the reference sources exist):
    python tests/golden/make_golden.py [file.npz ...]   (default: all files)
The fixtures are committed; tests never need the reference sources.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import oracle  # noqa: E402
from xsolver_b200 import stencils as st  # noqa: E402

PROBLEMS = {
    "p2d_5pt_24": (lambda: st.poisson2d_5pt(24), 0, -1.0, 1.0),
    "p3d_7pt_9": (lambda: st.poisson3d_7pt(9), 1, -1.0, 1.0),
    "cd3d_27pt_7": (lambda: st.convdiff3d_27pt(7), 2, 0.0, 1.0),
    "vc3d_7pt_8": (lambda: st.varcoef3d_7pt(8, 3), 3, -1.0, 1.0),
}
METHODS = ["cg", "cgm", "bicgstab", "gcr", "igcr", "gmres", "fgmres"]
SINGLE_REDUCTION = ["icg", "icgm", "ibicgstab"]
IC0_MATRICES = {
    "p2d_5pt_15": lambda: st.poisson2d_5pt(15),
    "vc3d_7pt_7": lambda: st.varcoef3d_7pt(7, 2),
    "p3d_7pt_8": lambda: st.poisson3d_7pt(8),
    "vc3d_7pt_5": lambda: st.varcoef3d_7pt(5, 7),
}


def krylov(methods):
    kr = {}
    for name, (gen, seed, lo, hi) in PROBLEMS.items():
        A = gen()
        b = st.rhs_uniform(A.n, seed, lo, hi)
        kr[f"{name}/rowptr"] = A.rowptr
        kr[f"{name}/colidx"] = A.colidx
        kr[f"{name}/val"] = A.val
        kr[f"{name}/rhs"] = b
        for m in methods:
            sym = name.startswith(("p2d", "p3d", "vc3d"))
            if m in ("cg", "cgm", "icg", "icgm") and not sym:
                continue
            x, rv, used = oracle.ref_solve(m, A, b, tol=1e-9, maxiter=400, restart=20)
            kr[f"{name}/{m}/x"] = x
            kr[f"{name}/{m}/resvec"] = rv
            kr[f"{name}/{m}/usediter"] = np.array(used)
    return kr


def _zero_pivot():
    A = st.poisson2d_5pt(12)
    v = A.val.copy()
    v[A.rowptr[0]] = 0.0  # row 0's diagonal (its first entry)
    return st.CSRMatrix(A.n, A.rowptr, A.colidx, v, "p2d_5pt_12_zero_pivot")


THRESHOLD_MATRICES = {
    "p2d_5pt_16": lambda: st.poisson2d_5pt(16),
    "p3d_7pt_7": lambda: st.poisson3d_7pt(7),
    "vc3d_7pt_6": lambda: st.varcoef3d_7pt(6, 4),
    "p2d_zero_pivot": _zero_pivot,
}
ILUT_PARAMS = [(5, 1e-4), (2, 1e-2)]
ICT_PARAMS = [(5, 1e-4), (20, 1e-6)]
FACTOR_KEYS = ("lrp", "lci", "lv", "dinv", "urp", "uci", "uv")


def threshold_factors():
    out = {}
    for name, gen in THRESHOLD_MATRICES.items():
        A = gen()
        out[f"{name}/rowptr"] = A.rowptr
        out[f"{name}/colidx"] = A.colidx
        out[f"{name}/val"] = A.val
        for tag, params, fn in (("ilut", ILUT_PARAMS, oracle.ref_ilut_saad), ("ict", ICT_PARAMS, oracle.ref_ict)):
            for p, (fill, tol) in enumerate(params):
                F = fn(A, fill, tol)
                out[f"{name}/{tag}{p}/params"] = np.array([fill, tol])
                for k in FACTOR_KEYS:
                    out[f"{name}/{tag}{p}/{k}"] = getattr(F, k)
    return out


def factor_values(matrices, values):
    out = {}
    for name, gen in matrices.items():
        A = gen()
        out[f"{name}/rowptr"] = A.rowptr
        out[f"{name}/colidx"] = A.colidx
        out[f"{name}/val"] = A.val
        out[f"{name}/luv"] = values(A)
    return out


FILES = {
    "krylov_jacobi.npz": lambda: krylov(METHODS),
    "ilu0.npz": lambda: factor_values({k: v[0] for k, v in PROBLEMS.items()}, oracle.ref_ilu0_values),
    "krylov_single_reduction.npz": lambda: krylov(SINGLE_REDUCTION),
    "ic0.npz": lambda: factor_values(IC0_MATRICES, oracle.ref_ic0_values),
    "threshold_factors.npz": threshold_factors,
}


def main(names):
    oracle.build(ref=True)
    if oracle.ref_intel() is None:
        raise SystemExit("reference not built (needs the reference sources)")
    for fname in names or FILES:
        np.savez_compressed(os.path.join(HERE, fname), **FILES[fname]())
        print("wrote", fname)


if __name__ == "__main__":
    main(sys.argv[1:])
