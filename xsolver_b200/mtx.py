"""Matrix Market files through the library's reader (xs_mm_info /
xs_mm_read), and the reference driver's solve of one (hip/main_solve_base.cpp
with hip/solve_base.h: b = 1, x0 = 0, BiCGSTAB + ILUT(1e-4, 5), rtol 1e-4,
300 iterations)."""
import ctypes as C

import numpy as np

from ._lib import lib
from ._lib import check
from .api import Solver
from .stencils import CSRMatrix


def read_mtx(path, reference_quirks=True):
    """Returns (A, diag, symmetric).  reference_quirks=True gives the
    reference reader's matrix (general files negated, see
    include/xsolver_c.h); False keeps general files' values as written."""
    L = lib()
    m, n, nnz, sym = C.c_int(), C.c_int(), C.c_int(), C.c_int()
    check(L.xs_mm_info(str(path).encode(), C.byref(m), C.byref(n), C.byref(nnz), C.byref(sym)), "xs_mm_info")
    rp = np.zeros(m.value + 1, np.int32)
    ci = np.zeros(max(nnz.value, 1), np.int32)
    v = np.zeros(max(nnz.value, 1))
    d = np.zeros(max(m.value, 1))
    ip, dp = C.POINTER(C.c_int), C.POINTER(C.c_double)
    check(L.xs_mm_read(str(path).encode(), 1 if reference_quirks else 0, rp.ctypes.data_as(ip), ci.ctypes.data_as(ip),
                       v.ctypes.data_as(dp), d.ctypes.data_as(dp)), "xs_mm_read")
    if m.value != n.value:
        raise ValueError(f"{path}: {m.value} x {n.value} matrix is not square")
    A = CSRMatrix(m.value, rp, ci[: nnz.value], v[: nnz.value], str(path))
    return A, d[: m.value], bool(sym.value)


def solve_mtx(path, tol=1e-4, maxiter=300, ksp="bicgstab", pc="ilut", ilut=(1e-4, 5)):
    """The reference driver's flow on a file: its reader, b = 1, x0 = 0,
    restart = maxiter.  Returns (x, solver)."""
    A, _, _ = read_mtx(path)
    S = Solver(A).ksp_settype(ksp).ksp_setoption(tol, maxiter, maxiter).pc_settype(pc)
    if pc == "ilut":
        S.pc_setilut(*ilut)
    x = S.solve(np.ones(A.n))
    return x, S
