"""Python mirror of the reference's solver interface over the C ABI.

Two layers, matching include/xsolver_c.h:

* ``Solver`` — one handle of the status-returning API (xs_*): the same
  settype / setoption / solve sequence as the reference's setter API
  (hip/xsolver_c.h:37-49), raising ``XsError`` on a non-zero status.
* ``Plan`` — kernel-level calls on device tensors (SpMV, ILU factorisation,
  sync-free LU solves, timing) used by the tests and the benchmark.

Module-level ``xsolver_*`` functions forward to the global-state entry points
with the reference's names and argument meaning.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import XsError, check, lib
from .stencils import CSRMatrix

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)


def _d(a):
    return a.ctypes.data_as(_dp)


def _i(a):
    return a.ctypes.data_as(_ip)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _vec(a, shape, what):
    """A contiguous float64 host array of exactly `shape`: the C entry
    points read and write n (or nnz) elements with no length argument."""
    a = _f64(a)
    if a.shape != tuple(shape):
        raise ValueError(f"{what}: expected shape {tuple(shape)}, got {a.shape}")
    return a


def _dev(t, n, dtype, what):
    """A CUDA tensor the kernels may read or write n elements of."""
    if not getattr(t, "is_cuda", False):
        raise ValueError(f"{what}: expected a CUDA tensor")
    if str(t.dtype) != f"torch.{dtype}":
        raise ValueError(f"{what}: expected {dtype}, got {t.dtype}")
    if not t.is_contiguous() or t.numel() < n:
        raise ValueError(f"{what}: expected a contiguous tensor of at least {n} elements")
    return t


class Solver:
    """A solver handle: matrix, Krylov method, preconditioner, precision."""

    def __init__(self, A: CSRMatrix, fmt: str = "csr"):
        self._L = lib()
        self.A = A
        self.h = C.c_void_p()
        check(self._L.xs_create(C.byref(self.h)), "xs_create")
        self._rp, self._ci, self._v = A.rowptr, A.colidx, A.val
        check(self._L.xs_mat_setup(self.h, A.n, _i(self._rp), _i(self._ci), _d(self._v), 1 if fmt == "ell" else 0),
              "xs_mat_setup")
        self._used = C.c_int(0)
        self._resvec = None
        self.maxiter = 0

    def mat_update(self, val):
        """New values for the same pattern (caller entry order)."""
        self._v = _vec(val, (self.A.nnz,), "mat_update values")
        check(self._L.xs_mat_update(self.h, _d(self._v)), "xs_mat_update")
        return self

    def close(self):
        if self.h:
            self._L.xs_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- reference-style configuration
    def ksp_settype(self, name: str):
        check(self._L.xs_ksp_settype(self.h, name.encode()), f"ksp_settype({name})")
        return self

    def ksp_setoption(self, tol: float, maxiter: int, restart: int = 0):
        self.maxiter = maxiter
        self._resvec = np.zeros(maxiter + 2)
        check(self._L.xs_ksp_setoption(self.h, tol, maxiter, C.byref(self._used), _d(self._resvec), restart),
              "ksp_setoption")
        return self

    def ksp_set_absolute_tol(self, tol: float):
        check(self._L.xs_ksp_set_absolute_tol(self.h, tol), "ksp_set_absolute_tol")
        return self

    def pc_settype(self, name: str):
        check(self._L.xs_pc_settype(self.h, name.encode()), f"pc_settype({name})")
        return self

    def pc_setilut(self, tol: float, max_fill: int):
        check(self._L.xs_pc_setilut(self.h, tol, max_fill), "pc_setilut")
        return self

    def pc_setict(self, tol: float, max_fill: int):
        check(self._L.xs_pc_setict(self.h, tol, max_fill), "pc_setict")
        return self

    def pc_setparilu(self, sweeps: int):
        check(self._L.xs_pc_setparilu(self.h, sweeps), "pc_setparilu")
        return self

    def pc_setparilut(self, fill: float, sweeps: int, droptol: float = 0.0):
        check(self._L.xs_pc_setparilut(self.h, fill, sweeps, droptol), "pc_setparilut")
        return self

    def pc_set_trsv(self, mode: int):
        check(self._L.xs_pc_set_trsv(self.h, mode), "pc_set_trsv")
        return self

    def set_precision(self, outer="fp64", inner="fp64", factor="fp64"):
        check(self._L.xs_set_precision(self.h, outer.encode(), inner.encode(), factor.encode()), "set_precision")
        return self

    def set_inner(self, rtol: float, maxiter: int):
        check(self._L.xs_set_inner(self.h, rtol, maxiter), "set_inner")
        return self

    def set_refinement_mode(self, carry_krylov: bool):
        check(self._L.xs_set_refinement_mode(self.h, 1 if carry_krylov else 0), "set_refinement_mode")
        return self

    def set_compat(self, quirks: int):
        check(self._L.xs_set_compat(self.h, quirks), "set_compat")
        return self

    # -- solve
    def solve(self, b, x0=None, out=None) -> np.ndarray:
        """Host arrays.  out (float64, contiguous, e.g. a pinned buffer), if
        given, holds x0 on entry and receives the solution in place."""
        n = self.A.n
        b = _vec(b, (n,), "rhs")
        if out is not None:
            if out.dtype != np.float64 or not out.flags.c_contiguous or out.shape != (n,):
                raise ValueError(f"out must be a contiguous float64 array of shape ({n},)")
            x = out
        else:
            x = np.zeros(n) if x0 is None else _vec(x0, (n,), "x0").copy()
        check(self._L.xs_solve(self.h, _d(b), _d(x)), "xs_solve")
        return x

    def solve_device(self, b, x):
        """b, x: CUDA tensors (float64, n); x holds x0 and receives the solution."""
        _dev(b, self.A.n, "float64", "rhs")
        _dev(x, self.A.n, "float64", "x")
        check(self._L.xs_solve_device(self.h, C.c_void_p(b.data_ptr()), C.c_void_p(x.data_ptr())), "xs_solve_device")
        return x

    def solve_batch(self, B) -> np.ndarray:
        B = _f64(B)
        if B.ndim != 2 or B.shape[1] != self.A.n:
            raise ValueError(f"solve_batch: expected shape (k, {self.A.n}), got {B.shape}")
        X = np.zeros_like(B)
        check(self._L.xs_solve_batch(self.h, B.shape[0], _d(B), _d(X)), "xs_solve_batch")
        return X

    def batch_iterations(self, k: int):
        it = np.zeros(k, np.int32)
        check(self._L.xs_batch_iterations(self.h, k, _i(it)), "xs_batch_iterations")
        return it

    @property
    def usediter(self) -> int:
        return self._used.value

    def resvec(self, count=None) -> np.ndarray:
        k = self.usediter + 1 if count is None else count
        return self._resvec[:k].copy()

    def timing(self):
        s, t, r = C.c_double(), C.c_double(), C.c_double()
        it = C.c_int()
        check(self._L.xs_last_timing(self.h, C.byref(s), C.byref(t), C.byref(it), C.byref(r)), "xs_last_timing")
        return {"setup_ms": s.value, "solve_ms": t.value, "iterations": it.value, "final_relres": r.value}

    def stream_ptr(self) -> int:
        p = C.c_void_p()
        check(self._L.xs_get_stream(self.h, C.byref(p)), "xs_get_stream")
        return p.value or 0

    def launches(self) -> int:
        c = C.c_longlong()
        check(self._L.xs_last_launches(self.h, C.byref(c)), "xs_last_launches")
        return c.value

    def outer_steps(self) -> int:
        o = C.c_int()
        check(self._L.xs_last_outer_steps(self.h, C.byref(o)), "xs_last_outer_steps")
        return o.value

    # -- adjoint
    def adjoint(self, dLdx, want_b=True, want_A=True):
        g = _vec(dLdx, (self.A.n,), "dLdx")
        db = np.zeros(self.A.n) if want_b else None
        dA = np.zeros(self.A.nnz) if want_A else None
        check(self._L.xs_adjoint(self.h, _d(g), _d(db) if db is not None else None, _d(dA) if dA is not None else None),
              "xs_adjoint")
        return db, dA

    def adjoint_batch(self, X, G):
        X = _f64(X)
        if X.ndim != 2 or X.shape[1] != self.A.n:
            raise ValueError(f"adjoint_batch: expected X of shape (k, {self.A.n}), got {X.shape}")
        G = _vec(G, X.shape, "adjoint_batch G")
        k = X.shape[0]
        DB = np.zeros_like(X)
        DA = np.zeros((k, self.A.nnz))
        check(self._L.xs_adjoint_batch(self.h, k, _d(X), _d(G), _d(DB), _d(DA)), "xs_adjoint_batch")
        return DB, DA


class Plan:
    """Kernel-level access on device tensors (torch CUDA tensors)."""

    FACTOR_KIND = {"ilu0": 0, "parilu": 1, "parilut": 2, "ic0": 3, "ilup": 4, "ict": 5}
    PREC = {"fp64": 0, "fp32": 1, "bf16": 2, "fp16": 3}
    OPS = {"csr64": 0, "ell64": 1, "csr32": 2, "lsolve": 3, "usolve": 4, "lusolve": 5, "ell32": 6}

    def __init__(self, A: CSRMatrix):
        self._L = lib()
        self.A = A
        self.p = C.c_void_p()
        self._keep = (A.rowptr, A.colidx, A.val)
        self._pending = []
        check(self._L.xs_plan_create(C.byref(self.p), A.n, _i(A.rowptr), _i(A.colidx), _d(A.val)), "xs_plan_create")
        self.ell_width = 0
        self.kind = None

    def close(self):
        if self.p:
            self._L.xs_plan_destroy(self.p)
            self.p = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def build_ell(self) -> int:
        w = C.c_int()
        check(self._L.xs_plan_build_ell(self.p, C.byref(w)), "build_ell")
        self.ell_width = w.value
        return w.value

    def _hold(self, *tensors):
        """Device tensors used by work queued on the plan's stream stay
        referenced until sync(): torch's allocator does not see that stream
        and could otherwise hand their memory to a new tensor first."""
        self._pending.extend(tensors)

    def spmv(self, x, y, fmt="csr", precision="fp64"):
        dt = "float64" if precision == "fp64" else "float32"
        _dev(x, self.A.n, dt, "x")
        _dev(y, self.A.n, dt, "y")
        check(self._L.xs_plan_spmv(self.p, 1 if fmt == "ell" else 0, 0 if precision == "fp64" else 1,
                                   C.c_void_p(x.data_ptr()), C.c_void_p(y.data_ptr())), "spmv")
        self._hold(x, y)
        return y

    def spmv_t(self, x, y):
        _dev(x, self.A.n, "float64", "x")
        _dev(y, self.A.n, "float64", "y")
        check(self._L.xs_plan_spmv_t(self.p, C.c_void_p(x.data_ptr()), C.c_void_p(y.data_ptr())), "spmv_t")
        self._hold(x, y)
        return y

    def factor(self, kind="ilu0", sweeps=20, fill=2.0, droptol=0.0):
        check(self._L.xs_plan_factor(self.p, self.FACTOR_KIND[kind], sweeps, fill, droptol), f"factor({kind})")
        self.kind = kind
        return self

    def lu_values(self) -> np.ndarray:
        out = np.zeros(self.A.nnz)
        check(self._L.xs_plan_get_lu_values(self.p, _d(out)), "get_lu_values")
        return out

    def factors(self):
        nl, nu = C.c_int(), C.c_int()
        check(self._L.xs_plan_get_factors(self.p, C.byref(nl), C.byref(nu), None, None, None, None, None, None, None),
              "get_factors")
        n = self.A.n
        lrp = np.zeros(n + 1, np.int32); urp = np.zeros(n + 1, np.int32)
        lci = np.zeros(max(nl.value, 1), np.int32); uci = np.zeros(max(nu.value, 1), np.int32)
        lv = np.zeros(max(nl.value, 1)); uv = np.zeros(max(nu.value, 1)); dinv = np.zeros(n)
        check(self._L.xs_plan_get_factors(self.p, C.byref(nl), C.byref(nu), _i(lrp), _i(lci), _d(lv), _d(dinv),
                                          _i(urp), _i(uci), _d(uv)), "get_factors")
        return dict(lrp=lrp, lci=lci[:nl.value], lv=lv[:nl.value], dinv=dinv, urp=urp, uci=uci[:nu.value],
                    uv=uv[:nu.value])

    def set_factor_precision(self, prec="fp64"):
        check(self._L.xs_plan_set_factor_precision(self.p, self.PREC[prec]), "set_factor_precision")
        return self

    def set_trsv(self, mode: int):
        check(self._L.xs_plan_set_trsv(self.p, mode), "set_trsv")
        return self

    def lusolve(self, x, z):
        prec = 0 if str(x.dtype) == "torch.float64" else 1
        dt = "float64" if prec == 0 else "float32"
        _dev(x, self.A.n, dt, "x")
        _dev(z, self.A.n, dt, "z")
        check(self._L.xs_plan_lusolve(self.p, prec, C.c_void_p(x.data_ptr()), C.c_void_p(z.data_ptr())), "lusolve")
        self._hold(x, z)
        return z

    def lusolve_batch(self, X, Z):
        """k LU solves on (n, k) row-major CUDA tensors (column c of row i at
        i*k + c), FP64."""
        if X.dim() != 2 or X.shape[0] != self.A.n or tuple(Z.shape) != tuple(X.shape):
            raise ValueError(f"lusolve_batch: expected X and Z of shape ({self.A.n}, k)")
        _dev(X, X.numel(), "float64", "X")
        _dev(Z, Z.numel(), "float64", "Z")
        check(self._L.xs_plan_lusolve_batch(self.p, X.shape[1], C.c_void_p(X.data_ptr()), C.c_void_p(Z.data_ptr())),
              "lusolve_batch")
        self._hold(X, Z)
        return Z

    def lusolve_t(self, x, z):
        _dev(x, self.A.n, "float64", "x")
        _dev(z, self.A.n, "float64", "z")
        check(self._L.xs_plan_lusolve_t(self.p, C.c_void_p(x.data_ptr()), C.c_void_p(z.data_ptr())), "lusolve_t")
        self._hold(x, z)
        return z

    def sync(self):
        try:
            check(self._L.xs_plan_sync(self.p), "plan sync")
        finally:
            self._pending.clear()

    def stream(self):
        """The plan's CUDA stream as a torch stream object: work ordered on it
        (or made to wait on it with events) follows the plan's calls without
        a sync().  The plan owns the stream and destroys it in close(), so a
        tensor must not be given to it with record_stream(): torch's
        allocator would record an event on it when the tensor is freed,
        which can be after the plan is gone.  The plan itself keeps the
        tensors of its queued work referenced until sync()."""
        import torch

        s = C.c_void_p()
        check(self._L.xs_plan_get_stream(self.p, C.byref(s)), "plan stream")
        return torch.cuda.ExternalStream(s.value or 0, device=torch.device("cuda", torch.cuda.current_device()))

    def debug_break_dependency(self, position: int, enable: bool = True):
        check(self._L.xs_plan_debug_break_dependency(self.p, position, 1 if enable else 0), "debug_break_dependency")

    def levels(self):
        a, b = C.c_int(), C.c_int()
        check(self._L.xs_plan_levels(self.p, C.byref(a), C.byref(b)), "levels")
        return a.value, b.value

    def time_op(self, op: str, reps: int = 20, flush_l2: bool = True) -> float:
        ms = C.c_double()
        check(self._L.xs_plan_time_op(self.p, self.OPS[op], reps, 1 if flush_l2 else 0, C.byref(ms)), f"time_op({op})")
        return ms.value

    def op_bytes(self, op: str) -> float:
        b = C.c_double()
        check(self._L.xs_plan_op_bytes(self.p, self.OPS[op], C.byref(b)), f"op_bytes({op})")
        return b.value


# ---------------------------------------------------------------- reference-style globals
_g = {}


def xsolver_mat_setup(n, rowptr, colidx, val, advanced_pam=(0, 0, 1)):
    rp = np.ascontiguousarray(rowptr, np.int32)
    ci = np.ascontiguousarray(colidx, np.int32)
    v = np.ascontiguousarray(val, np.float64)
    pam = np.ascontiguousarray(advanced_pam, np.int32)
    _g["keep"] = (rp, ci, v, pam)
    lib().xsolver_mat_setup(n, _i(rp), _i(ci), _d(v), _i(pam))
    return _lib.last_error()


def xsolver_ksp_settype(name):
    lib().xsolver_ksp_settype(name.encode())
    return _lib.last_error()


def xsolver_ksp_setoption(tol, maxiter, restart=0):
    _g["used"] = C.c_int(0)
    _g["resvec"] = np.zeros(maxiter + 2)
    lib().xsolver_ksp_setoption(tol, maxiter, C.byref(_g["used"]), _d(_g["resvec"]), restart)
    return _lib.last_error()


def xsolver_pc_settype(name):
    lib().xsolver_pc_settype(name.encode())
    return _lib.last_error()


def xsolver_pc_setilut(tol, max_fill):
    lib().xsolver_pc_setilut(tol, max_fill)
    return _lib.last_error()


def xsolver_pc_setict(tol, max_fill):
    lib().xsolver_pc_setict(tol, max_fill)
    return _lib.last_error()


def xsolver_solve(rhs, sol):
    rhs = _f64(rhs)
    if "keep" in _g:  # the system set by xsolver_mat_setup fixes the length
        n = len(_g["keep"][0]) - 1
        rhs = _vec(rhs, (n,), "rhs")
        if sol.shape != (n,):
            raise ValueError(f"sol: expected shape ({n},), got {sol.shape}")
    if sol.dtype != np.float64 or not sol.flags["C_CONTIGUOUS"]:
        raise ValueError("sol must be a contiguous float64 array (x0 in, solution out)")
    lib().xsolver_solve(_d(rhs), _d(sol))
    return _lib.last_error()


def xsolver_usediter():
    return _g["used"].value


def xsolver_resvec():
    return _g["resvec"]


def xsolver_free():
    lib().xsolver_free()
    return _lib.last_error()


__all__ = ["Solver", "Plan", "XsError", "xsolver_mat_setup", "xsolver_ksp_settype", "xsolver_ksp_setoption",
           "xsolver_pc_settype", "xsolver_pc_setilut", "xsolver_pc_setict", "xsolver_solve", "xsolver_free", "xsolver_usediter",
           "xsolver_resvec"]


def _host_factor(fn, name, A, fill, droptol, cap):
    n = A.n
    rp = np.ascontiguousarray(A.rowptr, np.int32); ci = np.ascontiguousarray(A.colidx, np.int32)
    v = np.ascontiguousarray(A.val, np.float64)
    cap = max(cap, 1)
    lrp = np.zeros(n + 1, np.int32); urp = np.zeros(n + 1, np.int32)
    lci = np.zeros(cap, np.int32); uci = np.zeros(cap, np.int32)
    lv = np.zeros(cap); uv = np.zeros(cap); dinv = np.zeros(max(n, 1))
    nl, nu = C.c_int(), C.c_int()
    check(fn(n, _i(rp), _i(ci), _d(v), fill, droptol, C.byref(nl), C.byref(nu), _i(lrp), _i(lci), _d(lv), _d(dinv),
             _i(urp), _i(uci), _d(uv)), name)
    return dict(lrp=lrp, lci=lci[:nl.value].copy(), lv=lv[:nl.value].copy(), dinv=dinv[:n].copy(), urp=urp,
                uci=uci[:nu.value].copy(), uv=uv[:nu.value].copy())


def host_ilut(A, lfil: int, droptol: float):
    """Saad ILUT(droptol, lfil) of A computed by the library on the host (no
    device needed), in the L / dinv / U' layout of Plan.factors()."""
    return _host_factor(lib().xs_host_ilut, "host_ilut", A, int(lfil), float(droptol), A.n * int(lfil))


def host_ict(A, maxfil: int, droptol: float):
    """ICT(droptol, maxfil) of the symmetric A computed by the library on the
    host, in the L / dinv / U' layout of Plan.factors()."""
    m = min(int(maxfil), max(A.n - 1, 0))
    return _host_factor(lib().xs_host_ict, "host_ict", A, int(maxfil), float(droptol), A.n * m)
