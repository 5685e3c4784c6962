"""ORACLE — test infrastructure only.

ctypes bindings for
  liboracle.so              CPU restatement of the reference Krylov path
                            (xs_oracle.cpp, every function cites the reference
                            file:line it restates), and
  _ref/libxsref_intel.so    the reference's own intel/ CPU solver compiled from
  _ref/libxsref_ilu0.so     its sources, its hip ilu0_simple and ilutp_final,
  _ref/libxsref_ic0.so      IC(0) and
  _ref/libxsref_ict.so      ICT (Makefile), and
  liboracle_mt.so           the threaded BiCGSTAB + ILU(0) of the benchmark's
                            CPU reference arm (xs_oracle_mt.cpp; timing only).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may use
this package, as the checker or the timed CPU baseline.  The product path
(xsolver_b200) never imports it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None
_LIB_MT = None
_REF_INTEL = None
_REF_ILU0 = None
_REF_MMIO = None

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)


def build(ref: bool = True) -> None:
    """Compile liboracle.so (and the reference libraries when the reference
    sources are present)."""
    subprocess.run(["make", "-s", "-C", HERE, "all"], check=True)
    # the reference sources: XS_REFERENCE_DIR, else the directory "reference"
    # beside this repository's root
    refdir = os.environ.get("XS_REFERENCE_DIR",
                            os.path.normpath(os.path.join(HERE, "..", "..", "reference")))
    if ref and os.path.isdir(os.path.join(refdir, "intel")):
        subprocess.run(["make", "-s", "-C", HERE, "ref", f"REFERENCE={refdir}"], check=True)


def _p(a, t=np.float64):
    if a is None:
        return None
    assert a.dtype == t and a.flags["C_CONTIGUOUS"], (a.dtype, t)
    return a.ctypes.data_as(_dp if t == np.float64 else _ip)


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            build(ref=False)
        _LIB = C.CDLL(path)
    return _LIB


def lib_mt():
    global _LIB_MT
    if _LIB_MT is None:
        path = os.path.join(HERE, "liboracle_mt.so")
        if not os.path.exists(path):
            build(ref=False)
        L = C.CDLL(path)
        L.orcmt_bicgstab.restype = C.c_int
        _LIB_MT = L
    return _LIB_MT


def bicgstab_threads(A, b, F, tol=1e-10, maxiter=1000, threads=0, x0=None):
    """The reference BiCGSTAB + ILU(0) loop (intel/mpisolver-C-v1.cpp:365-482,
    LU apply hip/HostMatrix/HostMatrixCSR.cpp:385-409) with its SpMV and
    vector operations on `threads` host threads (0: all) and the triangular
    solves sequential; dot products in a fixed blocked order.  For timing
    (the benchmark's CPU reference arm); parity tests use solve().
    Returns (x, iterations, final relative residual)."""
    n = A.n
    x = np.zeros(n) if x0 is None else np.array(x0, dtype=np.float64)
    rsm = C.c_double()
    it = lib_mt().orcmt_bicgstab(n, _p(A.rowptr, np.int32), _p(A.colidx, np.int32), _p(A.val), _p(F.lrp, np.int32),
                                 _p(F.lci, np.int32), _p(F.lv), _p(F.dinv), _p(F.urp, np.int32),
                                 _p(F.uci, np.int32), _p(F.uv), _p(np.ascontiguousarray(b, np.float64)), _p(x),
                                 C.c_double(tol), int(maxiter), int(threads), C.byref(rsm))
    if it < 0:
        raise ValueError("orcmt_bicgstab: bad arguments")
    return x, it, rsm.value


def ref_intel():
    """The compiled reference intel/ solver, or None if it was not built."""
    global _REF_INTEL
    if _REF_INTEL is None:
        path = os.path.join(HERE, "_ref", "libxsref_intel.so")
        if not os.path.exists(path):
            return None
        _REF_INTEL = C.CDLL(path)
    return _REF_INTEL


def ref_ilu0():
    global _REF_ILU0
    if _REF_ILU0 is None:
        path = os.path.join(HERE, "_ref", "libxsref_ilu0.so")
        if not os.path.exists(path):
            return None
        _REF_ILU0 = C.CDLL(path)
    return _REF_ILU0


def ref_mmio():
    """The reference's compiled Matrix Market reader, or None."""
    global _REF_MMIO
    if _REF_MMIO is None:
        path = os.path.join(HERE, "_ref", "libxsref_mmio.so")
        if not os.path.exists(path):
            return None
        _REF_MMIO = C.CDLL(path)
    return _REF_MMIO


def ref_read_mtx(path):
    """(m, n, rowptr, colidx, val, diag, symmetric) from the reference's own
    reader, or None when it was not built."""
    R = ref_mmio()
    if R is None:
        return None
    m, n, nnz, sym = C.c_int(), C.c_int(), C.c_int(), C.c_int()
    assert R.ref_mmio_info(C.byref(m), C.byref(n), C.byref(nnz), C.byref(sym), path.encode()) == 0
    rp = np.zeros(max(m.value, n.value) + 1, np.int32)
    ci = np.zeros(max(nnz.value, 1), np.int32)
    v = np.zeros(max(nnz.value, 1))
    d = np.zeros(m.value)
    assert R.ref_mmio_data(_p(rp, np.int32), _p(ci, np.int32), _p(v), _p(d), path.encode()) == 0
    return m.value, n.value, rp[: m.value + 1], ci[: nnz.value], v[: nnz.value], d, sym.value


def read_mtx(path):
    """Restatement of the reference's Matrix Market reader
    (hip/Tool/ReadMatrix/csr_mmio_highlevel.h:118-233, mmio_data; sizes as
    mmio_info :8-116) for real/integer coordinate files: 1-based indices made
    0-based; general files store -value (the reference's negation), symmetric
    and hermitian files store value at (i, j) and, off the diagonal, at
    (j, i) too; diag[i] = value of entry (i, i) as read; rows filled in file
    order by a counting sort (:200-214).  Returns (m, n, rowptr, colidx, val,
    diag, symmetric)."""
    with open(path) as f:
        lines = f.read().split("\n")
    banner = lines[0].lower().split()
    symmetric = int("symmetric" in banner or "hermitian" in banner)
    k = 1
    while lines[k].startswith("%") or not lines[k].strip():
        k += 1
    m, n, nnz_rep = (int(t) for t in lines[k].split()[:3])
    rows, cols, vals = [], [], []
    diag = np.zeros(m)
    cnt = np.zeros(m + 1, np.int64)
    for line in lines[k + 1 : k + 1 + nnz_rep]:
        t = line.split()
        i, j, v = int(t[0]) - 1, int(t[1]) - 1, float(t[2])
        if not symmetric:
            rows.append(i); cols.append(j); vals.append(-v)
            cnt[i] += 1
        else:
            rows.append(i); cols.append(j); vals.append(v)
            cnt[i] += 1
            if i != j:
                rows.append(j); cols.append(i); vals.append(v)
                cnt[j] += 1
        if i == j:
            diag[i] = v
    rp = np.zeros(m + 1, np.int32)
    rp[1:] = np.cumsum(cnt[:m])
    nnz = int(rp[m])
    ci = np.zeros(nnz, np.int32)
    va = np.zeros(nnz)
    fill = rp[:-1].astype(np.int64).copy()
    for r, c, v in zip(rows, cols, vals):
        ci[fill[r]] = c
        va[fill[r]] = v
        fill[r] += 1
    return m, n, rp, ci, va, diag, symmetric


class LU:
    """Factors in the seqilu0 layout: L strict lower (unit diagonal implied),
    dinv = 1/u_ii, U' = dinv_i * u_ij strict upper (row-scaled)."""

    def __init__(self, n, lrp, lci, lv, dinv, urp, uci, uv):
        self.n = n
        self.lrp, self.lci, self.lv = lrp, lci, lv
        self.dinv = dinv
        self.urp, self.uci, self.uv = urp, uci, uv

    def args(self):
        return (_p(self.lrp, np.int32), _p(self.lci, np.int32), _p(self.lv), _p(self.dinv),
                _p(self.urp, np.int32), _p(self.uci, np.int32), _p(self.uv))


def _counts(A):
    rows = np.repeat(np.arange(A.n), np.diff(A.rowptr))
    nl = int((A.colidx < rows).sum())
    nu = int((A.colidx > rows).sum())
    return nl, nu


def ilu0(A) -> LU:
    nl, nu = _counts(A)
    n = A.n
    lrp = np.zeros(n + 1, np.int32); urp = np.zeros(n + 1, np.int32)
    lci = np.zeros(max(nl, 1), np.int32); uci = np.zeros(max(nu, 1), np.int32)
    lv = np.zeros(max(nl, 1)); uv = np.zeros(max(nu, 1)); dinv = np.zeros(n)
    rc = lib().orc_ilu0(n, _p(A.rowptr, np.int32), _p(A.colidx, np.int32), _p(A.val),
                        _p(lrp, np.int32), _p(lci, np.int32), _p(lv), _p(dinv),
                        _p(urp, np.int32), _p(uci, np.int32), _p(uv))
    if rc != 0:
        raise ValueError("matrix has a row without a diagonal entry")
    return LU(n, lrp, lci[:nl], lv[:nl], dinv, urp, uci[:nu], uv[:nu])


IC0_SMALLNUM = 1e-4  # Precond_ic0 defaults (hip/Precond/precon_ic0.h:14-15)
IC0_DROPTOL = 1e-4


def ic0_values(A, smallnum=IC0_SMALLNUM, droptol=IC0_DROPTOL) -> np.ndarray:
    """IC(0) factor in A's layout (lower part; inverted diagonals)."""
    out = np.zeros(A.nnz)
    rc = lib().orc_ic0_values(A.n, _p(A.rowptr, np.int32), _p(A.colidx, np.int32), _p(A.val), C.c_double(smallnum),
                              C.c_double(droptol), _p(out))
    if rc != 0:
        raise ValueError("matrix has a row without a diagonal entry")
    return out


def ic0(A, smallnum=IC0_SMALLNUM, droptol=IC0_DROPTOL) -> LU:
    """IC(0) as the seqilu0 factors of the LU solve (HostMatrixCSR::seqic0)."""
    nl, _ = _counts(A)
    n = A.n
    lrp = np.zeros(n + 1, np.int32); urp = np.zeros(n + 1, np.int32)
    lci = np.zeros(max(nl, 1), np.int32); uci = np.zeros(max(nl, 1), np.int32)
    lv = np.zeros(max(nl, 1)); uv = np.zeros(max(nl, 1)); dinv = np.zeros(n)
    rc = lib().orc_ic0(n, _p(A.rowptr, np.int32), _p(A.colidx, np.int32), _p(A.val), C.c_double(smallnum),
                       C.c_double(droptol), _p(lrp, np.int32), _p(lci, np.int32), _p(lv), _p(dinv),
                       _p(urp, np.int32), _p(uci, np.int32), _p(uv))
    if rc != 0:
        raise ValueError("matrix has a row without a diagonal entry")
    return LU(n, lrp, lci[:nl], lv[:nl], dinv, urp, uci[:nl], uv[:nl])


def ref_ic0_values(A, smallnum=IC0_SMALLNUM, droptol=IC0_DROPTOL):
    """The reference's own ic0_csr_A (compiled into oracle/_ref), mapped
    into A's layout, or None when it was not built."""
    path = os.path.join(HERE, "_ref", "libxsref_ic0.so")
    if not os.path.exists(path):
        return None
    R = C.CDLL(path)
    n = A.n
    cap = A.nnz + n
    lptr = np.zeros(n + 1, np.int32)
    lval = np.zeros(cap)
    lcol = np.zeros(cap, np.int32)
    R.ref_ic0_csr_A(n, _p(A.rowptr, np.int32), _p(np.ascontiguousarray(A.val)), _p(A.colidx, np.int32),
                    _p(lptr, np.int32), _p(lval), _p(lcol, np.int32), C.c_double(smallnum), C.c_double(droptol))
    out = A.val.astype(np.float64).copy()
    for i in range(n):
        k = A.rowptr[i]
        for q in range(lptr[i], lptr[i + 1]):
            assert A.colidx[k] == lcol[q]
            out[k] = lval[q]
            k += 1
    return out


def ilu0_values(A) -> np.ndarray:
    out = np.zeros(A.nnz)
    lib().orc_ilu0_values(A.n, _p(A.rowptr, np.int32), _p(A.colidx, np.int32), _p(A.val), _p(out))
    return out


def ref_ilu0_values(A):
    """Combined ILU(0) values from the reference's own ilu0_simple."""
    r = ref_ilu0()
    if r is None:
        return None
    out = np.zeros(A.nnz)
    uptr = np.zeros(A.n, np.int32)
    val = A.val.copy()
    rp = A.rowptr.copy(); ci = A.colidx.copy()
    r.ref_ilu0_simple(_p(out), _p(val), _p(rp, np.int32), _p(ci, np.int32), C.c_int(A.n), _p(uptr, np.int32))
    return out


def split_lu(A, luv) -> LU:
    nl, nu = _counts(A)
    n = A.n
    lrp = np.zeros(n + 1, np.int32); urp = np.zeros(n + 1, np.int32)
    lci = np.zeros(max(nl, 1), np.int32); uci = np.zeros(max(nu, 1), np.int32)
    lv = np.zeros(max(nl, 1)); uv = np.zeros(max(nu, 1)); dinv = np.zeros(n)
    luv = np.ascontiguousarray(luv, dtype=np.float64)
    rc = lib().orc_split_lu(n, _p(A.rowptr, np.int32), _p(A.colidx, np.int32), _p(luv),
                            _p(lrp, np.int32), _p(lci, np.int32), _p(lv), _p(dinv),
                            _p(urp, np.int32), _p(uci, np.int32), _p(uv))
    if rc != 0:
        raise ValueError("matrix has a row without a diagonal entry")
    return LU(n, lrp, lci[:nl], lv[:nl], dinv, urp, uci[:nu], uv[:nu])


def parilu_values(A, sweeps=20) -> np.ndarray:
    out = np.zeros(A.nnz)
    rc = lib().orc_parilu(A.n, _p(A.rowptr, np.int32), _p(A.colidx, np.int32), _p(A.val), C.c_int(sweeps), _p(out))
    if rc != 0:
        raise ValueError("matrix has a row without a diagonal entry")
    return out


def parilu_inplace_values(A, sweeps=20, order_seed=0) -> np.ndarray:
    """ParILU with the reference's in-place (asynchronous-style) updates:
    entries overwritten as they are computed, in A's order (order_seed 0)
    or a seeded random order per sweep."""
    out = np.zeros(A.nnz)
    rc = lib().orc_parilu_inplace(A.n, _p(A.rowptr, np.int32), _p(A.colidx, np.int32), _p(A.val), C.c_int(sweeps),
                                  C.c_uint(order_seed), _p(out))
    if rc != 0:
        raise ValueError("matrix has a row without a diagonal entry")
    return out


def parilu_inplace(A, sweeps=20, order_seed=0) -> LU:
    return split_lu(A, parilu_inplace_values(A, sweeps, order_seed))


def factor_residual(A, F: LU) -> float:
    """||(A - L U)|_pattern(A)||_F / ||A||_F for factors in the seqilu0
    layout (unit L, U = diag(1/dinv) U')."""
    import scipy.sparse as sp

    n = A.n
    Ls = sp.csr_matrix((F.lv, F.lci, F.lrp), shape=(n, n)) + sp.identity(n, format="csr")
    d = 1.0 / F.dinv
    Us = sp.diags(d) @ sp.csr_matrix((F.uv, F.uci, F.urp), shape=(n, n)) + sp.diags(d)
    P = (Ls @ Us).tocsr()
    rows = np.repeat(np.arange(n), np.diff(A.rowptr))
    lu = np.asarray(P[rows, A.colidx]).ravel()
    return float(np.linalg.norm(A.val - lu) / np.linalg.norm(A.val))


def parilu(A, sweeps=20) -> LU:
    return split_lu(A, parilu_values(A, sweeps))


def parilut(A, fill=2.0, sweeps=5, droptol=0.0) -> LU:
    L = C.CDLL  # placeholder to keep linters quiet
    ptrs = [C.POINTER(C.c_int)(), C.POINTER(C.c_int)(), C.POINTER(C.c_double)(), C.POINTER(C.c_double)(),
            C.POINTER(C.c_int)(), C.POINTER(C.c_int)(), C.POINTER(C.c_double)()]
    f = lib().orc_parilut
    rc = f(A.n, _p(A.rowptr, np.int32), _p(A.colidx, np.int32), _p(A.val), C.c_double(fill), C.c_int(sweeps),
           C.c_double(droptol), *[C.byref(p) for p in ptrs])
    if rc != 0:
        raise ValueError("matrix has a row without a diagonal entry")
    n = A.n
    lrp = np.ctypeslib.as_array(ptrs[0], (n + 1,)).copy()
    urp = np.ctypeslib.as_array(ptrs[4], (n + 1,)).copy()
    nl, nu = int(lrp[-1]), int(urp[-1])
    lci = np.ctypeslib.as_array(ptrs[1], (max(nl, 1),))[:nl].copy()
    lv = np.ctypeslib.as_array(ptrs[2], (max(nl, 1),))[:nl].copy()
    dinv = np.ctypeslib.as_array(ptrs[3], (n,)).copy()
    uci = np.ctypeslib.as_array(ptrs[5], (max(nu, 1),))[:nu].copy()
    uv = np.ctypeslib.as_array(ptrs[6], (max(nu, 1),))[:nu].copy()
    for p in ptrs:
        lib().orc_free(C.cast(p, C.c_void_p))
    del L
    return LU(n, lrp, lci, lv, dinv, urp, uci, uv)


ICT_SMALLNUM = 1e-4  # the constant the reference's seqict passes (hip/HostMatrix/HostMatrixCSR.cpp:331)


def _tri_out(n, cap):
    cap = max(cap, 1)
    return (np.zeros(n + 1, np.int32), np.zeros(cap, np.int32), np.zeros(cap), np.zeros(max(n, 1)),
            np.zeros(n + 1, np.int32), np.zeros(cap, np.int32), np.zeros(cap))


def _tri_lu(n, o):
    lrp, lci, lv, dinv, urp, uci, uv = o
    nl, nu = int(lrp[-1]), int(urp[-1])
    return LU(n, lrp, lci[:nl].copy(), lv[:nl].copy(), dinv[:n].copy(), urp, uci[:nu].copy(), uv[:nu].copy())


def ilut_saad(A, lfil=20, droptol=1e-5) -> LU:
    """Saad ILUT (restatement of ilutp_final + seqilut) in the seqilu0 layout."""
    o = _tri_out(A.n, A.n * lfil)
    lib().orc_ilut_saad(A.n, _p(A.rowptr, np.int32), _p(A.colidx, np.int32), _p(A.val), C.c_int(lfil),
                        C.c_double(droptol), *[_p(a, a.dtype.type) for a in o])
    return _tri_lu(A.n, o)


def ict(A, maxfil=100, droptol=1e-8) -> LU:
    """ICT (restatement of ict_csr_A_l + seqict) in the seqilu0 layout."""
    m = min(maxfil, max(A.n - 1, 0))
    o = _tri_out(A.n, A.n * m)
    rc = lib().orc_ict(A.n, _p(A.rowptr, np.int32), _p(A.colidx, np.int32), _p(A.val), C.c_int(maxfil),
                       C.c_double(droptol), *[_p(a, a.dtype.type) for a in o])
    if rc >= 0:
        raise ValueError(f"row {rc} has no diagonal entry")
    return _tri_lu(A.n, o)


def ref_ilut_saad(A, lfil=20, droptol=1e-5):
    """The reference's own ilutp_final (compiled into oracle/_ref) split as
    its seqilut does (hip/HostMatrix/HostMatrixCSR.cpp:230-268), or None
    when it was not built."""
    r = ref_ilu0()
    if r is None or not hasattr(r, "ref_ilutp_final"):
        return None
    n = A.n
    cap = (2 * lfil + 2) * n
    luval = np.zeros(cap); lucols = np.zeros(cap, np.int32)
    lurows = np.zeros(n + 1, np.int32); uptr = np.zeros(n + 1, np.int32); diag = np.zeros(max(n, 1))
    r.ref_ilutp_final(_p(luval), _p(A.val.copy()), _p(A.rowptr.copy(), np.int32), _p(A.colidx.copy(), np.int32),
                      C.c_int(n), _p(diag), C.c_int(lfil), _p(lucols, np.int32), _p(lurows, np.int32),
                      _p(uptr, np.int32), C.c_double(droptol))
    lrp = [0]; urp = [0]; lci = []; lv = []; uci = []; uv = []
    for i in range(n):
        lci.extend(lucols[lurows[i]:uptr[i]]); lv.extend(luval[lurows[i]:uptr[i]])
        uci.extend(lucols[uptr[i] + 1:lurows[i + 1]]); uv.extend(luval[uptr[i] + 1:lurows[i + 1]] * diag[i])
        lrp.append(len(lci)); urp.append(len(uci))
    return LU(n, np.array(lrp, np.int32), np.array(lci, np.int32), np.array(lv), diag[:n].copy(),
              np.array(urp, np.int32), np.array(uci, np.int32), np.array(uv))


def ref_ict(A, maxfil=100, droptol=1e-8):
    """The reference's own ict_csr_A_l (compiled into oracle/_ref), converted
    as its seqict does (hip/HostMatrix/HostMatrixCSR.cpp:327-384), or None
    when it was not built."""
    path = os.path.join(HERE, "_ref", "libxsref_ict.so")
    if not os.path.exists(path):
        return None
    R = C.CDLL(path)
    n = A.n
    m = min(maxfil, n - 1)  # hip/Precond/precon_ict.cpp:3-4
    cap = m * n + n
    lp = np.zeros(n + 1, np.int32); lval = np.zeros(cap); lcol = np.zeros(cap, np.int32)
    R.ref_ict_csr_A_l(n, _p(A.rowptr.copy(), np.int32), _p(A.val.copy()), _p(A.colidx.copy(), np.int32),
                      _p(lp, np.int32), _p(lval), _p(lcol, np.int32), C.c_double(ICT_SMALLNUM), C.c_double(droptol),
                      C.c_int(m))
    d = lval[lp[1:] - 1]
    lrp = [0]; lci = []; lv = []
    ucols = [[] for _ in range(n)]
    for i in range(n):
        for q in range(lp[i], lp[i + 1] - 1):
            j = int(lcol[q]); x = lval[q] * d[j]
            lci.append(j); lv.append(x); ucols[j].append((i, x))
        lrp.append(len(lci))
    urp = [0]; uci = []; uv = []
    for j in range(n):
        for i, x in ucols[j]:
            uci.append(i); uv.append(x)
        urp.append(len(uci))
    return LU(n, np.array(lrp, np.int32), np.array(lci, np.int32), np.array(lv), d * d,
              np.array(urp, np.int32), np.array(uci, np.int32), np.array(uv))


def lusolve(F: LU, x) -> np.ndarray:
    x = np.ascontiguousarray(x, dtype=np.float64)
    y = np.zeros(F.n)
    lib().orc_lusolve(F.n, *F.args()[:4], *F.args()[4:], _p(x), _p(y))
    return y


def lusolve_t(F: LU, x) -> np.ndarray:
    x = np.ascontiguousarray(x, dtype=np.float64)
    y = np.zeros(F.n)
    lib().orc_lusolve_t(F.n, *F.args(), _p(x), _p(y))
    return y


def spmv(A, x) -> np.ndarray:
    x = np.ascontiguousarray(x, dtype=np.float64)
    y = np.zeros(A.n)
    lib().orc_csr_spmv(A.n, _p(A.rowptr, np.int32), _p(A.colidx, np.int32), _p(A.val), _p(x), _p(y))
    return y


def spmv_t(A, x) -> np.ndarray:
    x = np.ascontiguousarray(x, dtype=np.float64)
    y = np.zeros(A.n)
    lib().orc_csr_spmv_t(A.n, _p(A.rowptr, np.int32), _p(A.colidx, np.int32), _p(A.val), _p(x), _p(y))
    return y


def levels_lower(n, rp, ci):
    lev = np.zeros(n, np.int32)
    nlev = lib().orc_levels_lower(n, _p(rp, np.int32), _p(ci, np.int32), _p(lev, np.int32))
    return lev, nlev


PC = {"none": 0, "jacobi": 1, "lu": 2}


DOT_MODES = {"sequential": 0, "pairwise": 1, "reverse": 2, "simd8": 3, "blocked": 4, "simd4": 5, "blocked256": 6,
             "strided4096": 7, "strided151552": 8}


def set_dot_mode(mode: str):
    """'sequential' (the reference's order) or another valid summation order:
    'pairwise', 'reverse', 'simd8', 'blocked', 'simd4', 'blocked256',
    'strided4096', 'strided151552'."""
    lib().orc_set_dot_mode(DOT_MODES[mode])


def solve(method, A, rhs, x0=None, tol=1e-8, maxiter=1000, restart=30, pc="jacobi", factors: LU | None = None,
          quirk=1):
    """Run a restated Krylov loop.  method: cg, cgm, icg, icgm, bicgstab,
    ibicgstab, gcr, igcr, hip_igcr, gmres, fgmres.  pc: none / jacobi / lu (needs factors).

    Returns (x, resvec, usediter).  resvec follows the restated loop's own
    convention: intel loops give relative residuals indexed by iteration;
    hip_igcr gives absolute residuals with resvec[0] = ||r0||."""
    n = A.n
    rhs = np.ascontiguousarray(rhs, dtype=np.float64)
    x = np.zeros(n) if x0 is None else np.ascontiguousarray(x0, dtype=np.float64).copy()
    x0c = x.copy()
    resvec = np.zeros(maxiter + 2)
    used = C.c_int(0)
    kind = PC[pc]
    fargs = factors.args() if (kind == 2) else (None,) * 7
    common = (n, _p(A.rowptr, np.int32), _p(A.colidx, np.int32), _p(A.val), kind, *fargs)
    L = lib()
    if method in ("cg", "cgm", "icg", "icgm", "bicgstab", "ibicgstab"):
        f = {"cg": L.orc_cg, "cgm": L.orc_cgm, "icg": L.orc_icg, "icgm": L.orc_icgm, "bicgstab": L.orc_bicgstab,
             "ibicgstab": L.orc_ibicgstab}[method]
        w = f(*common, _p(rhs), _p(x), C.c_double(tol), C.c_int(maxiter), _p(x0c), C.byref(used), _p(resvec))
    elif method in ("gcr", "igcr"):
        w = L.orc_gcr(*common, _p(rhs), _p(x), C.c_int(restart), C.c_double(tol), C.c_int(maxiter), _p(x0c),
                      C.byref(used), _p(resvec), C.c_int(1 if method == "igcr" else 0))
    elif method == "hip_igcr":
        w = L.orc_hip_igcr(*common, _p(rhs), _p(x), C.c_int(restart), C.c_double(tol), C.c_int(maxiter), _p(x0c),
                           C.byref(used), _p(resvec))
    elif method in ("gmres", "fgmres"):
        w = L.orc_gmres(*common, _p(rhs), _p(x), C.c_int(restart), C.c_double(tol), C.c_int(maxiter), _p(x0c),
                        C.byref(used), _p(resvec), C.c_int(1 if method == "fgmres" else 0), C.c_int(quirk))
    else:
        raise ValueError(method)
    return x, resvec[:w].copy(), used.value


def ref_solve(method, A, rhs, x0=None, tol=1e-8, maxiter=1000, restart=30):
    """Run the compiled reference intel/ solver with its Jacobi
    preconditioner (the only one it supports).  Returns (x, resvec, usediter)
    in the intel convention, or None when the reference was not built."""
    R = ref_intel()
    if R is None:
        return None
    n = A.n
    rows = np.repeat(np.arange(n), np.diff(A.rowptr))
    off = A.colidx != rows
    diag = np.zeros(n)
    diag[rows[~off]] = A.val[~off]
    offval = np.ascontiguousarray(A.val[off])
    offcol = np.ascontiguousarray(A.colidx[off])
    offptr = np.zeros(n + 1, np.int32)
    np.cumsum(np.bincount(rows[off], minlength=n), out=offptr[1:])
    nI, nH, nS = C.c_int(n), C.c_int(0), C.c_int(int(off.sum()))
    R.cpu_mat_setup(C.byref(nI), C.byref(nH), C.byref(nS), _p(diag), _p(offval), _p(offptr, np.int32),
                    _p(offcol, np.int32))
    R.cpu_preconditioner_setup(C.c_char_p(b"Jacobi"))
    rhs = np.ascontiguousarray(rhs, dtype=np.float64).copy()
    x = np.zeros(n) if x0 is None else np.ascontiguousarray(x0, dtype=np.float64).copy()
    x0c = x.copy()
    resvec = np.zeros(maxiter + 2)
    used = C.c_int(-1)
    t, mi, rs = C.c_double(tol), C.c_int(maxiter), C.c_int(restart)
    if method in ("cg", "cgm", "icg", "icgm", "bicgstab", "ibicgstab"):
        f = {"cg": R.cpu_cg_solve, "cgm": R.cpu_cgm_solve, "icg": R.cpu_icg_solve, "icgm": R.cpu_icgm_solve,
             "bicgstab": R.cpu_bicgstab_solve, "ibicgstab": R.cpu_ibicgstab_solve}[method]
        f(_p(rhs), _p(x), C.byref(t), C.byref(mi), _p(x0c), C.byref(used), _p(resvec))
    else:
        f = {"gcr": R.cpu_gcr_solve, "igcr": R.cpu_igcr_solve, "gmres": R.cpu_gmres_solve,
             "fgmres": R.cpu_fgmres_solve}[method]
        f(_p(rhs), _p(x), C.byref(rs), C.byref(t), C.byref(mi), _p(x0c), C.byref(used), _p(resvec))
    R.cpu_preconditioner_free(C.c_char_p(b"Jacobi"))
    return x, resvec, used.value
