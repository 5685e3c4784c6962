"""The C-ABI library loads on a machine without a GPU, exports every symbol
include/xsolver_c.h declares, and refuses compute calls without a device."""
import ctypes as C

import numpy as np
import pytest

from xsolver_b200 import _lib
from xsolver_b200.build import LIB


def test_library_exports_every_declared_symbol():
    L = _lib.lib()
    names = _lib.declared_symbols()
    assert len(names) >= 60
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_reference_entry_points_present():
    L = _lib.lib()
    for n in ["xsolver_mat_setup", "xsolver_ksp_settype", "xsolver_ksp_set_absolute_tol", "xsolver_ksp_setoption",
              "xsolver_pc_settype", "xsolver_pc_setilut", "xsolver_pc_setict", "xsolver_solve", "xsolver_free",
              "cpu_mat_setup", "gpu_mat_setup", "gpu_mat_format", "gpu_preconditioner_setup", "gpu_cg_solve",
              "gpu_cgm_solve", "gpu_bicgstab_solve", "gpu_gcr_solve", "gpu_igcr_solve", "gpu_gmres_solve",
              "gpu_fgmres_solve"]:
        assert hasattr(L, n), n


def test_version_and_error_strings():
    L = _lib.lib()
    assert b"sm_100a" in L.xs_version()
    assert L.xsolver_error_string(5) == b"sync-free triangular solve timed out"


def test_host_only_level_analysis():
    """xs_tri_levels runs on the host: level of each row of a strict lower
    pattern and the level order; every dependency sits at a smaller position
    (the property that makes the ticket-ordered sync-free solve deadlock-free)."""
    import oracle
    from xsolver_b200 import stencils as st

    L = _lib.lib()
    for A in (st.poisson3d_7pt(7), st.convdiff3d_27pt(5), st.poisson2d_5pt(9)):
        n = A.n
        rows = np.repeat(np.arange(n), np.diff(A.rowptr))
        for upper in (0, 1):
            m = (A.colidx > rows) if upper else (A.colidx < rows)
            rp = np.zeros(n + 1, np.int32)
            np.cumsum(np.bincount(rows[m], minlength=n), out=rp[1:])
            ci = np.ascontiguousarray(A.colidx[m])
            lev = np.zeros(n, np.int32)
            perm = np.zeros(n, np.int32)
            nl = C.c_int()
            ip = C.POINTER(C.c_int)
            assert L.xs_tri_levels(n, rp.ctypes.data_as(ip), ci.ctypes.data_as(ip), upper, lev.ctypes.data_as(ip),
                                   perm.ctypes.data_as(ip), C.byref(nl)) == 0
            if not upper:
                ref, nref = oracle.levels_lower(n, rp, ci)
                assert np.array_equal(lev, ref) and nl.value == nref
            pos = np.empty(n, np.int64)
            pos[perm] = np.arange(n)
            for i in range(n):
                for k in range(rp[i], rp[i + 1]):
                    assert pos[ci[k]] < pos[i]
                    assert lev[ci[k]] < lev[i]
            assert sorted(perm.tolist()) == list(range(n))


def test_compute_calls_fail_loudly_without_gpu():
    from conftest import gpu_available

    if gpu_available():
        pytest.skip("a GPU is present")
    L = _lib.lib()
    h = C.c_void_p()
    assert L.xs_create(C.byref(h)) == 12  # XS_ERR_NO_GPU
    assert L.xs_device_count() == 0
    from xsolver_b200 import api, stencils as st

    with pytest.raises(api.XsError):
        api.Solver(st.poisson2d_5pt(4))


def test_library_path_is_in_tree():
    assert LIB.endswith("xsolver_b200/libxsolver_b200.so")


def test_wrapper_refuses_arrays_the_c_calls_would_overrun():
    """The C entry points take n (or nnz) elements with no length argument;
    the Python wrapper checks shapes, dtypes and devices before calling."""
    import torch

    from xsolver_b200 import api

    assert api._vec([1, 2, 3], (3,), "b").dtype == np.float64
    with pytest.raises(ValueError):
        api._vec(np.zeros(2), (3,), "b")
    with pytest.raises(ValueError):
        api._vec(np.zeros((3, 1)), (3,), "b")
    with pytest.raises(ValueError):
        api._dev(torch.zeros(3, dtype=torch.float64), 3, "float64", "x")  # host tensor
