"""ctypes loader for libxsolver_b200.so (the in-tree CUDA build).

There is no fallback: importing works without a GPU (so the ABI can be
inspected), but every compute entry point fails with an explicit error when
the library is missing or no CUDA device is visible.
"""
from __future__ import annotations

import ctypes as C
import os
import re

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libxsolver_b200.so")
HEADER = os.path.join(HERE, "..", "include", "xsolver_c.h")

_lib = None

XS_STATUS = {
    0: "XS_OK", 1: "XS_ERR_INVALID", 2: "XS_ERR_CUDA", 3: "XS_ERR_NOMEM", 4: "XS_ERR_NO_DIAG",
    5: "XS_ERR_TRSV_TIMEOUT", 6: "XS_ERR_BREAKDOWN", 7: "XS_ERR_NAN", 8: "XS_ERR_ORDER",
    9: "XS_ERR_ELL_WIDTH", 10: "XS_ERR_UNSUPPORTED", 11: "XS_ERR_CAPACITY", 12: "XS_ERR_NO_GPU",
}


class XsError(RuntimeError):
    def __init__(self, code: int, what: str = ""):
        self.code = code
        super().__init__(f"{what}: {XS_STATUS.get(code, code)}")


def lib() -> C.CDLL:
    """Load the CUDA library; raises if it was not built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(
                f"libxsolver_b200.so not found at {LIB_PATH}; build it with `python -m xsolver_b200.build`")
        _lib = C.CDLL(LIB_PATH)
        _declare(_lib)
    return _lib


_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)
_vp = C.c_void_p


def _declare(L):
    sig = {
        "xs_create": [C.POINTER(C.c_void_p)],
        "xs_destroy": [C.c_void_p],
        "xs_mat_setup": [C.c_void_p, C.c_int, _ip, _ip, _dp, C.c_int],
        "xs_mat_update": [C.c_void_p, _dp],
        "xs_set_refinement_mode": [C.c_void_p, C.c_int],
        "xs_ksp_settype": [C.c_void_p, C.c_char_p],
        "xs_ksp_setoption": [C.c_void_p, C.c_double, C.c_int, _ip, _dp, C.c_int],
        "xs_ksp_set_absolute_tol": [C.c_void_p, C.c_double],
        "xs_pc_settype": [C.c_void_p, C.c_char_p],
        "xs_pc_setilut": [C.c_void_p, C.c_double, C.c_int],
        "xs_pc_setict": [C.c_void_p, C.c_double, C.c_int],
        "xs_host_ilut": [C.c_int, _ip, _ip, _dp, C.c_int, C.c_double, _ip, _ip, _ip, _ip, _dp, _dp, _ip, _ip, _dp],
        "xs_host_ict": [C.c_int, _ip, _ip, _dp, C.c_int, C.c_double, _ip, _ip, _ip, _ip, _dp, _dp, _ip, _ip, _dp],
        "xs_pc_setparilu": [C.c_void_p, C.c_int],
        "xs_pc_setparilut": [C.c_void_p, C.c_double, C.c_int, C.c_double],
        "xs_pc_set_trsv": [C.c_void_p, C.c_int],
        "xs_set_precision": [C.c_void_p, C.c_char_p, C.c_char_p, C.c_char_p],
        "xs_set_inner": [C.c_void_p, C.c_double, C.c_int],
        "xs_set_compat": [C.c_void_p, C.c_int],
        "xs_solve": [C.c_void_p, _dp, _dp],
        "xs_solve_device": [C.c_void_p, _vp, _vp],
        "xs_solve_batch": [C.c_void_p, C.c_int, _dp, _dp],
        "xs_adjoint": [C.c_void_p, _dp, _dp, _dp],
        "xs_adjoint_batch": [C.c_void_p, C.c_int, _dp, _dp, _dp, _dp],
        "xs_last_timing": [C.c_void_p, _dp, _dp, _ip, _dp],
        "xs_last_outer_steps": [C.c_void_p, _ip],
        "xs_get_stream": [C.c_void_p, C.POINTER(C.c_void_p)],
        "xs_last_launches": [C.c_void_p, C.POINTER(C.c_longlong)],
        "xs_plan_create": [C.POINTER(C.c_void_p), C.c_int, _ip, _ip, _dp],
        "xs_plan_destroy": [C.c_void_p],
        "xs_plan_build_ell": [C.c_void_p, _ip],
        "xs_plan_spmv": [C.c_void_p, C.c_int, C.c_int, _vp, _vp],
        "xs_plan_spmv_t": [C.c_void_p, _vp, _vp],
        "xs_plan_factor": [C.c_void_p, C.c_int, C.c_int, C.c_double, C.c_double],
        "xs_plan_get_factors": [C.c_void_p, _ip, _ip, _ip, _ip, _dp, _dp, _ip, _ip, _dp],
        "xs_plan_get_lu_values": [C.c_void_p, _dp],
        "xs_plan_set_factor_precision": [C.c_void_p, C.c_int],
        "xs_plan_lusolve": [C.c_void_p, C.c_int, _vp, _vp],
        "xs_plan_set_trsv": [C.c_void_p, C.c_int],
        "xs_plan_lusolve_t": [C.c_void_p, _vp, _vp],
        "xs_plan_lusolve_batch": [C.c_void_p, C.c_int, _vp, _vp],
        "xs_plan_sync": [C.c_void_p],
        "xs_plan_get_stream": [C.c_void_p, C.POINTER(C.c_void_p)],
        "xs_plan_debug_break_dependency": [C.c_void_p, C.c_int, C.c_int],
        "xs_plan_levels": [C.c_void_p, _ip, _ip],
        "xs_plan_time_op": [C.c_void_p, C.c_int, C.c_int, C.c_int, _dp],
        "xs_plan_op_bytes": [C.c_void_p, C.c_int, _dp],
        "xs_device_count": [],
        "xs_tri_levels": [C.c_int, _ip, _ip, C.c_int, _ip, _ip, _ip],
        "xs_mm_info": [C.c_char_p, _ip, _ip, _ip, _ip],
        "xs_mm_read": [C.c_char_p, C.c_int, _ip, _ip, _dp, _dp],
        "xs_set_trsv_tuning": [C.c_int, C.c_int, C.c_int],
        "xs_set_trsv_tiles": [C.c_int, C.c_int, C.c_int, C.c_int, C.c_int],
        "xs_tri_tiles": [C.c_int, _ip, _ip, C.c_int, C.c_int, C.c_int, C.c_int, _ip, _ip, _ip, _ip, _ip, _ip, _ip,
                         _ip, _ip],
        "xs_set_ell_index_bits": [C.c_int],
        "xs_set_trsv_block_rows": [C.c_int],
        "xs_set_trsv_block_staging": [C.c_int],
        "xs_set_ilu_tiles": [C.c_int],
        "xs_set_sweep_fusion": [C.c_int],
        "xs_set_launch_overlap": [C.c_int],
        "xs_set_vector_fusion": [C.c_int],
        "xs_set_batch_kernels": [C.c_int],
        "xs_set_persistent_iteration": [C.c_int],
        "xs_batch_iterations": [C.c_void_p, C.c_int, _ip],
        "xs_lusolve_noalloc": [C.c_int, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp],
        "xsolver_last_error": [],
    }
    for name, args in sig.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = C.c_int
    L.xs_version.restype = C.c_char_p
    L.xsolver_error_string.restype = C.c_char_p
    L.xsolver_error_string.argtypes = [C.c_int]
    for name in ("xsolver_ksp_settype", "xsolver_pc_settype"):
        getattr(L, name).argtypes = [C.c_char_p]
        getattr(L, name).restype = None
    L.xsolver_mat_setup.argtypes = [C.c_int, _ip, _ip, _dp, _ip]
    L.xsolver_mat_setup.restype = None
    L.xsolver_ksp_setoption.argtypes = [C.c_double, C.c_int, _ip, _dp, C.c_int]
    L.xsolver_ksp_setoption.restype = None
    L.xsolver_ksp_set_absolute_tol.argtypes = [C.c_double]
    L.xsolver_ksp_set_absolute_tol.restype = None
    L.xsolver_pc_setilut.argtypes = [C.c_double, C.c_int]
    L.xsolver_pc_setilut.restype = None
    L.xsolver_pc_setict.argtypes = [C.c_double, C.c_int]
    L.xsolver_pc_setict.restype = None
    L.xsolver_solve.argtypes = [_dp, _dp]
    L.xsolver_solve.restype = None
    L.xsolver_free.argtypes = []
    L.xsolver_free.restype = None
    L.xsolver_set_precision.argtypes = [C.c_char_p, C.c_char_p, C.c_char_p]
    L.xsolver_set_precision.restype = None
    L.xsolver_set_inner.argtypes = [C.c_double, C.c_int]
    L.xsolver_set_inner.restype = None
    L.xsolver_pc_setparilu.argtypes = [C.c_int]
    L.xsolver_pc_setparilu.restype = None
    L.xsolver_pc_setparilut.argtypes = [C.c_double, C.c_int, C.c_double]
    L.xsolver_pc_setparilut.restype = None
    L.xsolver_pc_set_trsv.argtypes = [C.c_int]
    L.xsolver_pc_set_trsv.restype = None
    L.xsolver_set_compat.argtypes = [C.c_int]
    L.xsolver_set_compat.restype = None
    L.xsolver_adjoint.argtypes = [_dp, _dp, _dp]
    L.xsolver_adjoint.restype = None
    L.cpu_mat_setup.argtypes = [_ip, _ip, _ip, _dp, _dp, _ip, _ip]
    L.cpu_mat_setup.restype = None
    L.cpu_mat_update.argtypes = [_dp, _dp]
    L.cpu_mat_update.restype = None
    for name in ("gpu_mat_setup", "gpu_mat_update", "gpu_mat_free"):
        getattr(L, name).argtypes = []
        getattr(L, name).restype = None
    L.gpu_mat_format.argtypes = [C.c_char_p, _ip]
    L.gpu_mat_format.restype = None
    for name in ("gpu_preconditioner_setup", "gpu_preconditioner_update", "gpu_preconditioner_free"):
        getattr(L, name).argtypes = [C.c_char_p]
        getattr(L, name).restype = None
    for name in ("gpu_cg_solve", "gpu_cgm_solve", "gpu_icg_solve", "gpu_icgm_solve", "gpu_bicgstab_solve",
                 "gpu_ibicgstab_solve"):
        getattr(L, name).argtypes = [_dp, _dp, _dp, _ip, _dp, _ip, _dp]
        getattr(L, name).restype = None
    for name in ("gpu_gcr_solve", "gpu_igcr_solve", "gpu_gmres_solve", "gpu_fgmres_solve"):
        getattr(L, name).argtypes = [_dp, _dp, _ip, _dp, _ip, _dp, _ip, _dp]
        getattr(L, name).restype = None


def check(rc: int, what: str = "xsolver_b200"):
    if rc != 0:
        raise XsError(rc, what)


def last_error() -> int:
    return lib().xsolver_last_error()


def declared_symbols(header: str = HEADER):
    """Names of every function the public header declares."""
    text = open(header).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = set()
    for m in re.finditer(r"\b((?:xs|xsolver|gpu|cpu)_[A-Za-z0-9_]*)\s*\(", text):
        names.add(m.group(1))
    return sorted(names)
