"""xs_lusolve_noalloc: the LU solve for callers that cannot allocate device
memory (allocator-owned pools, fixed budgets after start-up, caller-owned
buffers only).  Its scratch is a fixed __device__ array inside the library.

Checked through the C ABI against the plan-based sync-free solve
(xs_plan_lusolve) on the same factors, on two calls in a row: FP64 results
must be identical (the tolerance the FP64 LU-solve tests use is bitwise).
This file is named to be collected last."""
import ctypes as C

import numpy as np
import pytest

from xsolver_b200 import stencils as st

pytestmark = pytest.mark.gpu


def _vp(t):
    return C.c_void_p(t.data_ptr())


def test_noalloc_lusolve_matches_plan_two_calls(cuda):
    import torch
    from xsolver_b200 import _lib
    from xsolver_b200.api import Plan

    L = _lib.lib()
    A = st.poisson3d_7pt(24)
    P = Plan(A).factor("ilu0")
    F = P.factors()
    d = {k: torch.from_numpy(np.ascontiguousarray(v)).to(cuda) for k, v in F.items()}
    for seed in (1, 2):  # two calls in a row: the shared scratch is re-armed per call
        x = torch.from_numpy(st.rhs_uniform(A.n, seed)).to(cuda)
        z_ref = torch.zeros(A.n, dtype=torch.float64, device=cuda)
        P.lusolve(x, z_ref)
        P.sync()
        z = torch.full((A.n,), -7.0, dtype=torch.float64, device=cuda)
        torch.cuda.synchronize()
        rc = L.xs_lusolve_noalloc(A.n, _vp(d["lrp"]), _vp(d["lci"]), _vp(d["lv"]), _vp(d["dinv"]), _vp(d["urp"]),
                                  _vp(d["uci"]), _vp(d["uv"]), _vp(x), _vp(z), None)
        assert rc == 0, rc
        assert torch.equal(z, z_ref), seed


def test_noalloc_rejects_oversize(cuda):
    from xsolver_b200 import _lib

    L = _lib.lib()
    rc = L.xs_lusolve_noalloc(262145, None, None, None, None, None, None, None, None, None, None)
    assert rc in (1, 11)  # invalid pointers or capacity: refused before any GPU work
    dummy = C.c_void_p(16)
    rc = L.xs_lusolve_noalloc(262145, dummy, dummy, dummy, dummy, dummy, dummy, dummy, dummy, dummy, None)
    assert rc == 11  # XS_ERR_CAPACITY
