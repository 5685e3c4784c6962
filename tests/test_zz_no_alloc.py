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


def _noalloc(L, n, d, x, z):
    return L.xs_lusolve_noalloc(n, _vp(d["lrp"]), _vp(d["lci"]), _vp(d["lv"]), _vp(d["dinv"]), _vp(d["urp"]),
                                _vp(d["uci"]), _vp(d["uv"]), _vp(x), _vp(z), None)


@pytest.mark.parametrize("grid", [24, 64])  # 64^3 = 262144 rows: the documented limit, the array full
def test_noalloc_lusolve_matches_plan_two_calls(cuda, grid):
    import torch
    from xsolver_b200 import _lib
    from xsolver_b200.api import Plan

    L = _lib.lib()
    A = st.poisson3d_7pt(grid)
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
        rc = _noalloc(L, A.n, d, x, z)
        assert rc == 0, rc
        assert torch.equal(z, z_ref), seed


def test_noalloc_wait_runs_out_then_recovers(cuda):
    """One L row names itself as a dependency: its value is never published,
    so its bounded wait runs out after about 1 s, every kernel returns, and
    the call reports XS_ERR_TRSV_TIMEOUT.  The next call, with the proper
    factor, succeeds and matches the plan solve bitwise."""
    import torch
    from xsolver_b200 import _lib
    from xsolver_b200.api import Plan

    L = _lib.lib()
    A = st.poisson3d_7pt(12)
    P = Plan(A).factor("ilu0")
    F = P.factors()
    d = {k: torch.from_numpy(np.ascontiguousarray(v)).to(cuda) for k, v in F.items()}
    lrp, lci = F["lrp"], F["lci"].copy()
    row = A.n // 2
    assert lrp[row + 1] > lrp[row]
    lci[lrp[row + 1] - 1] = row  # in range: the row waits on its own value
    bad = dict(d, lci=torch.from_numpy(lci).to(cuda))
    x = torch.from_numpy(st.rhs_uniform(A.n, 3)).to(cuda)
    z = torch.zeros(A.n, dtype=torch.float64, device=cuda)
    torch.cuda.synchronize()
    assert _noalloc(L, A.n, bad, x, z) == 5  # XS_ERR_TRSV_TIMEOUT
    z_ref = torch.zeros(A.n, dtype=torch.float64, device=cuda)
    P.lusolve(x, z_ref)
    P.sync()
    assert _noalloc(L, A.n, d, x, z) == 0
    assert torch.equal(z, z_ref)


def test_noalloc_rejects_null_factor_arrays(cuda):
    import torch
    from xsolver_b200 import _lib

    L = _lib.lib()
    buf = torch.zeros(64, dtype=torch.float64, device=cuda)
    ok = _vp(buf)
    for k in range(8):  # lci, lv, uci, uv (and the others) may not be NULL when n > 0
        args = [ok] * 9
        args[k] = None
        assert L.xs_lusolve_noalloc(8, *args, None) == 1, k  # XS_ERR_INVALID


def test_noalloc_rejects_oversize(cuda):
    from xsolver_b200 import _lib

    L = _lib.lib()
    rc = L.xs_lusolve_noalloc(262145, None, None, None, None, None, None, None, None, None, None)
    assert rc in (1, 11)  # invalid pointers or capacity: refused before any GPU work
    dummy = C.c_void_p(16)
    rc = L.xs_lusolve_noalloc(262145, dummy, dummy, dummy, dummy, dummy, dummy, dummy, dummy, dummy, None)
    assert rc == 11  # XS_ERR_CAPACITY
