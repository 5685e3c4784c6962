"""Box-scheduled exact triangular solves on the GPU.

The box schedule (xs_tri_tiles) replaces the row-per-thread dependency flags
of the reference's sync-free solves (hip/Precond/gpuparilu.cpp:257-364) on
grid-shaped patterns.  It changes only which CTA computes a row and where a
dependency is read from (shared memory instead of a polled global value);
each row's entries are summed in the same order with the same operations,
so results must be bitwise identical to the oracle's LUsolve
(hip/HostMatrix/HostMatrixCSR.cpp:385-409) in FP64 and to the level-ordered
solve in every precision."""
import numpy as np
import pytest

import oracle
from xsolver_b200 import stencils as st

pytestmark = pytest.mark.gpu


def _dev(a, cuda):
    import torch

    return torch.from_numpy(np.ascontiguousarray(a)).to(cuda)


class tiles_forced:
    """Box-scheduled solves for every triangle of at least `min_rows` rows
    (plans built inside the block), restored to the defaults afterwards."""

    def __init__(self, box=(16, 16, 16), min_rows=8, enable=1):
        self.args = (enable, *box, min_rows)

    def __enter__(self):
        from xsolver_b200 import _lib

        L = _lib.lib()
        assert L.xs_set_trsv_tiles(*self.args) == 0
        assert L.xs_set_trsv_block_rows(0) == 0  # no single-CTA solve: the multi-CTA path runs
        return self

    def __exit__(self, *exc):
        from xsolver_b200 import _lib

        L = _lib.lib()
        L.xs_set_trsv_tiles(1, 16, 16, 8, 65536)
        L.xs_set_trsv_block_rows(1 << 30)


def _solve64(P, x, cuda, reps=1):
    import torch

    z = torch.zeros(len(x), dtype=torch.float64, device=cuda)
    dx = _dev(x, cuda)
    out = []
    for _ in range(reps):
        P.lusolve(dx, z)
        P.sync()
        out.append(z.cpu().numpy().copy())
    return out


@pytest.mark.parametrize("box", [(16, 16, 16), (8, 8, 8), (4, 8, 16)])
def test_tiled_lusolve_fp64_bitwise_vs_oracle(cuda, box):
    from xsolver_b200.api import Plan

    with tiles_forced(box):
        for A in (st.poisson3d_7pt(40), st.convdiff3d_27pt(22), st.varcoef3d_7pt(30, 2)):
            P = Plan(A).factor("ilu0")
            F = oracle.ilu0(A)
            x = st.rhs_uniform(A.n, 7)
            ref = oracle.lusolve(F, x)
            for rep, z in enumerate(_solve64(P, x, cuda, reps=3)):  # buffers re-armed between solves
                assert np.array_equal(z, ref), (A.name, box, rep)


def test_tiled_parilut_fill_bitwise_vs_oracle(cuda):
    """ParILUT factors reach several grid steps (a sheared box grid)."""
    from xsolver_b200.api import Plan

    A = st.convdiff3d_27pt(24)
    F = oracle.parilut(A, fill=2.0, sweeps=5, droptol=1e-4)
    x = st.rhs_uniform(A.n, 5)
    with tiles_forced():
        P = Plan(A).factor("parilut", sweeps=5, fill=2.0, droptol=1e-4)
        (z,) = _solve64(P, x, cuda)
    assert np.array_equal(z, oracle.lusolve(F, x))


@pytest.mark.parametrize("prec", ["fp32", "bf16", "fp16"])
def test_tiled_equals_level_ordered_reduced_precision(cuda, prec):
    import torch
    from xsolver_b200.api import Plan

    A = st.convdiff3d_27pt(22)
    x = st.rhs_uniform(A.n, 9).astype(np.float32)
    outs = []
    for enable in (1, 0):
        with tiles_forced(enable=enable):
            P = Plan(A).factor("ilu0").set_factor_precision(prec)
            z = torch.zeros(A.n, dtype=torch.float32, device=cuda)
            dx = _dev(x, cuda)
            P.lusolve(dx, z)
            P.sync()
            outs.append(z.cpu().numpy())
    assert np.array_equal(outs[0], outs[1])


def test_tiled_wait_times_out_and_recovers(cuda):
    """A halo value nothing publishes before the wait (one of the box's own
    rows): the bounded wait gives up after about 1 s, the error is
    reported, and the plan works again once the halo entry is restored."""
    from xsolver_b200.api import Plan, XsError

    A = st.poisson3d_7pt(24)
    F = oracle.ilu0(A)
    x = st.rhs_uniform(A.n, 1)
    with tiles_forced((8, 8, 8)):
        P = Plan(A).factor("ilu0")
        P.debug_break_dependency(A.n - 1, True)
        with pytest.raises(XsError) as e:
            _solve64(P, x, cuda)
        assert e.value.code == 5  # XS_ERR_TRSV_TIMEOUT
        P.debug_break_dependency(A.n - 1, False)
        (z,) = _solve64(P, x, cuda)
    assert np.array_equal(z, oracle.lusolve(F, x))


def test_solver_with_tiles_matches_level_ordered(cuda):
    """A whole FP64 BiCGSTAB + ILU(0) solve: identical iterates either way."""
    from xsolver_b200.api import Solver

    A = st.poisson3d_7pt(36)
    b = st.rhs_uniform(A.n, 4)
    res = []
    for enable in (1, 0):
        with tiles_forced(enable=enable):
            S = Solver(A).ksp_settype("bicgstab").ksp_setoption(1e-10, 500).pc_settype("ilu0")
            x = S.solve(b)
            res.append((x, S.resvec()))
            S.close()
    assert np.array_equal(res[0][0], res[1][0]) and np.array_equal(res[0][1], res[1][1])
