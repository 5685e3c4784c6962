"""Row-block decomposition (xsolver_b200.distributed) on CPU ranks (gloo):
halo plans, the point-to-point halo exchange, BiCGSTAB with reduced dot
products and block-Jacobi ILU(0), against the oracle's serial BiCGSTAB with
ILU(0) factors of the block-diagonal part of A; and a rank that fails on the
host making its peers' next exchange end with an error instead of hanging.
The local work runs in CpuBackend below (test infrastructure: the same
operations as the library's DeviceBackend, on the host)."""
import datetime
import os
import socket
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


class CpuBackend:
    def __init__(self, plan, val):
        import scipy.sparse as sp

        import oracle
        from xsolver_b200.stencils import CSRMatrix

        n, nh = plan.n_local, plan.n_halo
        self.A = sp.csr_matrix((val, plan.colidx_aug, plan.rowptr), shape=(n, n + nh))
        rows = np.repeat(np.arange(n), np.diff(plan.rowptr))
        own = plan.colidx_aug < n
        brp = np.zeros(n + 1, np.int32)
        np.cumsum(np.bincount(rows[own], minlength=n), out=brp[1:])
        self.F = oracle.ilu0(CSRMatrix(n, brp, plan.colidx_aug[own].astype(np.int32), val[own], "block"))
        self._lus = oracle.lusolve

    def spmv(self, x_aug):
        import torch

        return torch.from_numpy(self.A @ x_aug.numpy())

    def precond(self, r):
        import torch

        return torch.from_numpy(self._lus(self.F, r.numpy()))


def _problem(name):
    from xsolver_b200 import stencils as st

    A = {"p3": st.poisson3d_7pt(10), "c3": st.convdiff3d_27pt(9, pe=5.0)}[name]
    return A, st.rhs_uniform(A.n, 3)


def _worker(rank, ws, port, q, name, fail_rank, pc="block", method="bicgstab"):
    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    from xsolver_b200 import distributed as dd

    dist.init_process_group("gloo", rank=rank, world_size=ws, timeout=datetime.timedelta(seconds=10))
    try:
        A, b = _problem(name)
        bounds = dd.row_bounds(A.n, ws)
        rp, ci, v = dd.local_rows(A, bounds, rank)
        plan = dd.HaloPlan(rp, ci, bounds, rank, "cpu")
        be = CpuBackend(plan, v)
        if rank == fail_rank:
            raise RuntimeError("injected failure before the first exchange")
        M = dd.JacobiPC(plan, v, "cpu") if pc == "jacobi" else None
        bl = b[bounds[rank]:bounds[rank + 1]]
        if method == "gmres":
            x, rv, used = dd.gmres(be, plan, bl, tol=1e-10, maxiter=500, restart=20, pc=M)
        else:
            solve = dd.pcg if method == "cgm" else dd.bicgstab
            x, rv, used = solve(be, plan, bl, tol=1e-10, maxiter=500, pc=M)
        q.put((rank, "ok", x.numpy(), rv, used, plan.n_halo, [p for p, _, _ in plan.recv]))
    except Exception as e:  # reported to the test, then the rank leaves
        q.put((rank, "error", repr(e), None, None, None, None))
    finally:
        try:
            dist.destroy_process_group()
        except Exception:
            pass


def _run(ws, name, fail_rank=-1, wait=120, pc="block", method="bicgstab"):
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, ws, port, q, name, fail_rank, pc, method)) for r in range(ws)]
    for p in procs:
        p.start()
    out = sorted([q.get(timeout=wait) for _ in range(ws)], key=lambda t: t[0])
    for p in procs:
        p.join(timeout=60)
    return out


@pytest.mark.parametrize("ws,name", [(2, "p3"), (3, "c3")])
def test_block_jacobi_bicgstab_matches_serial_oracle(ws, name):
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle
    from parity import count_ok, history_ok, iteration_range, reference_with_bounds
    from xsolver_b200 import distributed as dd
    from xsolver_b200.stencils import CSRMatrix

    out = _run(ws, name)
    assert all(o[1] == "ok" for o in out), [o[2] for o in out if o[1] != "ok"]
    A, b = _problem(name)
    bounds = dd.row_bounds(A.n, ws)
    # halo neighbours: the adjacent blocks
    for r, o in enumerate(out):
        assert o[6] == [q for q in (r - 1, r + 1) if 0 <= q < ws], (r, o[6])
        assert o[5] > 0
    x = np.concatenate([o[2] for o in out])
    rv, used = out[0][3], out[0][4]
    assert all(o[4] == used for o in out) and all(np.array_equal(o[3], rv) for o in out)
    # serial reference: BiCGSTAB with ILU(0) of A's block-diagonal part
    rows = np.repeat(np.arange(A.n), np.diff(A.rowptr))
    blk = np.searchsorted(bounds, rows, side="right") == np.searchsorted(bounds, A.colidx, side="right")
    rp = np.zeros(A.n + 1, np.int32)
    np.cumsum(np.bincount(rows[blk], minlength=A.n), out=rp[1:])
    F = oracle.ilu0(CSRMatrix(A.n, rp, A.colidx[blk].astype(np.int32), A.val[blk], "blockdiag"))
    kw = dict(tol=1e-10, maxiter=500, pc="lu", factors=F)
    xo, ho, uo, hb, xb = reference_with_bounds("bicgstab", A, b, **kw)
    assert count_ok(used, uo, iteration_range("bicgstab", A, b, **kw)), (used, uo)
    ok, worst = history_ok(rv, ho, hb)
    assert ok, worst
    assert np.linalg.norm(x - xo) / np.linalg.norm(xo) < xb
    assert np.linalg.norm(b - A.to_scipy() @ x) / np.linalg.norm(b) < 1e-9


@pytest.mark.parametrize("ws,method,name", [(2, "bicgstab", "c3"), (3, "bicgstab", "c3"), (2, "cgm", "p3"),
                                            (3, "cgm", "p3"), (2, "gmres", "c3"), (3, "gmres", "p3")])
def test_jacobi_solvers_match_compiled_reference(ws, method, name):
    """The reference MPI driver's method (hip/mpi_solve_base.h: BiCGSTAB +
    Jacobi), PCG ("cgm") and GMRES(20) with Jacobi on ws CPU ranks against
    the reference's own compiled cpu_*_solve on the whole system (bounds
    from the restatement, which equals it bitwise)."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle
    from parity import count_ok, history_ok, iteration_range, reference_with_bounds

    if oracle.ref_intel() is None:
        pytest.skip("compiled reference not present")
    out = _run(ws, name, pc="jacobi", method=method)
    assert all(o[1] == "ok" for o in out), [o[2] for o in out if o[1] != "ok"]
    A, b = _problem(name)
    x = np.concatenate([o[2] for o in out])
    rv, used = out[0][3], out[0][4]
    xr, rr, ur = oracle.ref_solve(method, A, b, tol=1e-10, maxiter=500, restart=20)
    kw = dict(tol=1e-10, maxiter=500, restart=20, pc="jacobi")
    xo, ho, uo, hb, xb = reference_with_bounds(method, A, b, **kw)
    assert uo == ur and np.array_equal(xo, xr)
    assert count_ok(used, ur, iteration_range(method, A, b, **kw)), (used, ur)
    # the restatement's history is indexed by the global iteration (the
    # reference overwrites GMRES entries per restart cycle)
    ok, worst = history_ok(rv, ho, hb)
    assert ok, worst
    assert np.linalg.norm(x - xr) / np.linalg.norm(xr) < xb


def test_failed_rank_ends_the_peers_exchange():
    """Rank 1 fails on the host after setup; rank 0's first halo exchange
    must end with an error within the process-group timeout, not hang."""
    out = _run(2, "p3", fail_rank=1, wait=90)
    assert out[1][1] == "error" and "injected" in out[1][2]
    assert out[0][1] == "error", out[0]


class _Slice:
    """The renumbered rows of one rank as HaloPlan computes them, built
    here without a process group (only the fields the backend reads)."""

    def __init__(self, A, bounds, rank):
        from xsolver_b200 import distributed as dd

        r0, r1 = bounds[rank], bounds[rank + 1]
        self.rowptr, ci, self.val = dd.local_rows(A, bounds, rank)
        cols = ci.astype(np.int64)
        out = (cols < r0) | (cols >= r1)
        halo = np.unique(cols[out])
        self.n_local, self.n_halo = r1 - r0, len(halo)
        aug = np.empty(len(cols), np.int64)
        aug[~out] = cols[~out] - r0
        aug[out] = self.n_local + np.searchsorted(halo, cols[out])
        self.colidx_aug = aug.astype(np.int32)
        self.halo = halo


@pytest.mark.gpu
def test_device_backend_local_operator(cuda):
    """DeviceBackend on rank 0's rows of a 2-way split: the SpMV of the
    augmented rows (owned + halo columns) equals the host product, and the
    block-Jacobi apply equals the oracle's LU solve with ILU(0) of the owned
    block."""
    import torch

    import oracle
    from xsolver_b200 import distributed as dd
    from xsolver_b200.stencils import CSRMatrix

    A, _ = _problem("c3")
    bounds = dd.row_bounds(A.n, 2)
    s = _Slice(A, bounds, 0)
    be = dd.DeviceBackend(s, s.val, cuda)
    rng = np.random.default_rng(1)
    x_aug = rng.uniform(-1, 1, s.n_local + s.n_halo)
    y = be.spmv(torch.from_numpy(x_aug).to(cuda)).cpu().numpy()
    import scipy.sparse as sp

    ref = sp.csr_matrix((s.val, s.colidx_aug, s.rowptr), shape=(s.n_local, s.n_local + s.n_halo)) @ x_aug
    assert np.allclose(y, ref, rtol=1e-13, atol=1e-13)
    cpu = CpuBackend(s, s.val)
    r = rng.uniform(-1, 1, s.n_local)
    z = be.precond(torch.from_numpy(r).to(cuda)).cpu().numpy()
    assert np.array_equal(z, oracle.lusolve(cpu.F, r))


@pytest.mark.gpu
def test_device_backend_single_rank_solve(cuda):
    """World size 1 over NCCL: the distributed BiCGSTAB with DeviceBackend
    equals the serial oracle (ILU(0) of the whole matrix) within the
    calibrated bounds."""
    import torch.distributed as dist

    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle
    from parity import count_ok, history_ok, iteration_range, reference_with_bounds
    from xsolver_b200 import distributed as dd

    A, b = _problem("p3")
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{_free_port()}", rank=0, world_size=1,
                            timeout=datetime.timedelta(seconds=30))
    try:
        bounds = dd.row_bounds(A.n, 1)
        rp, ci, v = dd.local_rows(A, bounds, 0)
        plan = dd.HaloPlan(rp, ci, bounds, 0, cuda)
        be = dd.DeviceBackend(plan, v, cuda)
        x, rv, used = dd.bicgstab(be, plan, b, tol=1e-10, maxiter=500)
        x = x.cpu().numpy()
    finally:
        dist.destroy_process_group()
    kw = dict(tol=1e-10, maxiter=500, pc="lu", factors=oracle.ilu0(A))
    xo, ho, uo, hb, xb = reference_with_bounds("bicgstab", A, b, **kw)
    assert count_ok(used, uo, iteration_range("bicgstab", A, b, **kw)), (used, uo)
    ok, worst = history_ok(rv, ho, hb)
    assert ok, worst
    assert np.linalg.norm(x - xo) / np.linalg.norm(xo) < xb


@pytest.mark.gpu
def test_device_pcg_jacobi_single_rank(cuda):
    """World size 1 over NCCL: the decomposition's PCG with the reference's
    Jacobi on the GPU (DeviceBackend SpMV, JacobiPC on the device) against
    the serial oracle (bitwise equal to the compiled reference)."""
    import torch.distributed as dist

    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from parity import count_ok, history_ok, iteration_range, reference_with_bounds
    from xsolver_b200 import distributed as dd

    A, b = _problem("p3")
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{_free_port()}", rank=0, world_size=1,
                            timeout=datetime.timedelta(seconds=30))
    try:
        bounds = dd.row_bounds(A.n, 1)
        rp, ci, v = dd.local_rows(A, bounds, 0)
        plan = dd.HaloPlan(rp, ci, bounds, 0, cuda)
        be = dd.DeviceBackend(plan, v, cuda)
        x, rv, used = dd.pcg(be, plan, b, tol=1e-10, maxiter=500, pc=dd.JacobiPC(plan, v, cuda))
        x = x.cpu().numpy()
    finally:
        dist.destroy_process_group()
    kw = dict(tol=1e-10, maxiter=500, pc="jacobi")
    xo, ho, uo, hb, xb = reference_with_bounds("cgm", A, b, **kw)
    assert count_ok(used, uo, iteration_range("cgm", A, b, **kw)), (used, uo)
    ok, worst = history_ok(rv, ho, hb)
    assert ok, worst
    assert np.linalg.norm(x - xo) / np.linalg.norm(xo) < xb


def _exchange_worker(rank, ws, port, q):
    """One-directional coupling: rank 0 only sends, the last rank only
    receives, the middle rank does both; each rank checks its halo values and
    its rows of A x against the global product."""
    import torch
    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    from xsolver_b200 import distributed as dd
    from xsolver_b200.stencils import CSRMatrix

    dist.init_process_group("gloo", rank=rank, world_size=ws, timeout=datetime.timedelta(seconds=10))
    try:
        n = 12
        rows, cols, vals = [], [], []
        for i in range(n):
            entries = {i: 2.0}
            if i > 0:
                entries[i - 1] = -1.0  # reads the previous row (from the rank below at a block edge)
            if i == n - 1:
                entries[0] = 0.5  # the last rank also reads from rank 0
            for c in sorted(entries):
                rows.append(i), cols.append(c), vals.append(entries[c])
        rp = np.zeros(n + 1, np.int32)
        np.cumsum(np.bincount(rows, minlength=n), out=rp[1:])
        A = CSRMatrix(n, rp, np.array(cols, np.int32), np.array(vals), "bidiagonal+corner")
        bounds = dd.row_bounds(n, ws)
        lrp, lci, lv = dd.local_rows(A, bounds, rank)
        plan = dd.HaloPlan(lrp, lci, bounds, rank, "cpu")
        xg = 1.5 * np.arange(n) + 1.0
        aug = torch.zeros(plan.n_local + plan.n_halo, dtype=torch.float64)
        aug[: plan.n_local] = torch.from_numpy(xg[bounds[rank]:bounds[rank + 1]])
        plan.exchange(aug)
        halo_cols = np.unique(lci[(lci < bounds[rank]) | (lci >= bounds[rank + 1])])
        ok_halo = np.array_equal(aug[plan.n_local:].numpy(), xg[halo_cols])
        import scipy.sparse as sp

        Aloc = sp.csr_matrix((lv, plan.colidx_aug, plan.rowptr), shape=(plan.n_local, plan.n_local + plan.n_halo))
        y = Aloc @ aug.numpy()
        ok_y = np.array_equal(y, (A.to_scipy() @ xg)[bounds[rank]:bounds[rank + 1]])
        q.put((rank, "ok", ok_halo, ok_y, len(plan.send), len(plan.recv)))
    except Exception as e:
        q.put((rank, "error", repr(e), None, None, None))
    finally:
        try:
            dist.destroy_process_group()
        except Exception:
            pass


def test_one_directional_halo_exchange():
    import torch.multiprocessing as mp

    ws = 3
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_exchange_worker, args=(r, ws, port, q)) for r in range(ws)]
    for p in procs:
        p.start()
    out = sorted([q.get(timeout=120) for _ in range(ws)], key=lambda t: t[0])
    for p in procs:
        p.join(timeout=60)
    for rank, status, ok_halo, ok_y, nsend, nrecv in out:
        assert status == "ok", (rank, ok_halo)
        assert ok_halo and ok_y, rank
    # rank 0 sends to ranks 1 and 2 and receives nothing; rank 2 only receives
    assert (out[0][4], out[0][5]) == (2, 0)
    assert (out[1][4], out[1][5]) == (1, 1)
    assert (out[2][4], out[2][5]) == (0, 2)


@pytest.mark.parametrize("method,name", [("bicgstab", "c3"), ("cgm", "p3")])
def test_result_does_not_depend_on_the_check_interval(method, name):
    """The decomposition solvers keep their scalars on the device and read
    the convergence flag on the host only every check_every iterations;
    iterations after convergence must leave the solution, the history and
    the count as they were.  So every interval gives the same bits, down to
    an interval longer than the iteration limit (which runs the loop to
    maxiter on frozen state)."""
    import torch.distributed as dist

    from xsolver_b200 import distributed as dd

    A, b = _problem(name)
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{_free_port()}", rank=0, world_size=1,
                            timeout=datetime.timedelta(seconds=30))
    try:
        bounds = dd.row_bounds(A.n, 1)
        rp, ci, v = dd.local_rows(A, bounds, 0)
        plan = dd.HaloPlan(rp, ci, bounds, 0, "cpu")
        be = CpuBackend(plan, v)
        solve = dd.pcg if method == "cgm" else dd.bicgstab
        runs = [solve(be, plan, b, tol=1e-10, maxiter=300, check_every=k) for k in (1, 4, 16, 1000)]
    finally:
        dist.destroy_process_group()
    x0, rv0, used0 = runs[0]
    assert used0 < 299 and rv0[-1] < 1e-10
    for x, rv, used in runs[1:]:
        assert used == used0
        assert np.array_equal(rv, rv0)
        assert np.array_equal(x.numpy(), x0.numpy())
