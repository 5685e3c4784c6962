"""Row-block domain decomposition of the Krylov solve over torch.distributed
(NCCL between GPUs, gloo between CPU ranks), replacing the reference's MPI
path: the halo exchange and reductions of intel/mpicpu.cpp:17-120
(communicator_init / communicator_p2p / communicator_p2p_waitall /
communicator_sum), the distributed setup hip/xsolver_c.cpp:294-306 and the
MPI driver hip/main_solve_mpi.cpp.

Rank r owns rows [bounds[r], bounds[r+1]) of A (contiguous blocks).  Its
local operator has the owned rows with columns renumbered into an augmented
vector [owned values (n_local) | halo values (n_halo)]: owned columns first,
then the columns owned by other ranks, grouped by owner and ascending (the
reference's interior-then-ghost layout).  Entries keep their order within a
row.  Before each SpMV the halo is exchanged point to point: every rank sends
each neighbour the owned values that neighbour reads and receives the halo
values it reads itself, as the reference's communicator_p2p does; the
exchange lists are built once, at setup, from the row patterns.

The solvers are the reference's BiCGSTAB (intel/mpisolver-C-v1.cpp:365-482,
right preconditioned, solution M^-1 phi), PCG ("cgm", :193-272) and
left-preconditioned GMRES(m) (:933-1087, modified Gram-Schmidt, Givens
rotations on the host), with every dot product a local dot
summed over the ranks (communicator_sum), preconditioned either by block
Jacobi (the local operator's own preconditioner on the owned diagonal
block: ILU(0) of that block on the GPU) or by the reference MPI driver's
pointwise Jacobi (JacobiPC, intel/HostMatrix.h:127-147).  The local work goes through a backend object
with spmv(x_aug) -> y and precond(r) -> z on the rank's device;
DeviceBackend uses this library's CUDA kernels.
"""
import contextlib

import numpy as np
import torch
import torch.distributed as dist

from .stencils import CSRMatrix


def row_bounds(n, world):
    """Contiguous row blocks of near-equal size: bounds[r]..bounds[r+1]."""
    return [n * r // world for r in range(world + 1)]


class HaloPlan:
    """Renumbered local rows and the exchange lists of one rank.  Built
    collectively (every rank calls it once, with its own rows)."""

    def __init__(self, rowptr, colidx, bounds, rank, device):
        world = len(bounds) - 1
        r0, r1 = bounds[rank], bounds[rank + 1]
        self.rank, self.world, self.r0, self.r1 = rank, world, r0, r1
        self.n_local = r1 - r0
        cols = np.asarray(colidx, dtype=np.int64)
        outside = (cols < r0) | (cols >= r1)
        halo = np.unique(cols[outside])  # ascending, so grouped by owner
        owners = np.searchsorted(np.asarray(bounds), halo, side="right") - 1
        self.n_halo = len(halo)
        aug = np.empty(len(cols), np.int64)
        aug[~outside] = cols[~outside] - r0
        aug[outside] = self.n_local + np.searchsorted(halo, cols[outside])
        self.rowptr = np.asarray(rowptr, np.int32)
        self.colidx_aug = aug.astype(np.int32)
        # what this rank reads from each owner, in its halo order
        self.recv = []  # (peer, offset into the halo, count)
        requests = {}
        for q in range(world):
            sel = np.flatnonzero(owners == q)
            if len(sel):
                self.recv.append((q, int(sel[0]), len(sel)))
                requests[q] = halo[sel]
        # every rank learns which of its rows each neighbour reads
        allreq = [None] * world
        dist.all_gather_object(allreq, {q: v.tolist() for q, v in requests.items()})
        self.send = []  # (peer, owned positions to send, in the peer's order)
        for p in range(world):
            rows = allreq[p].get(rank)
            if p != rank and rows:
                self.send.append((p, torch.as_tensor(np.asarray(rows, np.int64) - r0, device=device)))
        self.device = device

    def exchange(self, x_aug):
        """Fill x_aug[n_local:] with the neighbours' values (x_aug[:n_local]
        holds this rank's)."""
        if self.world == 1 or (not self.send and not self.recv):
            return x_aug
        bufs = [x_aug.index_select(0, idx).contiguous() for _, idx in self.send]
        # One batch: NCCL runs the point-to-point calls between a pair of
        # ranks on one stream, so a receive posted alone would block the
        # send behind it while the peer's receive waits for that send.
        ops = [dist.P2POp(dist.irecv, x_aug[self.n_local + off:self.n_local + off + cnt], q)
               for q, off, cnt in self.recv]
        ops += [dist.P2POp(dist.isend, buf, p) for (p, _), buf in zip(self.send, bufs)]
        for r in dist.batch_isend_irecv(ops):
            r.wait()
        return x_aug


def local_rows(A: CSRMatrix, bounds, rank):
    """Rows bounds[rank]..bounds[rank+1] of a global CSR (global columns)."""
    r0, r1 = bounds[rank], bounds[rank + 1]
    a, b = int(A.rowptr[r0]), int(A.rowptr[r1])
    rp = (A.rowptr[r0:r1 + 1] - a).astype(np.int32)
    return rp, A.colidx[a:b].astype(np.int32), A.val[a:b].astype(np.float64)


class DeviceBackend:
    """The rank's local operator on its GPU through this library: the SpMV
    of the augmented rows (embedded in a square matrix whose extra rows are
    the identity) and block-Jacobi ILU(0) of the owned diagonal block."""

    def __init__(self, plan: HaloPlan, val, device):
        from .api import Plan

        n, nh = plan.n_local, plan.n_halo
        rp, ci = plan.rowptr, plan.colidx_aug
        # square (n + nh) operator: the owned rows, then unit rows for the halo
        sq_rp = np.concatenate([rp, rp[-1] + 1 + np.arange(nh, dtype=np.int32)]).astype(np.int32)
        sq_ci = np.concatenate([ci, n + np.arange(nh, dtype=np.int32)]).astype(np.int32)
        sq_v = np.concatenate([val, np.ones(nh)])
        self.P_aug = Plan(CSRMatrix(n + nh, sq_rp, sq_ci, sq_v, "local+halo"))
        # owned diagonal block
        rows = np.repeat(np.arange(n), np.diff(rp))
        own = ci < n
        brp = np.zeros(n + 1, np.int32)
        np.cumsum(np.bincount(rows[own], minlength=n), out=brp[1:])
        self.P_blk = Plan(CSRMatrix(n, brp, ci[own].astype(np.int32), np.asarray(val)[own], "block")).factor("ilu0")
        self.n, self.nh, self.device = n, nh, device
        self._y = torch.zeros(n + nh, dtype=torch.float64, device=device)
        self.stream = self.P_aug.stream()
        self.s_blk = self.P_blk.stream()

    # The solvers run their torch work on self.stream (the SpMV plan's
    # stream); a call made from any other stream, and every block solve (its
    # plan has a stream of its own), is ordered against the caller's stream
    # with events in both directions: no host synchronisation per call.  The
    # plans keep the tensors of their queued work referenced until their
    # sync(), so no record_stream is used: that would make torch's allocator
    # record events on a plan's stream when the tensor is freed, which can be
    # after the plan has destroyed that stream.  checkpoint() is the solvers'
    # periodic host sync; it also releases those references.
    @staticmethod
    def _ordered(plan_stream, launch):
        cur = torch.cuda.current_stream()
        if cur == plan_stream:
            return launch()
        ev = torch.cuda.Event()
        ev.record(cur)
        plan_stream.wait_event(ev)
        out = launch()
        done = torch.cuda.Event()
        done.record(plan_stream)
        cur.wait_event(done)
        return out

    def spmv(self, x_aug):
        self._ordered(self.stream, lambda: self.P_aug.spmv(x_aug, self._y))
        return self._y[: self.n].clone()

    def precond(self, r):
        r = r.contiguous()
        z = torch.empty_like(r)
        self._ordered(self.s_blk, lambda: self.P_blk.lusolve(r, z))
        return z

    def checkpoint(self):
        self.P_aug.sync()
        self.P_blk.sync()


class JacobiPC:
    """The reference's Jacobi preconditioner on the owned rows
    (intel/HostMatrix.h:127-147): dinv_i = 1 / (a_ii + 1e-20), z = dinv * r,
    on the rank's device (a row without a diagonal entry has a_ii = 0)."""

    def __init__(self, plan: HaloPlan, val, device):
        n = plan.n_local
        rows = np.repeat(np.arange(n), np.diff(plan.rowptr))
        diag = np.zeros(n)
        on = plan.colidx_aug == rows
        diag[rows[on]] = np.asarray(val)[on]
        self.dinv = torch.as_tensor(1.0 / (diag + 1e-20), dtype=torch.float64, device=device)

    def precond(self, r):
        return self.dinv * r


def _gdot(a, b):
    t = torch.dot(a, b).reshape(1)
    dist.all_reduce(t)
    return float(t.item())


def _reduce(*dots):
    """The local dot products summed over the ranks, in one reduction of a
    device vector (NCCL orders it on the current stream: no host wait)."""
    t = torch.stack(list(dots))
    dist.all_reduce(t)
    return t


def _on_stream(backend):
    s = getattr(backend, "stream", None)
    return torch.cuda.stream(s) if s is not None else contextlib.nullcontext()


def _checkpoint(backend):
    f = getattr(backend, "checkpoint", None)
    if f is not None:
        f()


def bicgstab(backend, plan: HaloPlan, b_local, x0_local=None, tol=1e-8, maxiter=1000, pc=None, check_every=16):
    """The reference's BiCGSTAB (intel/mpisolver-C-v1.cpp:365-482) on the
    rank's rows; every rank calls it with its own pieces.  pc: an object
    with precond(r) (e.g. JacobiPC); default the backend's block Jacobi.
    Returns (x_local, resvec, usediter) in the reference's convention
    (resvec[k] = ||r_k|| / ||r_0||, usediter = index of the last
    iteration).

    The scalars stay on the device and each iteration takes three
    reductions ((u, r^), ((v, s), (v, v)), ((r, r), (r, r^)): the next
    iteration's beta comes with this one's residual norm).  The host reads
    the convergence flag every check_every iterations; an iteration after
    convergence leaves the solution and the history as they were, so the
    result is that of stopping at once.  The arithmetic is the reference
    loop's, operation by operation."""
    M = pc if pc is not None else backend
    dev = plan.device
    n, nh = plan.n_local, plan.n_halo
    small = 1e-20
    with _on_stream(backend):
        b = torch.as_tensor(b_local, dtype=torch.float64, device=dev)
        aug = torch.zeros(n + nh, dtype=torch.float64, device=dev)

        def A(v):
            aug[:n] = v
            plan.exchange(aug)
            return backend.spmv(aug)

        phi = torch.zeros(n, dtype=torch.float64, device=dev) if x0_local is None else \
            torch.as_tensor(x0_local, dtype=torch.float64, device=dev).clone()
        res = b - A(phi)
        reso = res.clone()
        t = _reduce(torch.dot(res, res), torch.dot(res, reso))
        res0 = torch.sqrt(t[0])
        beta_next = t[1]
        pk = torch.zeros_like(res)
        uk = torch.zeros_like(res)
        one = torch.ones((), dtype=torch.float64, device=dev)
        alpha, beto, gama = one.clone(), one.clone(), one.clone()
        hist = torch.zeros(max(maxiter, 1), dtype=torch.float64, device=dev)
        live = torch.ones((), dtype=torch.bool, device=dev)
        last = torch.zeros((), dtype=torch.int64, device=dev)
        for it in range(maxiter):
            beta = beta_next
            omega = (beta * gama) / (alpha * beto + small)
            beto = beta
            pk = pk + (-alpha) * uk
            pk = omega * pk
            pk = pk + res
            uk = A(M.precond(pk))
            tmp = _reduce(torch.dot(uk, reso))[0]
            gama = beta / (tmp + small)
            sk = res + (-gama) * uk
            vk = A(M.precond(sk))
            t = _reduce(torch.dot(vk, sk), torch.dot(vk, vk))
            alpha = t[0] / (t[1] + small)
            phi_new = phi + gama * pk
            phi_new = phi_new + alpha * sk
            phi = torch.where(live, phi_new, phi)
            res = sk + (-alpha) * vk
            t = _reduce(torch.dot(res, res), torch.dot(res, reso))
            rsm = torch.sqrt(t[0]) / (res0 + small)
            beta_next = t[1]
            hist[it] = torch.where(live, rsm, hist[it])
            last = torch.where(live, torch.full_like(last, it), last)
            live = live & ~(rsm < tol)
            if (it + 1) % check_every == 0 or it + 1 == maxiter:
                _checkpoint(backend)
                if not bool(live):
                    break
        x = M.precond(phi)
        used = int(last)
        resvec = hist[: used + 1].cpu().numpy()
        _checkpoint(backend)
    return x, resvec, used


def pcg(backend, plan: HaloPlan, b_local, x0_local=None, tol=1e-8, maxiter=1000, pc=None, check_every=16):
    """The reference's standard PCG, "cgm" (intel/mpisolver-C-v1.cpp:193-272),
    on the rank's rows with reduced dot products; pc as for bicgstab.
    Returns (x_local, resvec, usediter) in the reference's convention.
    Device scalars and periodic convergence checks as in bicgstab; two
    reductions per iteration ((p, Ap), ((r, z), (r, r)))."""
    M = pc if pc is not None else backend
    dev = plan.device
    n, nh = plan.n_local, plan.n_halo
    small = 1e-20
    with _on_stream(backend):
        b = torch.as_tensor(b_local, dtype=torch.float64, device=dev)
        aug = torch.zeros(n + nh, dtype=torch.float64, device=dev)

        def A(v):
            aug[:n] = v
            plan.exchange(aug)
            return backend.spmv(aug)

        phi = torch.zeros(n, dtype=torch.float64, device=dev) if x0_local is None else \
            torch.as_tensor(x0_local, dtype=torch.float64, device=dev).clone()
        res = b - A(phi)
        zk = M.precond(res)
        t = _reduce(torch.dot(res, res), torch.dot(res, zk))
        res0, tao = torch.sqrt(t[0]), t[1]
        pk = zk.clone()
        hist = torch.zeros(max(maxiter, 1), dtype=torch.float64, device=dev)
        live = torch.ones((), dtype=torch.bool, device=dev)
        last = torch.zeros((), dtype=torch.int64, device=dev)
        for it in range(maxiter):
            taoo = tao
            apk = A(pk)
            sigma = _reduce(torch.dot(pk, apk))[0]
            alpha = tao / (sigma + small)
            phi = torch.where(live, phi + alpha * pk, phi)
            res = res + (-alpha) * apk
            zk = M.precond(res)
            t = _reduce(torch.dot(res, zk), torch.dot(res, res))
            tao = t[0]
            beta = tao / (taoo + small)
            pk = beta * pk
            pk = pk + zk
            rsm = torch.sqrt(t[1]) / (res0 + small)
            hist[it] = torch.where(live, rsm, hist[it])
            last = torch.where(live, torch.full_like(last, it), last)
            live = live & ~(rsm < tol)
            if (it + 1) % check_every == 0 or it + 1 == maxiter:
                _checkpoint(backend)
                if not bool(live):
                    break
        used = int(last)
        resvec = hist[: used + 1].cpu().numpy()
        _checkpoint(backend)
    return phi, resvec, used


def _rotate(dx, dy, c, s):
    """intel/mpisolver-C-v1.cpp:1249-1258 (applyplanerotationc)"""
    t = c * dx + s * dy
    return t, -s * dx + c * dy


def _generate(dx, dy):
    """intel/mpisolver-C-v1.cpp:1260-1279 (generateplanerotationc)"""
    if dy == 0.0:
        return 1.0, 0.0
    if abs(dy) > abs(dx):
        t = dx / dy
        sn = 1.0 / (1.0 + t * t) ** 0.5
        return t * sn, sn
    t = dy / dx
    cs = 1.0 / (1.0 + t * t) ** 0.5
    return cs, t * cs


def gmres(backend, plan: HaloPlan, b_local, x0_local=None, tol=1e-8, maxiter=1000, restart=30, pc=None):
    """The reference's left-preconditioned GMRES(restart)
    (intel/mpisolver-C-v1.cpp:933-1087): modified Gram-Schmidt with each dot
    product reduced over the ranks, Givens rotations and the back
    substitution (updatec, :1281-1301) on the host, the reference's update
    with i columns on convergence.  Returns (x_local, resvec, usediter);
    resvec is indexed by the global iteration."""
    M = pc if pc is not None else backend
    dev = plan.device
    n, nh = plan.n_local, plan.n_halo
    small = 1e-20
    m = restart
    b = torch.as_tensor(b_local, dtype=torch.float64, device=dev)
    aug = torch.zeros(n + nh, dtype=torch.float64, device=dev)

    def A(v):
        aug[:n] = v
        plan.exchange(aug)
        return backend.spmv(aug)

    def update(phi, k, H, s, V):
        y = list(s[:k])
        for i in range(k - 1, -1, -1):
            y[i] = y[i] / (H[i][i] + small)
            for j in range(i - 1, -1, -1):
                y[j] = y[j] - H[j][i] * y[i]
        for i in range(k):
            phi = phi + y[i] * V[i]
        return phi

    phi = torch.zeros(n, dtype=torch.float64, device=dev) if x0_local is None else \
        torch.as_tensor(x0_local, dtype=torch.float64, device=dev).clone()
    res = M.precond(b - A(phi))
    res0 = _gdot(res, res) ** 0.5
    beta = res0
    resvec, used, j = [], 0, 0
    while j < maxiter:
        H = [[0.0] * m for _ in range(m + 1)]
        s, cs, sn = [0.0] * (m + 1), [0.0] * (m + 1), [0.0] * (m + 1)
        res = (1.0 / (beta + small)) * res
        V = [res.clone()]
        s[0] = beta
        i = 0
        while i < m and j < maxiter:
            w = M.precond(A(V[i]))
            for k in range(i + 1):
                t = _gdot(w, V[k])
                H[k][i] = t
                w = w + (-t) * V[k]
            t = _gdot(w, w) ** 0.5
            H[i + 1][i] = t
            w = (1.0 / (t + small)) * w
            V.append(w)
            for k in range(i):
                H[k][i], H[k + 1][i] = _rotate(H[k][i], H[k + 1][i], cs[k], sn[k])
            cs[i], sn[i] = _generate(H[i][i], H[i + 1][i])
            H[i][i], H[i + 1][i] = _rotate(H[i][i], H[i + 1][i], cs[i], sn[i])
            s[i], s[i + 1] = _rotate(s[i], s[i + 1], cs[i], sn[i])
            err = abs(s[i + 1]) / (res0 + small)
            resvec.append(err)
            if err < tol:
                return update(phi, i, H, s, V), np.asarray(resvec), j
            i += 1
            j += 1
        phi = update(phi, m, H, s, V)
        res = M.precond(b - A(phi))
        beta = abs(s[m])
        used = j
    return phi, np.asarray(resvec), used
