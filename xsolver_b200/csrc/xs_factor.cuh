// ILU(0) factorisations on A's sparsity pattern.
//
// Exact ILU(0): the reference factorises on the CPU (hip/Precond/
// ilut_diag_in_csr.cpp:347-405, ilu0_simple: IKJ order, pivots clamped to
// 1e-20).  Here the same up-looking row update runs on the GPU: row i is
// processed by one thread once every row k it references (its strictly lower
// columns) is final, so rows of one dependency level run in parallel.  The
// row update is performed in exactly the CPU order (pivot division, then the
// merge with row k's upper part), so the factors are bitwise identical to the
// reference's.  Completion of a row is published with a release store of the
// launch's epoch in a flag array; waiters poll with acquire loads (bounded).
//
// ParILU: the reference's fixed-point sweep (hip/Precond/gpuparilu.cpp:46-102,
// ilu0_ij_aw, one thread per nonzero, pivot clamp 1e-10) applied as
// synchronous sweeps (read the previous iterate, write the next), which makes
// the result deterministic; the reference updates in place asynchronously.
//
// Split: the combined values are rewritten into the seqilu0 layout
// (hip/HostMatrix/HostMatrixCSR.cpp:164-197): L entries unchanged, diagonal
// entry := dinv_i = 1/u_ii, U entries := u_ij * dinv_i.
#pragma once
#include "xs_internal.cuh"

namespace xs {


// exact ILU(0), thread per row in level order (perm/level from the L analysis)
__global__ void __launch_bounds__(128) k_ilu0_rows(int n, const int *__restrict__ rp, const int *__restrict__ ci,
                                                  const int *__restrict__ uptr, const int *__restrict__ perm, double *luv,
                                                  int *flag, int epoch, int *err, unsigned *ticket)
{
    __shared__ int s_blk;
    if (threadIdx.x == 0) {
        unsigned t = atomicAdd(ticket, 1u);
        if (t == gridDim.x - 1) *ticket = 0u;
        s_blk = (int)t;
    }
    __syncthreads();
    const int p = s_blk * 128 + (int)threadIdx.x;
    if (p >= n) return;
    const int i = perm[p];
    const int rs = rp[i], re = rp[i + 1], up = uptr[i];
    for (int j = rs; j < up; j++) {
        const int k = ci[j];
        long spins = 0;
        unsigned long long t0 = 0;
        while (ld_acquire(flag + k) != epoch) {
            __nanosleep(32);  // yield point: the producer may be a lane of this warp
            if ((++spins & 255) == 0) {
                const unsigned long long t = gtimer();
                if (t0 == 0) t0 = t;
                else if (t - t0 > WAIT_LIMIT_NS) {
                    atomicOr(err, DEV_FACTOR_TIMEOUT);
                    return;
                }
                if (*(volatile int *)err) return;
            }
        }
        const int ukp = uptr[k];
        const int kend = rp[k + 1];
        double piv = __ldcg(luv + ukp);
        if (fabs(piv) < 1e-20) piv = 1e-20;  // no-op: row k clamped its own pivot
        const double lij = luv[j] / piv;
        luv[j] = lij;
        int subptr = ukp;
        for (int jj = j + 1; jj < re; jj++) {
            const int kk = ci[jj];
            while (subptr < kend && __ldg(ci + subptr) < kk) subptr++;
            if (subptr < kend) {
                if (__ldg(ci + subptr) == kk) {
                    const double t = lij * __ldcg(luv + subptr);
                    luv[jj] = luv[jj] - t;
                }
            } else
                break;
        }
    }
    double d = luv[up];
    if (fabs(d) < 1e-20) {
        d = 1e-20;
        luv[up] = d;
    }
    __threadfence();
    st_release(flag + i, epoch);
}

// one synchronous ParILU sweep over A's nonzeros
//   rowof[k]  row of entry k;  uptr[i] diagonal position of row i
//   ucp/ucpos: upper part by columns: for column j, positions ucpos[ucp[j]..ucp[j+1])
//              of the entries (r, j) with r <= j, rows ascending (diagonal last)
__global__ void k_parilu_sweep(long nnz, const int *__restrict__ rp, const int *__restrict__ ci,
                               const int *__restrict__ rowof, const int *__restrict__ uptr, const int *__restrict__ ucp,
                               const int *__restrict__ ucpos, const double *__restrict__ a, const double *__restrict__ cur,
                               double *__restrict__ nxt)
{
    for (long k = blockIdx.x * (long)blockDim.x + threadIdx.x; k < nnz; k += (long)gridDim.x * blockDim.x) {
        const int i = rowof[k], j = ci[k];
        double s = a[k], sp = 0.0;
        int il = rp[i];
        const int ilend = uptr[i] + 1;  // position uptr[i] stands for L's unit diagonal
        int iu = ucp[j];
        const int iuend = ucp[j + 1];
        while (il < ilend && iu < iuend) {
            sp = 0.0;
            const int jl = ci[il];
            const int upos = ucpos[iu];
            const int ju = rowof[upos];
            const double lval = (il == uptr[i]) ? 1.0 : cur[il];
            const double uval = cur[upos];
            sp = (jl == ju) ? lval * uval : sp;
            s = (jl == ju) ? s - sp : s;
            il = (jl <= ju) ? il + 1 : il;
            iu = (jl >= ju) ? iu + 1 : iu;
        }
        s += sp;  // undo the last subtraction (the k = min(i,j) term)
        double out;
        if (i > j) {
            double t = cur[uptr[j]];
            if (fabs(t) < 1e-10) t = (t >= 0 ? 1e-10 : -1e-10);
            t = s / t;
            out = isfinite(t) ? t : cur[k];
        } else {
            if (i == j && fabs(s) < 1e-10) s = (s >= 0 ? 1e-10 : -1e-10);
            out = isfinite(s) ? s : cur[k];
        }
        nxt[k] = out;
    }
}

// combined LU values -> seqilu0 layout (in place into fv)
__global__ void k_split_lu(int n, const int *__restrict__ rp, const int *__restrict__ ci, const int *__restrict__ uptr,
                           const double *__restrict__ luv, double *__restrict__ fv)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int up = uptr[i];
        const double dinv = 1 / luv[up];
        for (int k = rp[i]; k < up; k++) fv[k] = luv[k];
        fv[up] = dinv;
        for (int k = up + 1; k < rp[i + 1]; k++) fv[k] = luv[k] * dinv;
    }
}

// Jacobi: dinv_i = 1/(a_ii + 1e-20) (intel/HostMatrix.h:127-137)
template <typename DT>
__global__ void k_jacobi_init(int n, const int *__restrict__ uptr, const double *__restrict__ a, DT *dinv)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const double t = a[uptr[i]] + 1e-20;
        dinv[i] = (DT)(1.0 / t);
    }
}

}  // namespace xs
