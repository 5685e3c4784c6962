// Multi-right-hand-side PCG and exact ILU solves.
//
// The reference solves one right-hand side per call (hip/xsolver_c.cpp:
// 274-292, xsolver_solve); the batch entry points here (xs_solve_batch,
// xs_adjoint_batch) used to loop over right-hand sides.  For PCG with an
// exact preconditioner solve they now carry k right-hand sides through one
// iteration together: k vectors are stored interleaved by row (element
// (i, c) at i*k + c), so one pass over the matrix serves k products, and one
// dependency chain of the triangular solves serves k solves (the chain's
// latency, not its bytes, bounds the exact solve).  Every column has its own
// scalars and convergence state (one KState per column); a converged column
// stops changing exactly where its own solve would have stopped, and the
// iteration ends when every column has.
//
// Row sums (SpMV and triangular solves) use the operations and entry order
// of the single-right-hand-side kernels, so they give the same bits; dot
// products reduce in their own deterministic order (per column: threads in
// block order, then blocks in order), so the scalars agree with a single
// solve's to rounding.
#pragma once
#include <vector>
#include "xs_solvers.cuh"

namespace xs {

constexpr int BATCH_MAX = 16;
constexpr int BATCH_THREADS = 256;

// batched kernels on (1, default) or the right-hand sides solved one by one (0)
struct BatchTuning {
    int enabled = 1;
};
BatchTuning &batch_tuning();

// ---------------------------------------------------------------- per-column reduction
// Every thread holds NV partial sums for column threadIdx.x % k (blockDim is
// a multiple of k and the grid stride keeps each thread on one column).
// Block partials per column go to slot.part[(v*k + c)*G + block]; the last
// block (ticket) sums them in block order.  Returns true in every thread of
// the last block, with the totals in tot[v*k + c].
template <int NV>
__device__ bool block_reduce_cols(const double (&v)[NV], int k, RedSlot slot, double *tot)
{
    __shared__ double sv[NV][BATCH_THREADS];
    __shared__ bool s_last;
    const int t = threadIdx.x, nb = blockDim.x, G = gridDim.x;
#pragma unroll
    for (int a = 0; a < NV; a++) sv[a][t] = v[a];
    __syncthreads();
    if (t < k) {
#pragma unroll
        for (int a = 0; a < NV; a++) {
            double s = 0.0;
            for (int q = t; q < nb; q += k) s += sv[a][q];
            slot.part[((long)a * k + t) * G + blockIdx.x] = s;
        }
        __threadfence();
    }
    __syncthreads();
    if (t == 0) {
        const unsigned tk = atomicAdd(slot.ticket, 1u);
        s_last = (tk == (unsigned)G - 1);
    }
    __syncthreads();
    if (!s_last) return false;
    __threadfence();
    const int per = nb / k, c = t % k, j = t / k;
    double s[NV];
#pragma unroll
    for (int a = 0; a < NV; a++) {
        s[a] = 0.0;
        for (int b = j; b < G; b += per) s[a] += __ldcg(slot.part + ((long)a * k + c) * G + b);
    }
    __syncthreads();
#pragma unroll
    for (int a = 0; a < NV; a++) sv[a][t] = s[a];
    __syncthreads();
    if (t < k) {
#pragma unroll
        for (int a = 0; a < NV; a++) {
            double acc = 0.0;
            for (int q = t; q < per * k; q += k) acc += sv[a][q];
            tot[a * k + t] = acc;
        }
    }
    if (t == 0) *slot.ticket = 0u;
    __syncthreads();
    return true;
}

inline int batch_block(int k) { return (BATCH_THREADS / k) * k; }
inline int batch_grid() { return geom().red_grid; }

// every column's solve has ended: the later kernels of the iteration skip
__device__ inline void batch_set_all_done(const KState *st, int k, int *all_done)
{
    int all = 1;
    for (int c = 0; c < k; c++) all &= st[c].done != 0;
    *all_done = all;
}

// ---------------------------------------------------------------- batched CSR SpMV
enum BSpmvMode { BS_RESID = 1, BS_DOT_SIGMA = 2 };

// MODE BS_RESID: Y = B - A X, per column r.r into sc[S_RES0SQ] (every column)
// MODE BS_DOT_SIGMA: Y = A X, per column w.y -> sigma, alpha = tao/(sigma + small)
//   (EpiDot1 with M_CGM_SIGMA), columns already converged skipped
template <int MODE>
__global__ void __launch_bounds__(BATCH_THREADS) k_bspmv(int n, int k, const int *__restrict__ rp,
                                                        const int *__restrict__ ci, const double *__restrict__ v,
                                                        const double *__restrict__ X, double *__restrict__ Y,
                                                        const double *__restrict__ W, KState *st, int *all_done,
                                                        RedSlot slot)
{
    __shared__ double tot[BATCH_MAX];
    if (*all_done) return;
    const int c = threadIdx.x % k;
    const bool active = MODE == BS_RESID || st[c].done == 0;
    const long m = (long)n * k;
    double acc[1] = {0.0};
    if (active) {
        for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < m; q += (long)gridDim.x * blockDim.x) {
            const int i = (int)(q / k);
            double sum = 0.0;
            for (int e = __ldg(rp + i); e < __ldg(rp + i + 1); e++) sum += __ldg(v + e) * __ldg(X + (long)__ldg(ci + e) * k + c);
            if (MODE == BS_RESID) {
                const double y = __ldg(W + q) - sum;  // W = B
                Y[q] = y;
                acc[0] += y * y;
            } else {
                Y[q] = sum;
                acc[0] += __ldg(W + q) * sum;  // W = P
            }
        }
    }
    if (block_reduce_cols<1>(acc, k, slot, tot)) {
        if (threadIdx.x < k) {
            KState *s = st + threadIdx.x;
            const double d = tot[threadIdx.x];
            if (MODE == BS_RESID) {
                s->sc[S_RES0SQ] = d;
            } else if (s->done == 0) {
                s->sc[S_SIGMA] = d;
                s->sc[S_ALPHA] = s->sc[S_TAO] / (d + KSMALL);
                if (!isfinite(d)) {
                    s->err |= DEV_BREAKDOWN;
                    s->done = 3;
                }
            }
        }
        __syncthreads();
        if (threadIdx.x == 0) batch_set_all_done(st, k, all_done);
    }
}

// ---------------------------------------------------------------- batched PCG vector ops
// The element operations are those of OpCgmInit / OpCgmUpdate / OpDotRZ /
// OpPUpdate (same expressions, so the same bits for the same scalars).
template <int OP>
__global__ void __launch_bounds__(BATCH_THREADS) k_bpcg(int n, int k, KState *st, int *all_done, double *X,
                                                       double *R, double *Z, double *P, const double *AP, RedSlot slot)
{
    constexpr int NV = OP == 0 ? 2 : (OP == 3 ? 0 : 1);
    __shared__ double tot[2 * BATCH_MAX];
    if (OP != 0 && *all_done) return;
    const int c = threadIdx.x % k;
    const bool active = OP == 0 || st[c].done == 0;
    const long m = (long)n * k;
    double acc[NV > 0 ? NV : 1] = {};
    double a = 0.0;
    if (OP == 1) a = st[c].sc[S_ALPHA];
    if (OP == 3) a = st[c].sc[S_BETA];
    if (active) {
        for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < m; q += (long)gridDim.x * blockDim.x) {
            if (OP == 0) {  // init: acc0 = r.r, acc1 = r.z ; p = z
                const double ri = R[q], zi = Z[q];
                acc[0] += ri * ri;
                acc[1] += ri * zi;
                P[q] = zi;
            } else if (OP == 1) {  // x += alpha p ; r -= alpha Ap ; acc r.r
                const double minalpha = -a;
                X[q] = X[q] + a * P[q];
                const double ri = R[q] + minalpha * AP[q];
                R[q] = ri;
                acc[0] += ri * ri;
            } else if (OP == 2) {  // acc r.z
                acc[0] += R[q] * Z[q];
            } else {  // p = beta p + z
                const double t = a * P[q];
                P[q] = t + Z[q];
            }
        }
    }
    if constexpr (NV > 0) {
        if (block_reduce_cols<NV>(acc, k, slot, tot)) {
            if (threadIdx.x < k) {
                KState *s = st + threadIdx.x;
                const int cc = threadIdx.x;
                if (OP == 0) {
                    s->sc[S_TAO] = tot[k + cc];
                    init_record(s, sqrt(tot[cc]));
                } else if (s->done == 0) {
                    if (OP == 1) {
                        record_and_test(s, sqrt(tot[cc]));
                    } else {
                        const double d = tot[cc];
                        s->sc[S_TAOO] = s->sc[S_TAO];
                        s->sc[S_TAO] = d;
                        s->sc[S_BETA] = d / (s->sc[S_TAOO] + KSMALL);
                        if (!isfinite(d)) {
                            s->err |= DEV_BREAKDOWN;
                            s->done = 3;
                        }
                    }
                }
            }
            __syncthreads();
            if (threadIdx.x == 0) batch_set_all_done(st, k, all_done);
        }
    }
}

// ---------------------------------------------------------------- batched triangular solves
// Level-ordered layout: work items are (position, column) pairs in position
// order (a dependency always sits at an earlier pair), taken by blocks
// through a ticket; otherwise as trsv_row.
template <bool UPPER>
__global__ void __launch_bounds__(TRSV_THREADS) k_trsv_level_multi(TrsvArgs<double> P, int k,
                                                                   const double *__restrict__ dinv, const double *rhs,
                                                                   double *self, double *out_user, double *reset_other,
                                                                   const int *all_done, int *err, unsigned *ticket,
                                                                   int backoff_ns)
{
    if (all_done && *all_done) return;
    __shared__ int s_blk;
    const long m = (long)P.n * k;
    const unsigned work = (unsigned)((m + TRSV_THREADS - 1) / TRSV_THREADS);
    const unsigned last = work + gridDim.x - 1;
    bool ok = true;
    while (true) {
        __syncthreads();
        if (threadIdx.x == 0) {
            const unsigned t = atomicAdd(ticket, 1u);
            if (t == last) *ticket = 0u;
            s_blk = (int)t;
        }
        __syncthreads();
        const long b = s_blk;
        if ((unsigned)b >= work) break;
        const long q = b * TRSV_THREADS + threadIdx.x;
        if (!ok || q >= m) continue;
        const int p = (int)(q / k), c = (int)(q % k);
        const int row = __ldg(P.perm + p);
        const long rq = (long)row * k + c;
        double acc = UPPER ? rhs[rq] * __ldg(dinv + p) : rhs[rq];
        if (reset_other) reset_other[rq] = Sentinel<double>::value();
        for (int e = __ldg(P.prp + p); e < __ldg(P.prp + p + 1) && ok; e++) {
            const double *dp = self + (long)__ldg(P.pci + e) * k + c;
            double y;
            ok = tile_poll<double>(dp, err, backoff_ns, y);
            acc = msub(acc, y, __ldg(P.pv + e));
        }
        if (!ok) continue;
        st_publish(self + rq, acc);
        if (out_user) out_user[rq] = acc;
    }
}

// Box layout: work items are (box, column group) pairs of KC columns, taken
// in box order.  As k_trsv_tiles, a box's rows, entries and (U) dinv are
// staged in shared memory by asynchronous copies and its right-hand sides
// gathered (KC per row) while the halo is polled; the internal levels then
// read shared memory only, the KC threads of a row lane handling the row for
// the group's columns.
constexpr int TILEM_THREADS = 512;

// shared-memory layout of one box item with KC columns (FP64)
struct TileSmemM {
    size_t y, rhs, dinv, pv, row, eptr, pci, total;
    static __host__ __device__ TileSmemM of(int rows, int halo, int entries, int kc)
    {
        auto al = [](size_t b) { return (b + 15) & ~(size_t)15; };
        TileSmemM m;
        m.y = 0;
        m.rhs = m.y + al((size_t)(rows + halo) * kc * sizeof(double));
        m.dinv = m.rhs + al((size_t)rows * kc * sizeof(double));
        m.pv = m.dinv + al((size_t)rows * sizeof(double));
        m.row = m.pv + al((size_t)entries * sizeof(double) + 8);
        m.eptr = m.row + al((size_t)rows * sizeof(int));
        m.pci = m.eptr + al((size_t)(rows + 1) * sizeof(int));
        m.total = m.pci + al((size_t)entries * sizeof(int));
        return m;
    }
};

template <int KC, bool UPPER>
__global__ void __launch_bounds__(TILEM_THREADS) k_trsv_tiles_multi(TileArgs<double> P, int k, int ngroups,
                                                                    const double *__restrict__ dinv, const double *rhs,
                                                                    double *self, double *out_user, double *reset_other,
                                                                    const int *all_done, int *err, unsigned *ticket,
                                                                    int backoff_ns)
{
    if (all_done && *all_done) return;
    extern __shared__ __align__(16) unsigned char tm_smem[];
    const TileSmemM L = TileSmemM::of(P.max_rows, P.max_halo, P.max_entries, KC);
    double *ysh = (double *)(tm_smem + L.y);
    double *s_rhs = (double *)(tm_smem + L.rhs);
    double *s_dinv = (double *)(tm_smem + L.dinv);
    double *s_pv = (double *)(tm_smem + L.pv);
    int *s_row = (int *)(tm_smem + L.row);
    int *s_eptr = (int *)(tm_smem + L.eptr);
    int *s_pci = (int *)(tm_smem + L.pci);
    __shared__ int s_item;
    const int items = P.ntiles * ngroups;
    const unsigned last = (unsigned)items + gridDim.x - 1;
    constexpr int RSTEP = TILEM_THREADS / KC;  // row lanes
    const int tid = threadIdx.x, pc = tid % KC, pr = tid / KC;
    bool ok = true;
    while (true) {
        __syncthreads();
        if (tid == 0) {
            const unsigned t = atomicAdd(ticket, 1u);
            if (t == last) *ticket = 0u;
            s_item = (int)t;
        }
        __syncthreads();
        const int it = s_item;
        if (it >= items) break;
        const int t = it / ngroups, g = it % ngroups;
        const int col = g * KC + pc;  // this thread's column
        const bool col_ok = col < k;
        const int p0 = __ldg(P.tile_pos + t), p1 = __ldg(P.tile_pos + t + 1);
        const int l0 = __ldg(P.tile_lvl + t), l1 = __ldg(P.tile_lvl + t + 1);
        const int h0 = __ldg(P.halo_ptr + t), h1 = __ldg(P.halo_ptr + t + 1);
        const int rows = p1 - p0;
        const int e0 = __ldg(P.prp + p0), e1 = __ldg(P.prp + p1);
        for (int i = tid; i < rows; i += TILEM_THREADS) cp_async4(s_row + i, P.perm + p0 + i);
        cp_async_commit();
        for (int i = tid; i <= rows; i += TILEM_THREADS) cp_async4(s_eptr + i, P.prp + p0 + i);
        for (int i = tid; i < e1 - e0; i += TILEM_THREADS) {
            cp_async4(s_pci + i, P.pci + e0 + i);
            cp_async8(s_pv + i, P.pv + e0 + i);
        }
        if (UPPER)
            for (int i = tid; i < rows; i += TILEM_THREADS) cp_async8(s_dinv + i, dinv + p0 + i);
        cp_async_commit();
        cp_async_wait<1>();
        __syncthreads();
        for (int i = pr; i < rows; i += RSTEP)
            if (col_ok) cp_async8(s_rhs + i * KC + pc, rhs + (long)s_row[i] * k + col);
        cp_async_commit();
        for (int h = h0 + pr; h < h1; h += RSTEP) {
            double y = 0.0;
            if (ok && col_ok) ok = tile_poll<double>(self + (long)__ldg(P.halo_row + h) * k + col, err, backoff_ns, y);
            ysh[(rows + (h - h0)) * KC + pc] = y;
        }
        cp_async_wait<0>();
        __syncthreads();
        for (int l = l0; l < l1; l++) {
            const int pa = __ldg(P.lvl_ptr + l) - p0, pb = __ldg(P.lvl_ptr + l + 1) - p0;
            for (int i = pa + pr; i < pb; i += RSTEP) {
                const int row = s_row[i];
                double acc = 0.0;
                if (col_ok) acc = UPPER ? s_rhs[i * KC + pc] * s_dinv[i] : s_rhs[i * KC + pc];
                const int k1 = s_eptr[i + 1] - e0;
                for (int q = s_eptr[i] - e0; q < k1; q++) acc = msub(acc, ysh[s_pci[q] * KC + pc], s_pv[q]);
                ysh[i * KC + pc] = acc;
                if (col_ok) {
                    const long rq = (long)row * k + col;
                    if (reset_other) reset_other[rq] = Sentinel<double>::value();
                    st_publish(self + rq, acc);
                    if (out_user) out_user[rq] = acc;
                }
            }
            __syncthreads();
        }
    }
}

// ---------------------------------------------------------------- batched preconditioner apply
struct BatchPrecond {
    DBuf<double> lb, ub;  // readiness buffers, n*k each (NaN sentinel)
    DBuf<unsigned> ticket;
    int n = 0, k = 0;
    void ensure(int nn, int kk, cudaStream_t s)
    {
        if (n == nn && k == kk && lb.p) return;
        n = nn;
        k = kk;
        lb.alloc((size_t)n * k);
        ub.alloc((size_t)n * k);
        k_fill_sentinel<double><<<256, 256, 0, s>>>(lb.p, (int)((size_t)n * k));
        k_fill_sentinel<double><<<256, 256, 0, s>>>(ub.p, (int)((size_t)n * k));
        if (!ticket.p) ticket.alloc(1);
        check_launch();
    }
    void rearm(cudaStream_t s)
    {
        if (!lb.p) return;
        k_fill_sentinel<double><<<256, 256, 0, s>>>(lb.p, (int)((size_t)n * k));
        k_fill_sentinel<double><<<256, 256, 0, s>>>(ub.p, (int)((size_t)n * k));
        check_launch();
    }
};

// column-group size of the box kernel: the most columns (<= 4) whose box
// and halo values fit in shared memory
inline int tiles_multi_kc(const TriDev &T, int k)
{
    int kc = std::min(k, 4);
    while (kc > 1 && TileSmemM::of(T.t_max_rows, T.t_max_halo, T.t_max_entries, kc).total > TILE_SMEM_MAX) kc--;
    return kc;
}

template <bool UPPER>
inline void launch_trsv_multi(const TriDev &T, int k, unsigned *ticket, const double *dinv, const double *rhs,
                              double *self, double *out_user, double *reset_other, const int *all_done, int *err,
                              cudaStream_t s)
{
    const int bo = trsv_tuning().backoff_ns;
    if (T.tiled) {
        const int kc = tiles_multi_kc(T, k);
        const int ng = (k + kc - 1) / kc;
        const size_t smem = TileSmemM::of(T.t_max_rows, T.t_max_halo, T.t_max_entries, kc).total;
        if (smem > TILE_SMEM_MAX) throw Status(XS_ERR_UNSUPPORTED);
        const int fit = std::max(1, (int)((220u * 1024u) / (smem + 1024)));
        const int g = std::min(T.ntiles * ng, geom().sms * std::min(2, fit));
        // the largest dynamic shared memory is enabled once per kernel, at
        // the first (uncaptured) apply of a solve
        static size_t attr[2][5] = {};
        size_t &at = attr[UPPER ? 1 : 0][kc];
        auto go = [&](auto kern) {
            if (smem > at) {
                XS_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
                at = smem;
            }
            kern<<<g, TILEM_THREADS, smem, s>>>(T.targs<double>(), k, ng, dinv, rhs, self, out_user, reset_other,
                                                all_done, err, ticket, bo);
        };
        if (kc == 4) go(k_trsv_tiles_multi<4, UPPER>);
        else if (kc == 3) go(k_trsv_tiles_multi<3, UPPER>);
        else if (kc == 2) go(k_trsv_tiles_multi<2, UPPER>);
        else go(k_trsv_tiles_multi<1, UPPER>);
    } else {
        if (T.chunked) throw Status(XS_ERR_UNSUPPORTED);
        const long m = (long)T.n * k;
        const long work = (m + TRSV_THREADS - 1) / TRSV_THREADS;
        const int g = (int)std::min<long>(work, (long)std::max(1, trsv_tuning().blocks_per_sm) * geom().sms);
        k_trsv_level_multi<UPPER><<<g, TRSV_THREADS, 0, s>>>(T.args<double>(), k, dinv, rhs, self, out_user,
                                                              reset_other, all_done, err, ticket, bo);
    }
    check_launch();
}

static __global__ void k_bdiag_scale(long m, int k, const double *__restrict__ d, const double *__restrict__ x,
                              double *__restrict__ y, const int *all_done)
{
    if (*all_done) return;
    for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < m; q += (long)gridDim.x * blockDim.x)
        y[q] = x[q] * d[q / k];
}
static __global__ void k_bcopy(long m, const double *__restrict__ x, double *__restrict__ y, const int *all_done)
{
    if (*all_done) return;
    for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < m; q += (long)gridDim.x * blockDim.x) y[q] = x[q];
}

// whether M can be applied to k interleaved columns (FP64; exact triangular
// solves for the ILU family)
inline bool batch_precond_ok(const PrecondDev &M)
{
    if (M.type == PC_NONE || M.type == PC_JACOBI) return true;
    if (pc_triangular(M.type))
        return M.trsv_mode == 0 && !M.L.chunked && !M.U.chunked && M.L.pv64.p && M.U.pv64.p && M.U.dinv64.p;
    return false;
}

// Z = M^{-1} X on k interleaved columns
inline void batch_apply(PrecondDev &M, BatchPrecond &B, int k, const double *X, double *Z, const int *all_done,
                        cudaStream_t s)
{
    const int n = M.n;
    const long m = (long)n * k;
    if (M.type == PC_NONE) {
        k_bcopy<<<geom().sms * 4, 256, 0, s>>>(m, X, Z, all_done);
    } else if (M.type == PC_JACOBI) {
        k_bdiag_scale<<<geom().sms * 4, 256, 0, s>>>(m, k, M.jdiag64.p, X, Z, all_done);
    } else {
        B.ensure(n, k, s);
        launch_trsv_multi<false>(M.L, k, B.ticket.p, nullptr, X, B.lb.p, nullptr, B.ub.p, all_done, M.err, s);
        launch_trsv_multi<true>(M.U, k, B.ticket.p, M.U.dinv64.p, B.lb.p, B.ub.p, Z, B.lb.p, all_done, M.err, s);
    }
    check_launch();
}

// ---------------------------------------------------------------- batched PCG
struct BatchState {
    DBuf<KState> st;  // one per column
    DBuf<int> all_done;
    DBuf<double> hist, part;
    DBuf<unsigned> ticket;
    std::vector<KState> h;
    int k = 0, cap = 0;
    void prepare(int kk, int maxiter, double tol, double abstol, cudaStream_t s)
    {
        if (kk != k || cap < maxiter + 2) {
            k = kk;
            cap = std::max(cap, maxiter + 2);
            st.alloc(k);
            hist.alloc((size_t)k * cap);
        }
        if (!all_done.p) all_done.alloc(1);
        if (!ticket.p) ticket.alloc(1);
        const size_t need = (size_t)2 * BATCH_MAX * batch_grid();
        if (part.n < need) part.alloc(need);
        h.assign(k, KState());
        for (int c = 0; c < k; c++) {
            std::memset(&h[c], 0, sizeof(KState));
            h[c].tol = tol;
            h[c].abstol = abstol;
            h[c].maxiter = maxiter;
            h[c].hist = hist.p + (size_t)c * cap;
            h[c].hist_rel = nullptr;
        }
        XS_CUDA(cudaMemcpyAsync(st.p, h.data(), sizeof(KState) * k, cudaMemcpyHostToDevice, s));
        XS_CUDA(cudaMemsetAsync(all_done.p, 0, sizeof(int), s));
    }
    RedSlot slot() const { return RedSlot{part.p, ticket.p}; }
    // read the states back (after the stream is synchronised by the caller)
    void fetch(cudaStream_t s)
    {
        XS_CUDA(cudaMemcpyAsync(h.data(), st.p, sizeof(KState) * k, cudaMemcpyDeviceToHost, s));
        XS_CUDA(cudaStreamSynchronize(s));
    }
};

struct BatchPcg {
    VecPool<double> pool;
    GraphCache gc;
    // B, X: k interleaved columns (X holds x0 on entry)
    void run(cudaStream_t s, const DevCsr &A, PrecondDev &M, BatchPrecond &BP, BatchState &S, int k, const double *B,
             double *X, long long *launches)
    {
        const int n = A.n;
        const long m = (long)n * k;
        if (pool.n != (int)m) pool.v.clear();
        double *R = pool.get(0, (int)m), *Z = pool.get(1, (int)m), *P = pool.get(2, (int)m), *AP = pool.get(3, (int)m);
        KState *st = S.st.p;
        int *ad = S.all_done.p;
        const RedSlot sl = S.slot();
        if (M.type != PC_NONE && M.type != PC_JACOBI) BP.ensure(n, k, s);  // before any capture
        const int G = batch_grid(), TB = batch_block(k);
        k_bspmv<BS_RESID><<<G, TB, 0, s>>>(n, k, A.rp, A.ci, A.v, X, R, B, st, ad, sl);
        batch_apply(M, BP, k, R, Z, ad, s);
        k_bpcg<0><<<G, TB, 0, s>>>(n, k, st, ad, X, R, Z, P, AP, sl);
        check_launch();
        if (launches) *launches += 5;
        auto body = [&]() {
            k_bspmv<BS_DOT_SIGMA><<<G, TB, 0, s>>>(n, k, A.rp, A.ci, A.v, P, AP, P, st, ad, sl);
            k_bpcg<1><<<G, TB, 0, s>>>(n, k, st, ad, X, R, Z, P, AP, sl);
            batch_apply(M, BP, k, R, Z, ad, s);
            k_bpcg<2><<<G, TB, 0, s>>>(n, k, st, ad, X, R, Z, P, AP, sl);
            k_bpcg<3><<<G, TB, 0, s>>>(n, k, st, ad, X, R, Z, P, AP, sl);
            check_launch();
        };
        // capture a chunk of iterations into a graph and replay it until
        // every column is done (the host polls all_done one chunk behind)
        std::vector<const void *> key{B, X, R, Z, P, AP, st, ad, &M, A.v, (const void *)(long)k,
                                      (const void *)(long)M.type};
        if (!gc.exec || gc.key != key) {
            gc.reset();
            cudaGraph_t g;
            XS_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeRelaxed));
            try {
                for (int r = 0; r < 8; r++) body();
            } catch (...) {
                cudaGraph_t junk;
                cudaStreamEndCapture(s, &junk);
                if (junk) cudaGraphDestroy(junk);
                throw;
            }
            XS_CUDA(cudaStreamEndCapture(s, &g));
            size_t nn = 0;
            cudaGraphGetNodes(g, nullptr, &nn);
            gc.nodes = nn;
            const cudaError_t e = cudaGraphInstantiate(&gc.exec, g, 0);
            cudaGraphDestroy(g);
            if (e != cudaSuccess) throw Status(XS_ERR_CUDA);
            gc.key = key;
        }
        gc.ensure_polling();
        int maxit = 0;
        for (int c = 0; c < k; c++) maxit = std::max(maxit, S.h[c].maxiter);
        const int max_launches = maxit / 8 + 3;
        bool stop = false;
        for (int l = 0; l < max_launches && !stop; l++) {
            XS_CUDA(cudaGraphLaunch(gc.exec, s));
            if (launches) *launches += (long long)gc.nodes;
            XS_CUDA(cudaMemcpyAsync(&gc.hflag[l & 1], ad, sizeof(int), cudaMemcpyDeviceToHost, s));
            XS_CUDA(cudaEventRecord(gc.ev[l & 1], s));
            if (l > 0) {
                XS_CUDA(cudaEventSynchronize(gc.ev[(l - 1) & 1]));
                if (gc.hflag[(l - 1) & 1]) stop = true;
            }
        }
        XS_CUDA(cudaStreamSynchronize(s));
    }
};

// ---------------------------------------------------------------- layout and gradients
// Y[i*k + c] = X[c*n + i]  (k vectors one after another -> interleaved)
static __global__ void k_interleave(int n, int k, const double *__restrict__ X, double *__restrict__ Y)
{
    const long m = (long)n * k;
    for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < m; q += (long)gridDim.x * blockDim.x) {
        const int c = (int)(q / n), i = (int)(q % n);
        Y[(long)i * k + c] = X[q];
    }
}
// X[c*n + i] = Y[i*k + c]
static __global__ void k_deinterleave(int n, int k, const double *__restrict__ Y, double *__restrict__ X)
{
    const long m = (long)n * k;
    for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < m; q += (long)gridDim.x * blockDim.x) {
        const int c = (int)(q / n), i = (int)(q % n);
        X[q] = Y[(long)i * k + c];
    }
}
// per column c: dLdb_c = lambda_c ; dLdA_c[e] = -lambda_c[i] * x_c[col(e)]
// (lambda and x interleaved; outputs one vector after another)
static __global__ void k_adjoint_grad_multi(int n, int k, long nnz, const int *__restrict__ rp, const int *__restrict__ ci,
                                     const double *__restrict__ lam, const double *__restrict__ x, double *dLdb,
                                     double *dLdA)
{
    const long m = (long)n * k;
    for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < m; q += (long)gridDim.x * blockDim.x) {
        const int c = (int)(q / n), i = (int)(q % n);
        const double li = lam[(long)i * k + c];
        if (dLdb) dLdb[q] = li;
        if (dLdA) {
            const double mli = -li;
            for (int e = rp[i]; e < rp[i + 1]; e++) dLdA[(long)c * nnz + e] = mli * __ldg(x + (long)ci[e] * k + c);
        }
    }
}

// per-handle state of the batched solves
struct BatchRuntime {
    BatchPcg pcg, pcg_t;    // forward and transposed (adjoint) iterations
    BatchPrecond bp, bpt;   // readiness buffers of the batched triangular solves
    BatchState S;
    DBuf<double> bB, bX, bY, tmp, gb, gA;
    std::vector<int> iters;  // per column, last batched solve
};

}  // namespace xs
