// BiCGSTAB with a Jacobi-sweep ILU apply as ONE persistent kernel.
//
// The graph-replayed iteration (BicgRun) is 11 kernels per iteration once
// the vector updates are fused into the sweep passes: at 128^3 with FP32
// vectors most of them move 10-40 MB and last 10-20 us, so the launch, ramp
// and tail of every kernel are a large share of the iteration.  Here the
// whole inner solve is one cooperative launch: every CTA stays resident, the
// phases of an iteration (the sweep passes of both applies, the two SpMVs
// with their dot products, the solution/residual update) run one after
// another separated by grid barriers, and the iteration loops on the device
// until the KState says done.  Each phase is the same device code as its
// stand-alone kernel (ell_rows, sweep_chunk, the SpMV epilogues, the vector
// operations and their finalizers), so the arithmetic per element is the
// same; only the grid, and therefore the order of the block partials of the
// dot products, differs.
//
// Requirements (else the graph path runs): BiCGSTAB, an ILU-family
// preconditioner applied by k >= 2 Jacobi sweeps, A and both triangles in
// diagonal-slot ELL storage with at most 8 slots (1-byte row masks).
//
// Every grid barrier waits at most BARRIER_LIMIT_NS; a barrier that runs out
// records DEV_TRSV_TIMEOUT and ends the solve (co-residency of all CTAs is
// guaranteed by the cooperative launch, so this is a safety net only).
#define XS_COHERENT_VECTOR_LOADS 1  // phases read vectors that earlier phases of the same launch wrote
#include "xs_internal.cuh"
#include "xs_spmv.cuh"
#include "xs_trsv.cuh"
#include "xs_precond.cuh"
#include "xs_krylov.cuh"
#include "xs_solvers.cuh"
#include "xs_persist.cuh"


namespace xs {

constexpr unsigned long long BARRIER_LIMIT_NS = 2000000000ull;

struct GridBar {
    unsigned *count;
    unsigned *gen;
};

// all CTAs of the grid meet; false if the wait ran out (recorded in *err)
__device__ __forceinline__ bool grid_barrier(GridBar b, int *err)
{
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        s_ok = 1;
        const unsigned g = ld_acquire((const int *)b.gen);
        __threadfence();
        if (atomicAdd(b.count, 1u) == gridDim.x - 1) {
            *b.count = 0u;
            __threadfence();
            st_release((int *)b.gen, (int)(g + 1));
        } else {
            const unsigned long long t0 = gtimer();
            unsigned ns = 32;
            while ((unsigned)ld_acquire((const int *)b.gen) == g) {
                __nanosleep(ns);
                if (ns < 256) ns <<= 1;
                if (gtimer() - t0 > BARRIER_LIMIT_NS) {
                    atomicOr(err, DEV_TRSV_TIMEOUT);
                    s_ok = 0;
                    break;
                }
            }
        }
    }
    __syncthreads();
    return s_ok != 0;
}

// ---------------------------------------------------------------- phases
// one sweep pass of a diagonal-slot triangle (body of k_trsv_sweep_ell)
template <typename VT, typename FT, typename DT, bool UPPER, bool FIRST2, class Src>
__device__ __forceinline__ void phase_sweep(int n, int w, const uint8_t *__restrict__ masks, const int *s_off,
                                            const FT *__restrict__ ev, const DT *__restrict__ dinv, const Src &x,
                                            const VT *__restrict__ yin, VT *__restrict__ yout)
{
    using CT = uint8_t;
    constexpr int R = ell_rows_for<FT>();
    const long ld = ell_ld(n);
    Src xs = x;
    xs.load();  // scalars the source needs (written before the barrier that began this phase)
    for (int i0 = (blockIdx.x * blockDim.x + threadIdx.x) * R; i0 < n; i0 += gridDim.x * blockDim.x * R) {
        VT acc[R];
#pragma unroll
        for (int q = 0; q < R; q++) {
            const int i = i0 + q;
            if (R == 1 || i < n) {
                const VT xi = xs.at(i);
                xs.put(i, xi);
                acc[q] = UPPER ? (VT)(xi * (VT)dinv[i]) : xi;
            } else {
                acc[q] = (VT)0;
            }
        }
        const CT *cp = masks + i0;
        const FT *vp = ev + i0;
        CT mask[R];
        ld_vec<R>(cp, mask);
        constexpr int CH = ell_chunk_for<FT>();
        for (int k0 = 0; k0 < w; k0 += CH) {
            const int m = min(CH, w - k0);
#define XS_PSWEEP(CC) \
    sweep_chunk<CC, R, VT, FT, DT, CT, UPPER, FIRST2, Src>(cp, vp, ld, i0, n, k0, mask, s_off, dinv, xs, yin, acc)
            if (m == CH) XS_PSWEEP(CH);
            else if (CH > 7 && m == 7) XS_PSWEEP(7);
            else if (CH > 6 && m == 6) XS_PSWEEP(6);
            else if (CH > 5 && m == 5) XS_PSWEEP(5);
            else if (CH > 4 && m == 4) XS_PSWEEP(4);
            else if (CH > 3 && m == 3) XS_PSWEEP(3);
            else if (CH > 2 && m == 2) XS_PSWEEP(2);
            else XS_PSWEEP(1);
#undef XS_PSWEEP
        }
#pragma unroll
        for (int q = 0; q < R; q++)
            if (R == 1 || i0 + q < n) yout[i0 + q] = acc[q];
    }
}

// diagonal-slot ELL SpMV with an epilogue and its reduction (body of k_ell_spmv)
template <typename VT, typename MT, class Epi>
__device__ __forceinline__ void phase_spmv(const EllArgs<MT, uint8_t> &A, const int *s_off, const VT *__restrict__ x,
                                           VT *__restrict__ y, const Epi &epi, RedSlot slot)
{
    constexpr int KK = Epi::K > 0 ? Epi::K : 1;
    constexpr int R = ell_rows_for<MT>();
    __shared__ double tot[KK];
    double acc[KK];
#pragma unroll
    for (int k = 0; k < KK; k++) acc[k] = 0.0;
    const int n = A.n;
    using AT = EllAcc<VT, MT>;
    for (int r0 = (blockIdx.x * blockDim.x + threadIdx.x) * R; r0 < n; r0 += gridDim.x * blockDim.x * R) {
        AT sum[R];
#pragma unroll
        for (int q = 0; q < R; q++) sum[q] = (AT)0;
        ell_rows<R, VT, MT, uint8_t, AT>(A.ci + r0, A.v + r0, A.w, A.ld, x, r0, n, s_off, sum);
#pragma unroll
        for (int q = 0; q < R; q++) {
            const int r = r0 + q;
            if (R == 1 || r < n) {
                VT o = epi.out(r, (double)sum[q]);
                y[r] = o;
                if (Epi::K > 0) epi.acc(r, (double)o, acc);
            }
        }
    }
    if (Epi::K > 0) {
        if (block_reduce_publish<KK>(acc, slot, tot)) {
            if (threadIdx.x == 0) epi.finalize(tot);
        }
    }
}

// vector operation with its reduction (body of k_vecop)
template <class Op>
__device__ __forceinline__ void phase_vecop(Op o, RedSlot slot)
{
    constexpr int KK = Op::K > 0 ? Op::K : 1;
    __shared__ double tot[KK];
    o.load();
    double acc[KK];
#pragma unroll
    for (int k = 0; k < KK; k++) acc[k] = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < o.n; i += gridDim.x * blockDim.x) o.elem(i, acc);
    if (Op::K > 0) {
        if (block_reduce_publish<KK>(acc, slot, tot)) {
            if (threadIdx.x == 0) o.finalize(tot);
        }
    }
}

// ---------------------------------------------------------------- the kernel
template <typename VT, typename FT>
struct PersistBicgArgs {
    int n, sweeps;
    EllArgs<VT, uint8_t> A;  // VT values: the FP32 copy with FP32 vectors
    int wl, wu;
    const uint8_t *ml, *mu;
    const int *offl, *offu;
    const FT *evl, *evu;
    const VT *dinv;  // natural order
    VT *r, *rhat, *p, *p2, *u, *s, *v, *z1, *z2, *x;
    VT *ta, *tb;  // sweep temporaries
    KState *st;
    RedSlot slot;
    GridBar bar;
    int max_iters;  // iterations this launch may run
};

// z = M^{-1} (first pass from src): L passes 2..k into ta/tb, then U passes
// ending in z (the same pass sequence as PrecondDev::apply_sweeps)
template <typename VT, typename FT, class Src>
__device__ __forceinline__ bool persist_apply(const PersistBicgArgs<VT, FT> &P, const int *offl, const int *offu,
                                              const Src &src, const VT *x_after, VT *z)
{
    const int n = P.n, k = P.sweeps;
    VT *cur = P.ta, *other = P.tb;
    phase_sweep<VT, FT, VT, false, true, Src>(n, P.wl, P.ml, offl, P.evl, nullptr, src, nullptr, cur);
    if (!grid_barrier(P.bar, &P.st->err)) return false;
    for (int t = 3; t <= k; t++) {
        phase_sweep<VT, FT, VT, false, false, SrcVec<VT>>(n, P.wl, P.ml, offl, P.evl, nullptr, SrcVec<VT>{x_after},
                                                         cur, other);
        if (!grid_barrier(P.bar, &P.st->err)) return false;
        VT *tmp = cur; cur = other; other = tmp;
    }
    const VT *yv = cur;
    const int passes = k - 1;
    VT *b0 = (passes % 2 == 1) ? z : other, *b1 = (passes % 2 == 1) ? other : z;
    phase_sweep<VT, FT, VT, true, true, SrcVec<VT>>(n, P.wu, P.mu, offu, P.evu, P.dinv, SrcVec<VT>{yv}, nullptr, b0);
    if (!grid_barrier(P.bar, &P.st->err)) return false;
    for (int t = 1; t < passes; t++) {
        VT *in = (t & 1) ? b0 : b1, *out = (t & 1) ? b1 : b0;
        phase_sweep<VT, FT, VT, true, false, SrcVec<VT>>(n, P.wu, P.mu, offu, P.evu, P.dinv, SrcVec<VT>{yv}, in, out);
        if (!grid_barrier(P.bar, &P.st->err)) return false;
    }
    return true;
}

template <typename VT, typename FT>
__global__ void __launch_bounds__(256, 4) k_persist_bicgstab(PersistBicgArgs<VT, FT> P)
{
    __shared__ int s_offa[ELL_DIA_MAX], s_offl[ELL_DIA_MAX], s_offu[ELL_DIA_MAX];
    if (threadIdx.x < (unsigned)P.A.w) s_offa[threadIdx.x] = P.A.doff[threadIdx.x];
    if (threadIdx.x < (unsigned)P.wl) s_offl[threadIdx.x] = P.offl[threadIdx.x];
    if (threadIdx.x < (unsigned)P.wu) s_offu[threadIdx.x] = P.offu[threadIdx.x];
    __syncthreads();
    KState *st = P.st;
    const int n = P.n;
    int parity = *(volatile int *)&st->pbuf;  // which p buffer holds p
    for (int it = 0; it < P.max_iters; it++) {
        if (*(volatile int *)&st->done) break;  // read after a barrier: the same value in every CTA
        VT *pin = parity ? P.p2 : P.p, *pout = parity ? P.p : P.p2;
        // p = omega (p - alpha u) + r inside the first L pass; z1 = M^{-1} p
        if (!persist_apply(P, s_offl, s_offu, SrcBicgP<VT>{pin, P.u, P.r, pout, st, (VT)0, (VT)0, parity ? 0 : 1},
                           pout, P.z1))
            return;
        parity ^= 1;
        // u = A z1 ; (rhat, u) -> gama
        phase_spmv<VT, VT>(P.A, s_offa, P.z1, P.u, EpiDot1<VT>{st, P.rhat, 0, M_BICG_GAMA}, P.slot);
        if (!grid_barrier(P.bar, &st->err)) return;
        if (*(volatile int *)&st->done) break;
        // s = r - gama u inside the first L pass; z2 = M^{-1} s
        if (!persist_apply(P, s_offl, s_offu, SrcBicgS<VT>{P.r, P.u, P.s, st, (VT)0}, P.s, P.z2)) return;
        // v = A z2 ; (s, v), (v, v) -> alpha
        phase_spmv<VT, VT>(P.A, s_offa, P.z2, P.v, EpiDot2<VT>{st, P.s, M_BICG_ALPHA}, P.slot);
        if (!grid_barrier(P.bar, &st->err)) return;
        if (*(volatile int *)&st->done) break;
        // x += gama z1 + alpha z2 ; r = s - alpha v ; convergence, beta, omega
        phase_vecop(OpBicgX<VT>{n, st, P.x, P.r, P.z1, P.z2, P.s, P.v, P.rhat, (VT)0, (VT)0}, P.slot);
        if (!grid_barrier(P.bar, &st->err)) return;
    }
}

// whether the persistent iteration serves this operator and preconditioner
template <typename VT>
inline bool persist_ok(const Operator &A, const PrecondDev &M)
{
    if (!pc_triangular(M.type)) return false;
    if (M.trsv_mode < 2) return false;
    if (A.format != 1 || !A.ell_dia || A.ell_w > 8 || !A.emask8.p) return false;
    for (const TriDev *T : {&M.L, &M.U})
        if (T->ell_w <= 0 || !T->ell_dia || T->ell_w > 8 || !T->emask8.p) return false;
    if constexpr (std::is_same<VT, float>::value) return A.ev32.p != nullptr;
    return A.ev.p != nullptr;
}

}  // namespace xs

namespace xs {

template <typename VT, typename FT>
static void persist_launch(SolveCtx &c, PersistBicgArgs<VT, FT> P, unsigned *bar)
{
    int per = 0;
    XS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_persist_bicgstab<VT, FT>, 256, 0));
    if (per < 1) throw Status(XS_ERR_CUDA);
    const int grid = per * geom().sms;
    P.bar = GridBar{bar, bar + 1};
    XS_CUDA(cudaMemsetAsync(bar, 0, 2 * sizeof(unsigned), c.s));  // a barrier that ran out leaves it mid-way
    void *args[] = {&P};
    XS_CUDA(cudaLaunchCooperativeKernel((const void *)k_persist_bicgstab<VT, FT>, dim3(grid), dim3(256), args, 0,
                                        c.s));
    if (c.launches) *c.launches += 1;
}

template <typename VT, typename FT>
static void persist_run(SolveCtx &c, const PersistVectors<VT> &V, int max_iters, unsigned *bar)
{
    const Operator &A = *c.A;
    const PrecondDev &M = *c.M;
    PersistBicgArgs<VT, FT> P;
    P.n = c.n;
    P.sweeps = M.trsv_mode;
    if constexpr (std::is_same<VT, double>::value) {
        P.A = A.ell<double, uint8_t>();
        P.dinv = M.U.dinv64_nat.p;
        P.ta = M.tmp64a.p; P.tb = M.tmp64b.p;
    } else {
        P.A = A.ell<float, uint8_t>();
        P.dinv = M.U.dinv32_nat.p;
        P.ta = M.tmp32a.p; P.tb = M.tmp32b.p;
    }
    P.wl = M.L.ell_w; P.wu = M.U.ell_w;
    P.ml = M.L.emask8.p; P.mu = M.U.emask8.p;
    P.offl = M.L.doff.p; P.offu = M.U.doff.p;
    P.evl = M.L.evals<FT>(); P.evu = M.U.evals<FT>();
    if (!P.evl || !P.evu || !P.dinv || !P.ta || !P.tb) throw Status(XS_ERR_ORDER);
    P.r = V.r; P.rhat = V.rhat; P.p = V.p; P.p2 = V.p2; P.u = V.u; P.s = V.s; P.v = V.v; P.z1 = V.z1; P.z2 = V.z2;
    P.x = V.x;
    P.st = c.W->st.p;
    P.slot = c.W->slot();
    P.max_iters = max_iters;
    persist_launch<VT, FT>(c, P, bar);
}

template <typename VT>
static bool persist_dispatch(SolveCtx &c, const PersistVectors<VT> &V, int max_iters, unsigned *bar)
{
    if (!persist_tuning().enabled || !persist_ok<VT>(*c.A, *c.M)) return false;
    if constexpr (std::is_same<VT, double>::value) {
        persist_run<double, double>(c, V, max_iters, bar);
    } else {
        switch (c.M->factor_prec) {
        case FP_BF16: persist_run<float, __nv_bfloat16>(c, V, max_iters, bar); break;
        case FP_F16: persist_run<float, __half>(c, V, max_iters, bar); break;
        default: persist_run<float, float>(c, V, max_iters, bar); break;
        }
    }
    return true;
}

bool persist_bicgstab(SolveCtx &c, const PersistVectors<float> &V, int max_iters, unsigned *bar)
{
    return persist_dispatch<float>(c, V, max_iters, bar);
}
bool persist_bicgstab(SolveCtx &c, const PersistVectors<double> &V, int max_iters, unsigned *bar)
{
    return persist_dispatch<double>(c, V, max_iters, bar);
}

}  // namespace xs
