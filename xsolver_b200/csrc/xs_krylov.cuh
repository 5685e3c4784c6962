// Krylov iteration bodies with device-resident scalars.
//
// The reference drives every iteration from the host and reads each dot
// product back (rocBLAS/cuBLAS ddot into a host double: DeviceVector.h:139-153,
// cuda/mpicudasolver-C-v1.cu), i.e. >= 5 host synchronisations per BiCGSTAB
// iteration.  Here one iteration is a short fixed sequence of fused kernels:
// every dot product is accumulated inside the kernel that produces or reads
// its operands (SpMV epilogue or vector update), reduced deterministically,
// and the last block computes the next scalars (alpha, beta, omega, ...) and
// the convergence test directly into KState.  Iterations are captured once
// into a CUDA graph (a chunk of several iterations) and replayed; every
// kernel exits immediately once KState::done is set, and the host polls the
// done flag once per chunk, one chunk behind, so the GPU never idles.
//
// Scalar recurrences follow the reference loops operation for operation
// (intel/mpisolver-C-v1.cpp with small = 1e-20), so the FP64 residual
// history matches the CPU reference to rounding:
//   cgm       (PCG)                      :193-272   (= hip/Solver/xsolver_cg.cpp:17-74)
//   cg        (CG on M^-1 A, left)        :26-102
//   bicgstab  (right preconditioned)      :365-482   (x updated with M^-1 p, M^-1 s as
//                                                     hip/Solver/xsolver_bicgstab.cpp:20-124)
//   gcr/igcr  (left, CGS / MGS)           :685-931
//   hip igcr  (right, MGS)                hip/Solver/xsolver_igcr.cpp:29-108
//   gmres     (left, MGS, Givens)         :933-1087, fgmres (right) :1089-1247
#pragma once
#include "xs_internal.cuh"
#include "xs_spmv.cuh"
#include "xs_precond.cuh"

namespace xs {

constexpr double KSMALL = 1e-20;

// 16 bytes of consecutive elements at a 16-byte aligned address
template <typename T, int W>
__device__ __forceinline__ void ld16(const T *p, T (&o)[W])
{
    static_assert(W * sizeof(T) == 16, "16-byte vector");
    const uint4 u = *reinterpret_cast<const uint4 *>(p);
    memcpy(o, &u, 16);
}
template <typename T, int W>
__device__ __forceinline__ void ldg16(const T *p, T (&o)[W])  // read-only for the whole launch
{
    static_assert(W * sizeof(T) == 16, "16-byte vector");
    const uint4 u = __ldg(reinterpret_cast<const uint4 *>(p));
    memcpy(o, &u, 16);
}
template <typename T, int W>
__device__ __forceinline__ void st16(T *p, const T (&v)[W])
{
    static_assert(W * sizeof(T) == 16, "16-byte vector");
    uint4 u;
    memcpy(&u, v, 16);
    *reinterpret_cast<uint4 *>(p) = u;
}
inline bool aligned16(std::initializer_list<const void *> ps)
{
    for (const void *p : ps)
        if (reinterpret_cast<uintptr_t>(p) % 16) return false;
    return true;
}

// ---------------------------------------------------------------- generic vector-op kernel
// An op may also provide elem_v(i, acc) for Op::V consecutive elements from
// a V-aligned i with one 16-byte access per vector (used when its vec_ok
// says every vector is 16-byte aligned): a thread then keeps V elements of
// each vector in flight instead of one.
template <class Op, class = void>
struct OpVecWidth {
    static constexpr int V = 1;
};
template <class Op>
struct OpVecWidth<Op, std::void_t<decltype(Op::V)>> {
    static constexpr int V = Op::V;
};

template <class Op>
__global__ void __launch_bounds__(256, 8) k_vecop(Op op, RedSlot slot)
{
    constexpr int KK = Op::K > 0 ? Op::K : 1;
    __shared__ double tot[KK];
    pdl_trigger();
    pdl_wait();
    if (op.st->done) return;
    Op o = op;
    o.load();
    double acc[KK];
#pragma unroll
    for (int k = 0; k < KK; k++) acc[k] = 0.0;
    const int tid = blockIdx.x * blockDim.x + threadIdx.x, stride = gridDim.x * blockDim.x;
    int i0 = 0;
    if constexpr (OpVecWidth<Op>::V > 1) {
        constexpr int V = OpVecWidth<Op>::V;
        if (o.vec_ok) {
            const int nv = o.n / V;
            for (int j = tid; j < nv; j += stride) o.elem_v(j * V, acc);
            i0 = nv * V;
        }
    }
    for (int i = i0 + tid; i < o.n; i += stride) o.elem(i, acc);
    if (Op::K > 0) {
        if (block_reduce_publish<KK>(acc, slot, tot)) {
            if (threadIdx.x == 0) o.finalize(tot);
        }
    }
}

template <class Op>
inline void vecop(const Op &op, RedSlot slot, cudaStream_t s)
{
    launch_pdl(k_vecop<Op>, dim3(geom().red_grid), dim3(256), 0, s, op, slot);
}

// single-thread scalar step
template <class F>
__global__ void k_scalar(F f)
{
    f();
}

// convergence bookkeeping shared by all methods (last block, thread 0)
//   resl: new residual norm of the method; writes hist / hist_rel, advances
//   iter, sets done.  Returns true if iteration continues.
__device__ inline bool record_and_test(KState *st, double resl)
{
    const double rsm = resl / (st->res0 + KSMALL);
    const int it = st->iter;
    st->rnorm = resl;
    if (st->hist) st->hist[it + 1] = resl;
    if (st->hist_rel) st->hist_rel[it] = rsm;
    st->iter = it + 1;
    if (!isfinite(resl)) {
        st->err |= DEV_NAN;
        st->done = 3;
        return false;
    }
    if (rsm < st->tol || resl <= st->abstol) {
        st->done = 1;
        return false;
    }
    if (st->iter >= st->maxiter) {
        st->done = 2;
        return false;
    }
    return true;
}

__device__ inline void init_record(KState *st, double res0)
{
    st->res0 = res0;
    st->rnorm = res0;
    st->iter = 0;
    if (st->hist) st->hist[0] = res0;
    if (!isfinite(res0)) {
        st->err |= DEV_NAN;
        st->done = 3;
    } else if (res0 == 0.0 || res0 <= st->abstol || st->maxiter <= 0) {
        st->done = 1;
    } else {
        st->done = 0;
    }
}

// ---------------------------------------------------------------- SpMV epilogues with state
// y = A x;  acc0 += w[r] * y   (w may be y's own partner vector)
template <typename VT>
struct EpiDot1 {
    static constexpr int K = 1;
    KState *st;
    const VT *w;
    int slot_out;  // sc[slot_out] = dot
    int mode;      // finalize action (method specific)
    __device__ bool active() const { return st->done == 0; }
    __device__ VT out(int, double ax) const { return (VT)ax; }
    __device__ void acc(int r, double y, double (&a)[1]) const { a[0] += (double)w[r] * y; }
    __device__ void finalize(const double *tot) const;
};

// y = A x; acc0 += w0[r]*y, acc1 += y*y
template <typename VT>
struct EpiDot2 {
    static constexpr int K = 2;
    KState *st;
    const VT *w0;
    int mode;
    __device__ bool active() const { return st->done == 0; }
    __device__ VT out(int, double ax) const { return (VT)ax; }
    __device__ void acc(int r, double y, double (&a)[2]) const
    {
        a[0] += y * (double)w0[r];
        a[1] += y * y;
    }
    __device__ void finalize(const double *tot) const;
};

// finalize modes
enum EpiMode {
    M_CGM_SIGMA = 1,      // alpha = tao/(sigma+small); taoo = tao
    M_BICG_GAMA = 2,      // gama = beta/(tmp+small)
    M_BICG_ALPHA = 3,     // alpha = t0/(t1+small)
    M_CG_SIGMA = 4,       // cg (left): alpha = taoo/(sigma+small)
    M_STORE = 5,          // sc[slot_out] = dot
    M_IBICG_NU = 6        // ibicgstab: nu = dot; sigma = mu - omega nu
};

// slot layout
enum {
    S_TAO = 0, S_TAOO, S_ALPHA, S_BETA, S_SIGMA, S_OMEGA, S_GAMA, S_BETO, S_T0, S_T1, S_TMP, S_RES0SQ,
    S_GCR_T0 = 12, S_GCR_T1, S_GCR_INV, S_GCR_COEF,
    S_H = 16  // GCR alpha[] (classical GS) stored from here (up to 32)
};
// ibicgstab scalars (GCR's slots from 16 on are free in this method)
enum {
    IB_ALPHA = 16, IB_ALPHAO, IB_ROU, IB_ROUO, IB_OMEGA, IB_PI, IB_TAU, IB_MU, IB_FAI, IB_SIGMA, IB_DELTA, IB_BETA,
    IB_TMP1, IB_TMP2, IB_THETA, IB_KAPPA, IB_NU
};

template <typename VT>
__device__ void EpiDot1<VT>::finalize(const double *tot) const
{
    double d = tot[0];
    if (mode == M_CGM_SIGMA) {
        st->sc[S_SIGMA] = d;
        st->sc[S_ALPHA] = st->sc[S_TAO] / (d + KSMALL);
    } else if (mode == M_CG_SIGMA) {
        st->sc[S_SIGMA] = d;
        st->sc[S_ALPHA] = st->sc[S_TAOO] / (d + KSMALL);
    } else if (mode == M_BICG_GAMA) {
        st->sc[S_TMP] = d;
        st->sc[S_GAMA] = st->sc[S_BETA] / (d + KSMALL);
    } else if (mode == M_IBICG_NU) {
        st->sc[IB_NU] = d;
        st->sc[IB_SIGMA] = st->sc[IB_MU] - st->sc[IB_OMEGA] * d;
    } else {
        st->sc[slot_out] = d;
    }
    if (!isfinite(d)) {
        st->err |= DEV_BREAKDOWN;
        st->done = 3;
    }
}
template <typename VT>
__device__ void EpiDot2<VT>::finalize(const double *tot) const
{
    if (mode == M_BICG_ALPHA) {
        st->sc[S_T0] = tot[0];
        st->sc[S_T1] = tot[1];
        st->sc[S_ALPHA] = tot[0] / (tot[1] + KSMALL);
    }
    if (!isfinite(tot[0]) || !isfinite(tot[1])) {
        st->err |= DEV_BREAKDOWN;
        st->done = 3;
    }
}

// y = A x, skipped once the solve is done
template <typename VT>
struct EpiActive {
    static constexpr int K = 0;
    KState *st;
    __device__ bool active() const { return st->done == 0; }
    __device__ VT out(int, double ax) const { return (VT)ax; }
    __device__ void acc(int, double, double (&)[1]) const {}
    __device__ void finalize(const double *) const {}
};
// y = b - A x, skipped once the solve is done
template <typename VT>
struct EpiResidActive {
    static constexpr int K = 0;
    KState *st;
    const VT *b;
    __device__ bool active() const { return st->done == 0; }
    __device__ VT out(int r, double ax) const { return (VT)((double)b[r] - ax); }
    __device__ void acc(int, double, double (&)[1]) const {}
    __device__ void finalize(const double *) const {}
};

// r = b - A x, acc0 += r*r, acc1 += r*w (w optional)
template <typename VT>
struct EpiResid {
    static constexpr int K = 1;
    KState *st;
    const VT *b;
    __device__ bool active() const { return true; }
    __device__ VT out(int r, double ax) const { return (VT)((double)b[r] - ax); }
    __device__ void acc(int r, double y, double (&a)[1]) const { a[0] += y * y; }
    __device__ void finalize(const double *tot) const { st->sc[S_RES0SQ] = tot[0]; }
};

// ---------------------------------------------------------------- vector ops
// Each op: fields n, st; load() reads scalars; elem(i, acc); finalize(tot).

// PCG init: acc0 = r.r, acc1 = r.z ; p = z
template <typename VT>
struct OpCgmInit {
    static constexpr int K = 2;
    int n;
    KState *st;
    const VT *r, *z;
    VT *p;
    __device__ void load() {}
    __device__ void elem(int i, double (&a)[2]) const
    {
        const VT ri = r[i], zi = z[i];
        a[0] += (double)ri * (double)ri;
        a[1] += (double)ri * (double)zi;
        p[i] = zi;
    }
    __device__ void finalize(const double *t) const
    {
        st->sc[S_TAO] = t[1];
        init_record(st, sqrt(t[0]));
    }
};

// x += alpha p ; r -= alpha Ap ; acc0 = r.r (convergence)
template <typename VT>
struct OpCgmUpdate {
    static constexpr int K = 1;
    int n;
    KState *st;
    VT *x, *r;
    const VT *p, *Ap;
    VT alpha;
    __device__ void load() { alpha = (VT)st->sc[S_ALPHA]; }
    __device__ void elem(int i, double (&a)[1]) const
    {
        const VT minalpha = -alpha;
        x[i] = x[i] + alpha * p[i];
        const VT ri = r[i] + minalpha * Ap[i];
        r[i] = ri;
        a[0] += (double)ri * (double)ri;
    }
    __device__ void finalize(const double *t) const
    {
        // pcg tests convergence after the p update; the value is the same
        // r.r, so test here and skip the rest of the iteration when done
        record_and_test(st, sqrt(t[0]));
    }
};

// tao = r.z ; beta = tao/(taoo + small)  then p = beta p + z  (two ops: the
// dot must complete before p can be updated)
template <typename VT>
struct OpDotRZ {
    static constexpr int K = 1;
    int n;
    KState *st;
    const VT *r, *z;
    __device__ void load() {}
    __device__ void elem(int i, double (&a)[1]) const { a[0] += (double)r[i] * (double)z[i]; }
    __device__ void finalize(const double *t) const
    {
        st->sc[S_TAOO] = st->sc[S_TAO];
        st->sc[S_TAO] = t[0];
        st->sc[S_BETA] = t[0] / (st->sc[S_TAOO] + KSMALL);
        if (!isfinite(t[0])) { st->err |= DEV_BREAKDOWN; st->done = 3; }
    }
};
template <typename VT>
struct OpPUpdate {  // p = beta*p + z
    static constexpr int K = 0;
    int n;
    KState *st;
    VT *p;
    const VT *z;
    VT beta;
    __device__ void load() { beta = (VT)st->sc[S_BETA]; }
    __device__ void elem(int i, double (&)[1]) const
    {
        const VT t = beta * p[i];
        p[i] = t + z[i];
    }
    __device__ void finalize(const double *) const {}
};

// ---- left CG (cg): res = M^-1(b - Ax) ; res0 = ||res||, taoo = res0^2 ; p = res
template <typename VT>
struct OpCgInit {
    static constexpr int K = 1;
    int n;
    KState *st;
    const VT *r;
    VT *p;
    __device__ void load() {}
    __device__ void elem(int i, double (&a)[1]) const
    {
        const VT ri = r[i];
        a[0] += (double)ri * (double)ri;
        p[i] = ri;
    }
    __device__ void finalize(const double *t) const
    {
        st->sc[S_TAOO] = t[0];
        init_record(st, sqrt(t[0]));
    }
};
// x += alpha p ; r -= alpha q ; acc r.r ; then beta = tao/(taoo+small), taoo = tao
template <typename VT>
struct OpCgUpdate {
    static constexpr int K = 1;
    int n;
    KState *st;
    VT *x, *r;
    const VT *p, *q;
    VT alpha;
    __device__ void load() { alpha = (VT)st->sc[S_ALPHA]; }
    __device__ void elem(int i, double (&a)[1]) const
    {
        const VT minalpha = -alpha;
        x[i] = x[i] + alpha * p[i];
        const VT ri = r[i] + minalpha * q[i];
        r[i] = ri;
        a[0] += (double)ri * (double)ri;
    }
    __device__ void finalize(const double *t) const
    {
        const double tao = t[0];
        if (!record_and_test(st, sqrt(tao))) return;
        st->sc[S_BETA] = tao / (st->sc[S_TAOO] + KSMALL);
        st->sc[S_TAOO] = tao;
    }
};
template <typename VT>
struct OpCgP {  // p = beta*p + r
    static constexpr int K = 0;
    int n;
    KState *st;
    VT *p;
    const VT *r;
    VT beta;
    __device__ void load() { beta = (VT)st->sc[S_BETA]; }
    __device__ void elem(int i, double (&)[1]) const
    {
        const VT t = beta * p[i];
        p[i] = t + r[i];
    }
    __device__ void finalize(const double *) const {}
};

// ---- single-reduction CG variants (intel/mpisolver-C-v1.cpp:104-191 icg,
// :273-363 icgm): every dot product of an iteration is taken in one pass

// icg: sigma = p.q, rho = r.q, theta = q.q (q = M^-1 A p); then
// alpha = taoo/(sigma+small), tao = taoo - 2 alpha rho + alpha^2 theta,
// beta = tao/(taoo+small) (the reference computes tao and beta after its
// convergence test; they do not depend on it)
template <typename VT>
struct OpIcgDots {
    static constexpr int K = 3;
    int n;
    KState *st;
    const VT *p, *r, *q;
    __device__ void load() {}
    __device__ void elem(int i, double (&a)[3]) const
    {
        const double qi = (double)q[i];
        a[0] += (double)p[i] * qi;
        a[1] += (double)r[i] * qi;
        a[2] += qi * qi;
    }
    __device__ void finalize(const double *t) const
    {
        const double sigma = t[0], rho = t[1], theta = t[2];
        const double taoo = st->sc[S_TAOO];
        const double alpha = taoo / (sigma + KSMALL);
        const double tao = taoo - 2.0 * alpha * rho + alpha * alpha * theta;
        st->sc[S_SIGMA] = sigma;
        st->sc[S_ALPHA] = alpha;
        st->sc[S_TAO] = tao;
        st->sc[S_BETA] = tao / (taoo + KSMALL);
        if (!isfinite(sigma) || !isfinite(rho) || !isfinite(theta)) {
            st->err |= DEV_BREAKDOWN;
            st->done = 3;
        }
    }
};
// icg: x += alpha p ; r -= alpha q ; p = beta p + r (new r) ; acc r.r, the
// convergence test; taoo = tao while the iteration continues
template <typename VT>
struct OpIcgUpdate {
    static constexpr int K = 1;
    int n;
    KState *st;
    VT *x, *r, *p;
    const VT *q;
    VT alpha, beta;
    __device__ void load()
    {
        alpha = (VT)st->sc[S_ALPHA];
        beta = (VT)st->sc[S_BETA];
    }
    __device__ void elem(int i, double (&a)[1]) const
    {
        const VT minalpha = -alpha;
        const VT pi = p[i];
        x[i] = x[i] + alpha * pi;
        const VT ri = r[i] + minalpha * q[i];
        r[i] = ri;
        const VT t = beta * pi;
        p[i] = t + ri;
        a[0] += (double)ri * (double)ri;
    }
    __device__ void finalize(const double *t) const
    {
        if (!record_and_test(st, sqrt(t[0]))) return;
        st->sc[S_TAOO] = st->sc[S_TAO];
    }
};

// icgm: sigma = p.Ap, rho = r.q, fai = Ap.z, theta = q.Ap and r.r (the
// residual before this iteration's update, which the reference tests at the
// end of the iteration); alpha = tau/(sigma+small),
// tau' = tau - alpha fai - alpha rho + alpha^2 theta, beta = tau'/(tau+small)
template <typename VT>
struct OpIcgmDots {
    static constexpr int K = 5;
    int n;
    KState *st;
    const VT *p, *r, *q, *Ap, *z;
    __device__ void load() {}
    __device__ void elem(int i, double (&a)[5]) const
    {
        const double api = (double)Ap[i], qi = (double)q[i], ri = (double)r[i];
        a[0] += (double)p[i] * api;
        a[1] += ri * qi;
        a[2] += api * (double)z[i];
        a[3] += qi * api;
        a[4] += ri * ri;
    }
    __device__ void finalize(const double *t) const
    {
        const double sigma = t[0], rho = t[1], fai = t[2], theta = t[3];
        const double tauo = st->sc[S_TAO];
        const double alpha = tauo / (sigma + KSMALL);
        const double tau = tauo - alpha * fai - alpha * rho + alpha * alpha * theta;
        st->sc[S_SIGMA] = sigma;
        st->sc[S_ALPHA] = alpha;
        st->sc[S_TAO] = tau;
        st->sc[S_BETA] = tau / (tauo + KSMALL);
        st->sc[S_T0] = t[4];
        bool ok = true;
        for (int k = 0; k < 5; k++) ok = ok && isfinite(t[k]);
        if (!ok) {
            st->err |= DEV_BREAKDOWN;
            st->done = 3;
        }
    }
};
// icgm: x += alpha p ; r -= alpha Ap ; then the convergence test on the
// residual norm taken before the update (the reference tests after z and p
// are updated; those updates do not change x, so a converged solve may skip
// them)
template <typename VT>
struct OpIcgmUpdate {
    static constexpr int K = 1;  // no sum; K = 1 for the finalize step
    int n;
    KState *st;
    VT *x, *r;
    const VT *p, *Ap;
    VT alpha;
    __device__ void load() { alpha = (VT)st->sc[S_ALPHA]; }
    __device__ void elem(int i, double (&)[1]) const
    {
        const VT minalpha = -alpha;
        x[i] = x[i] + alpha * p[i];
        r[i] = r[i] + minalpha * Ap[i];
    }
    __device__ void finalize(const double *) const { record_and_test(st, sqrt(st->sc[S_T0])); }
};

// ---- single-reduction BiCGSTAB (intel/mpisolver-C-v1.cpp:484-683,
// right preconditioned: the iterate phi lives in the preconditioned space)
// scalar prologue of an iteration, in the reference's evaluation order
__device__ inline void ib_prologue(KState *st)
{
    double *c = st->sc;
    c[IB_ROUO] = c[IB_ROU];
    c[IB_ROU] = c[IB_FAI] - c[IB_OMEGA] * c[IB_MU];
    c[IB_DELTA] = (c[IB_ROU] * c[IB_ALPHA]) / (c[IB_ROUO] + KSMALL);
    c[IB_BETA] = c[IB_DELTA] / (c[IB_OMEGA] + KSMALL);
    c[IB_TAU] = c[IB_SIGMA] + c[IB_BETA] * c[IB_TAU] - c[IB_DELTA] * c[IB_PI];
    c[IB_ALPHAO] = c[IB_ALPHA];
    c[IB_ALPHA] = c[IB_ROU] / (c[IB_TAU] + KSMALL);
    c[IB_TMP1] = (c[IB_BETA] * c[IB_ALPHA]) / (c[IB_ALPHAO] + KSMALL);
    c[IB_TMP2] = c[IB_ALPHA] * c[IB_DELTA];
}
// start-up: tk += pk (tk = A M^-1 res, pk = A M^-1 A phi) ; reso = res ;
// qk = vk = zk = 0 ; fai = res.res, sigma = res.tk ; the scalars of
// iteration 0
template <typename VT>
struct OpIbInit {
    static constexpr int K = 2;
    int n;
    KState *st;
    const VT *res, *pk;
    VT *tk, *reso, *qk, *vk, *zk;
    __device__ void load() {}
    __device__ void elem(int i, double (&a)[2]) const
    {
        const VT ri = res[i];
        const VT ti = tk[i] + pk[i];
        tk[i] = ti;
        reso[i] = ri;
        qk[i] = (VT)0;
        vk[i] = (VT)0;
        zk[i] = (VT)0;
        a[0] += (double)ri * (double)ri;
        a[1] += (double)ri * (double)ti;
    }
    __device__ void finalize(const double *t) const
    {
        double *c = st->sc;
        c[IB_ALPHA] = 1.0; c[IB_ALPHAO] = 1.0; c[IB_ROU] = 1.0; c[IB_ROUO] = 1.0; c[IB_OMEGA] = 1.0;
        c[IB_PI] = 0.0; c[IB_TAU] = 0.0; c[IB_MU] = 0.0;
        c[IB_FAI] = t[0];
        c[IB_SIGMA] = t[1];
        init_record(st, sqrt(t[0]));
        ib_prologue(st);
    }
};
// vk = tk - omega pk + beta vk - delta qk ; sk = res - alpha vk ;
// zk = tmp1 zk + alpha res - tmp2 vk_old   (the reference's daxpy sequences)
template <typename VT>
struct OpIbV {
    static constexpr int K = 0;
    int n;
    KState *st;
    const VT *tk, *pk, *qk, *res;
    VT *vk, *sk, *zk;
    VT minomega, beta, mindelta, minalpha, alpha, tmp1, mintmp2;
    __device__ void load()
    {
        const double *c = st->sc;
        minomega = -(VT)c[IB_OMEGA];
        beta = (VT)c[IB_BETA];
        mindelta = -(VT)c[IB_DELTA];
        alpha = (VT)c[IB_ALPHA];
        minalpha = -alpha;
        tmp1 = (VT)c[IB_TMP1];
        mintmp2 = -(VT)c[IB_TMP2];
    }
    __device__ void elem(int i, double (&)[1]) const
    {
        const VT vko = vk[i], ri = res[i];
        VT v = tk[i];
        v = v + minomega * pk[i];
        v = v + beta * vko;
        v = v + mindelta * qk[i];
        vk[i] = v;
        sk[i] = ri + minalpha * v;
        VT z = tmp1 * zk[i];
        z = z + alpha * ri;
        zk[i] = z + mintmp2 * vko;
    }
    __device__ void finalize(const double *) const {}
};
// tk = tk - omega pk - alpha qk ; fai = reso.sk, pi = reso.qk, theta = sk.tk,
// kappa = tk.tk, mu = reso.tk ; omega = theta/(kappa+small)
template <typename VT>
struct OpIbT {
    static constexpr int K = 5;
    int n;
    KState *st;
    VT *tk;
    const VT *pk, *qk, *sk, *reso;
    VT minomega, minalpha;
    __device__ void load()
    {
        minomega = -(VT)st->sc[IB_OMEGA];
        minalpha = -(VT)st->sc[IB_ALPHA];
    }
    __device__ void elem(int i, double (&a)[5]) const
    {
        VT t = tk[i] + minomega * pk[i];
        const VT qi = qk[i];
        t = t + minalpha * qi;
        tk[i] = t;
        const double ro = (double)reso[i], si = (double)sk[i], td = (double)t;
        a[0] += ro * si;
        a[1] += ro * (double)qi;
        a[2] += si * td;
        a[3] += td * td;
        a[4] += ro * td;
    }
    __device__ void finalize(const double *t) const
    {
        double *c = st->sc;
        c[IB_FAI] = t[0];
        c[IB_PI] = t[1];
        c[IB_THETA] = t[2];
        c[IB_KAPPA] = t[3];
        c[IB_MU] = t[4];
        c[IB_OMEGA] = t[2] / (t[3] + KSMALL);
        bool ok = true;
        for (int k = 0; k < 5; k++) ok = ok && isfinite(t[k]);
        if (!ok) {
            st->err |= DEV_BREAKDOWN;
            st->done = 3;
        }
    }
};
// res = sk - omega tk ; phi = phi + zk + omega sk ; acc res.res, the
// convergence test; then the next iteration's scalars
template <typename VT>
struct OpIbR {
    static constexpr int K = 1;
    int n;
    KState *st;
    VT *res, *phi;
    const VT *sk, *tk, *zk;
    VT omega;
    __device__ void load() { omega = (VT)st->sc[IB_OMEGA]; }
    __device__ void elem(int i, double (&a)[1]) const
    {
        const VT minomega = -omega;
        const VT si = sk[i];
        const VT ri = si + minomega * tk[i];
        res[i] = ri;
        VT f = phi[i] + zk[i];
        phi[i] = f + omega * si;
        a[0] += (double)ri * (double)ri;
    }
    __device__ void finalize(const double *t) const
    {
        if (!record_and_test(st, sqrt(t[0]))) return;
        ib_prologue(st);
    }
};

// ---- BiCGSTAB
// init: rhat = r ; acc r.r ; then beta = r.rhat = r.r, omega, beto
template <typename VT>
struct OpBicgInit {
    static constexpr int K = 1;
    int n;
    KState *st;
    const VT *r;
    VT *rhat, *p, *u;
    __device__ void load() {}
    __device__ void elem(int i, double (&a)[1]) const
    {
        const VT ri = r[i];
        rhat[i] = ri;
        p[i] = (VT)0;
        u[i] = (VT)0;
        a[0] += (double)ri * (double)ri;
    }
    __device__ void finalize(const double *t) const
    {
        st->sc[S_ALPHA] = 1.0;
        st->sc[S_BETO] = 1.0;
        st->sc[S_GAMA] = 1.0;
        init_record(st, sqrt(t[0]));
        const double beta = t[0];
        st->sc[S_BETA] = beta;
        st->sc[S_OMEGA] = (beta * st->sc[S_GAMA]) / (st->sc[S_ALPHA] * st->sc[S_BETO] + KSMALL);
        st->sc[S_BETO] = beta;
    }
};
// p = r + omega (p - alpha u)
template <typename VT>
struct OpBicgP {
    static constexpr int K = 0;
    int n;
    KState *st;
    VT *p;
    const VT *r, *u;
    VT alpha, omega;
    __device__ void load()
    {
        alpha = (VT)st->sc[S_ALPHA];
        omega = (VT)st->sc[S_OMEGA];
    }
    __device__ void elem(int i, double (&)[1]) const
    {
        const VT minalpha = -alpha;
        VT t = p[i] + minalpha * u[i];
        t = omega * t;
        p[i] = t + r[i];
    }
    __device__ void finalize(const double *) const {}
};
// s = r - gama u
template <typename VT>
struct OpBicgS {
    static constexpr int K = 0;
    int n;
    KState *st;
    VT *s;
    const VT *r, *u;
    VT gama;
    __device__ void load() { gama = (VT)st->sc[S_GAMA]; }
    __device__ void elem(int i, double (&)[1]) const
    {
        const VT mingama = -gama;
        s[i] = r[i] + mingama * u[i];
    }
    __device__ void finalize(const double *) const {}
};
// p = omega (p - alpha u) + r formed inside the first L pass of the
// preconditioner apply that reads p (OpBicgP's operations, so the same
// values).  The pass reads p from one buffer and stores the new p into the
// other (its neighbours' old values are still being read), and records in
// KState::pbuf which buffer now holds p.
template <typename VT>
struct SrcBicgP {
    const VT *p, *u, *r;
    VT *pout;
    KState *st;
    VT alpha, omega;
    int which;
    __device__ void load()
    {
        alpha = (VT)st->sc[S_ALPHA];
        omega = (VT)st->sc[S_OMEGA];
        if (blockIdx.x == 0 && threadIdx.x == 0) st->pbuf = which;
    }
    __device__ VT at(int c) const
    {
        const VT minalpha = -alpha;
        VT t = XS_VLD(p + c) + minalpha * XS_VLD(u + c);
        t = omega * t;
        return t + XS_VLD(r + c);
    }
    __device__ void put(int i, VT v) const { pout[i] = v; }
};
// bring p back into the first buffer before a resumed run (its graph starts
// from there), then mark it home
template <typename VT>
__global__ void k_bicg_p_home(int n, const KState *st, VT *pa, const VT *pb)
{
    if (st->pbuf != 1) return;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) pa[i] = pb[i];
}
static __global__ void k_bicg_p_homed(KState *st) { st->pbuf = 0; }

// s = r - gama u formed inside the first L pass of the preconditioner
// apply that reads s (the same operations as OpBicgS, so the same values;
// the pass stores s for the later passes and the next kernels)
template <typename VT>
struct SrcBicgS {
    const VT *r, *u;
    VT *s;
    const KState *st;
    VT mingama;
    __device__ void load() { mingama = -(VT)st->sc[S_GAMA]; }
    __device__ VT at(int c) const { return XS_VLD(r + c) + mingama * XS_VLD(u + c); }
    __device__ void put(int i, VT v) const { s[i] = v; }
};

// x += gama z1 + alpha z2 ; r = s - alpha v ; acc r.r, r.rhat
template <typename VT>
struct OpBicgX {
    static constexpr int K = 2;
    static constexpr int V = 16 / (int)sizeof(VT);
    int n;
    KState *st;
    VT *x, *r;
    const VT *z1, *z2, *s, *v, *rhat;
    VT gama, alpha;
    bool vec_ok = false;
    __device__ void load()
    {
        gama = (VT)st->sc[S_GAMA];
        alpha = (VT)st->sc[S_ALPHA];
    }
    __device__ void elem(int i, double (&a)[2]) const
    {
        VT xi = x[i] + gama * z1[i];
        x[i] = xi + alpha * z2[i];
        const VT minalpha = -alpha;
        const VT ri = s[i] + minalpha * v[i];
        r[i] = ri;
        a[0] += (double)ri * (double)ri;
        a[1] += (double)ri * (double)rhat[i];
    }
    // the same arithmetic per element, V elements per 16-byte access
    __device__ void elem_v(int i, double (&a)[2]) const
    {
        VT xv[V], z1v[V], z2v[V], sv[V], vv[V], hv[V], rv[V];
        ld16(x + i, xv);
        ldg16(z1 + i, z1v);
        ldg16(z2 + i, z2v);
        ldg16(s + i, sv);
        ldg16(v + i, vv);
        ldg16(rhat + i, hv);
        const VT minalpha = -alpha;
#pragma unroll
        for (int q = 0; q < V; q++) {
            const VT xi = xv[q] + gama * z1v[q];
            xv[q] = xi + alpha * z2v[q];
            rv[q] = sv[q] + minalpha * vv[q];
            a[0] += (double)rv[q] * (double)rv[q];
            a[1] += (double)rv[q] * (double)hv[q];
        }
        st16(x + i, xv);
        st16(r + i, rv);
    }
    __device__ void finalize(const double *t) const
    {
        if (!record_and_test(st, sqrt(t[0]))) return;
        const double beta = t[1];
        st->sc[S_BETA] = beta;
        st->sc[S_OMEGA] = (beta * st->sc[S_GAMA]) / (st->sc[S_ALPHA] * st->sc[S_BETO] + KSMALL);
        st->sc[S_BETO] = beta;
        if (!isfinite(beta)) { st->err |= DEV_BREAKDOWN; st->done = 3; }
    }
};

// Residual replacement in a running BiCGSTAB (mixed-precision refinement
// without restart): r was just overwritten by the true residual, so
// beta = (rhat, r) is recomputed and the pending omega, which is
// proportional to beta, rescaled with it.
template <typename VT>
struct OpBicgRho {
    static constexpr int K = 1;
    int n;
    KState *st;
    const VT *rhat, *r;
    __device__ void load() {}
    __device__ void elem(int i, double (&a)[1]) const { a[0] += (double)rhat[i] * (double)r[i]; }
    __device__ void finalize(const double *t) const
    {
        const double old = st->sc[S_BETA], beta = t[0];
        st->sc[S_OMEGA] = st->sc[S_OMEGA] * (beta / (old + KSMALL));
        st->sc[S_BETA] = beta;
        st->sc[S_BETO] = beta;
        if (!isfinite(beta)) { st->err |= DEV_BREAKDOWN; st->done = 3; }
    }
};

// continue a stopped solve: new stopping test (relative to res0), the
// iteration cap raised by `more`, done cleared; scalars and history kept
static __global__ void k_resume_state(KState *st, double res0, double tol, int more)
{
    st->res0 = res0;
    st->tol = tol;
    st->maxiter = st->iter + more;
    st->done = 0;
}

// restarted methods: res0 = ||res|| ; beta = res0
template <typename VT>
struct OpGmInit {
    static constexpr int K = 1;
    int n;
    KState *st;
    const VT *r;
    __device__ void load() {}
    __device__ void elem(int i, double (&a)[1]) const { a[0] += (double)r[i] * (double)r[i]; }
    __device__ void finalize(const double *t) const
    {
        const double r0 = sqrt(t[0]);
        init_record(st, r0);
        st->sc[S_BETA] = r0;
    }
};

// mixed-precision refinement: outer FP64 residual state
struct OuterState {
    double rnorm;
    double rnorm0;
    double scale;      // ||r|| (the inner rhs is r / ||r||)
    double scale_inv;
};

// ---- generic small ops used by GCR / GMRES
// acc0 = x.y  (finalize stores into a device address)
template <typename VT>
struct OpDotTo {
    static constexpr int K = 1;
    int n;
    KState *st;
    const VT *x, *y;
    double *dst;
    __device__ void load() {}
    __device__ void elem(int i, double (&a)[1]) const { a[0] += (double)x[i] * (double)y[i]; }
    __device__ void finalize(const double *t) const { *dst = t[0]; }
};

// w = w - h*v_prev ; acc0 = w.v_next  (MGS step fused with the next dot);
// coefficient read from *hptr; if v_next == null, acc0 = w.w
template <typename VT>
struct OpMgsStep {
    static constexpr int K = 1;
    int n;
    KState *st;
    VT *w;
    const VT *vprev, *vnext;
    const double *hptr;
    double *dst;
    VT h;
    __device__ void load() { h = vprev ? (VT)(*hptr) : (VT)0; }
    __device__ void elem(int i, double (&a)[1]) const
    {
        VT wi = w[i];
        if (vprev) {
            const VT minh = -h;
            wi = wi + minh * vprev[i];
            w[i] = wi;
        }
        const VT o = vnext ? vnext[i] : wi;
        a[0] += (double)wi * (double)o;
    }
    __device__ void finalize(const double *t) const { *dst = t[0]; }
};

// copy: dst = src
template <typename VT>
struct OpCopy {
    static constexpr int K = 0;
    int n;
    KState *st;
    VT *dst;
    const VT *src;
    __device__ void load() {}
    __device__ void elem(int i, double (&)[1]) const { dst[i] = src[i]; }
    __device__ void finalize(const double *) const {}
};

// ---------------------------------------------------------------- workspace
struct Workspace {
    DBuf<KState> st;
    KState *h_st = nullptr;  // pinned mirror
    DBuf<double> part;
    DBuf<unsigned> ticket;
    DBuf<double> hist, hist_rel;
    int hist_cap = 0;
    int part_cap = 0;
    RedSlot slot() const
    {
        if (!part.p || !ticket.p) throw Status(XS_ERR_ORDER);  // ensure() must run first
        return RedSlot{part.p, ticket.p};
    }
    void ensure(int max_k, int maxiter)
    {
        int G = std::max(geom().red_grid, geom().sms * 16);  // covers every reduction grid (ELL: <= 10 CTAs per SM)
        if (part_cap < max_k * G) {
            part.alloc((size_t)max_k * G);
            part_cap = max_k * G;
        }
        if (!ticket.p) ticket.alloc(1);
        if (!st.p) {
            st.alloc(1);
            XS_CUDA(cudaMallocHost((void **)&h_st, sizeof(KState)));
        }
        if (hist_cap < maxiter + 2) {
            hist.alloc(maxiter + 2);
            hist_rel.alloc(maxiter + 2);
            hist_cap = maxiter + 2;
        }
    }
    ~Workspace()
    {
        if (h_st) cudaFreeHost(h_st);
    }
};

}  // namespace xs
