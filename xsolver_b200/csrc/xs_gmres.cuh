// Restarted methods: GMRES(m) / FGMRES(m) and GCR(m).
//
// GMRES follows intel/mpisolver-C-v1.cpp:933-1087 (left preconditioned) and
// :1089-1247 (right preconditioned, flexible form with stored Z = M^-1 V):
// modified Gram-Schmidt, Givens rotations (:1249-1279), back-substitution and
// update (updatec, :1281-1301).  The Hessenberg matrix, rotations and the
// least-squares right-hand side live in device memory in FP64 and are updated
// by the last block of the norm reduction (one thread), so the host never
// sees them; the reference GPU path keeps H on the host
// (cuda/mpicudasolver-C-v1.cu:1199-1219).
//
// GCR follows intel cpu_gcr_solve / cpu_igcr_solve (:685-931, left
// preconditioned, classical / modified Gram-Schmidt) and hip
// Xsolver_igcr::xsolver (hip/Solver/xsolver_igcr.cpp:29-108, right
// preconditioned, modified Gram-Schmidt).
//
// One restart cycle (m steps, each a fixed kernel sequence that depends on the
// step index) is captured into one CUDA graph and replayed per cycle.
#pragma once
#include "xs_solvers.cuh"

namespace xs {

// KState slots used here
enum { S_GM_INV = 20, S_GM_UPDK = 21 };

struct GmDev {
    double *H;   // (m+1) x m, row-major H[r*m + c]
    double *s, *cs, *sn, *y;
    int m;
};

__device__ inline void gm_applyrot(double &dx, double &dy, double cs, double sn)
{
    const double t = cs * dx + sn * dy;
    dy = -sn * dx + cs * dy;
    dx = t;
}
__device__ inline void gm_genrot(double dx, double dy, double &cs, double &sn)
{
    if (dy == 0.0) {
        cs = 1.0;
        sn = 0.0;
    } else if (fabs(dy) > fabs(dx)) {
        const double t = dx / dy;
        sn = 1.0 / sqrt(1.0 + t * t);
        cs = t * sn;
    } else {
        const double t = dy / dx;
        cs = 1.0 / sqrt(1.0 + t * t);
        sn = t * cs;
    }
}

// w = w - h V_prev ; last step of MGS, acc = w.w, then Givens (thread 0 of last block)
template <typename VT>
struct OpGmNorm {
    static constexpr int K = 1;
    int n;
    KState *st;
    VT *w;
    const VT *vprev;
    const double *hptr;
    GmDev g;
    int i;
    int quirk;
    VT h;
    __device__ void load() { h = (VT)(*hptr); }
    __device__ void elem(int q, double (&a)[1]) const
    {
        const VT minh = -h;
        const VT wi = w[q] + minh * vprev[q];
        w[q] = wi;
        a[0] += (double)wi * (double)wi;
    }
    __device__ void finalize(const double *t) const
    {
        const int m = g.m;
        double *H = g.H;
        const double nrm = sqrt(t[0]);
        H[(i + 1) * m + i] = nrm;
        st->sc[S_GM_INV] = 1.0 / (nrm + KSMALL);
        for (int k = 0; k < i; k++) gm_applyrot(H[k * m + i], H[(k + 1) * m + i], g.cs[k], g.sn[k]);
        gm_genrot(H[i * m + i], H[(i + 1) * m + i], g.cs[i], g.sn[i]);
        gm_applyrot(H[i * m + i], H[(i + 1) * m + i], g.cs[i], g.sn[i]);
        gm_applyrot(g.s[i], g.s[i + 1], g.cs[i], g.sn[i]);
        const bool cont = record_and_test(st, fabs(g.s[i + 1]));
        if (!cont) {
            if (st->done == 1) st->kcols = quirk ? i : i + 1;
            else st->kcols = i + 1;
        }
    }
};

// dst = src * scale (scale from a KState slot)
template <typename VT>
struct OpScaleCopy {
    static constexpr int K = 0;
    int n;
    KState *st;
    VT *dst;
    VT *src;  // also scaled in place when src_inplace
    int slot;
    int src_inplace;
    VT sc;
    __device__ void load() { sc = (VT)st->sc[slot]; }
    __device__ void elem(int q, double (&)[1]) const
    {
        const VT v = src[q] * sc;
        if (src_inplace) src[q] = v;
        dst[q] = v;
    }
    __device__ void finalize(const double *) const {}
};

// start of a cycle: zero H, s, cs, sn; s[0] = beta; inv = 1/(beta+small)
static __global__ void k_gm_cycle_init(KState *st, GmDev g)
{
    if (st->done) return;
    const int m = g.m;
    for (int q = threadIdx.x; q < (m + 1) * m; q += blockDim.x) g.H[q] = 0.0;
    for (int q = threadIdx.x; q < m + 1; q += blockDim.x) {
        g.s[q] = 0.0;
        g.cs[q] = 0.0;
        g.sn[q] = 0.0;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        const double beta = st->sc[S_BETA];
        g.s[0] = beta;
        st->sc[S_GM_INV] = 1.0 / (beta + KSMALL);
    }
}

// end of a cycle: back-substitution (updatec) for k columns, y -> g.y
static __global__ void k_gm_backsub(KState *st, GmDev g)
{
    if (threadIdx.x != 0) return;
    if (st->finalized) {
        st->sc[S_GM_UPDK] = 0.0;
        return;
    }
    const int m = g.m;
    const int k = st->done ? st->kcols : m;
    for (int q = 0; q < k; q++) g.y[q] = g.s[q];
    for (int q = k - 1; q >= 0; q--) {
        g.y[q] = g.y[q] / (g.H[q * m + q] + KSMALL);
        for (int j = q - 1; j >= 0; j--) g.y[j] = g.y[j] - g.H[j * m + q] * g.y[q];
    }
    st->sc[S_GM_UPDK] = (double)k;
    if (st->done) st->finalized = 1;
    else st->sc[S_BETA] = fabs(g.s[m]);
}

// x += sum_{q<k} y_q B_q  (sequential in q per element, as consecutive daxpys)
template <typename VT>
__global__ void k_gm_update(int n, const KState *st, const double *y, const VT *basis, long stride, VT *x)
{
    const int k = (int)st->sc[S_GM_UPDK];
    if (k <= 0) return;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        VT xi = x[i];
        for (int q = 0; q < k; q++) xi = xi + (VT)y[q] * basis[q * stride + i];
        x[i] = xi;
    }
}

template <typename VT, typename MT>
struct GmresRun {
    VecPool<VT> pool;
    DBuf<VT> V, Z;
    DBuf<double> gm;
    int mcap = 0;
    GraphCache gc;
    void run(SolveCtx &c, const VT *b, VT *x, int m, bool right)
    {
        const int n = c.n;
        if (m < 1) m = 1;
        if (mcap != m || V.n != (size_t)(m + 1) * n) {
            V.alloc((size_t)(m + 1) * n);
            if (right) Z.alloc((size_t)(m + 1) * n);
            gm.alloc((size_t)(m + 1) * m + 5 * (m + 1));
            mcap = m;
            gc.reset();
        }
        if (right && Z.n != (size_t)(m + 1) * n) {
            Z.alloc((size_t)(m + 1) * n);
            gc.reset();
        }
        VT *res = pool.get(0, n), *w = pool.get(1, n);
        KState *st = c.W->st.p;
        RedSlot sl = c.W->slot();
        const int *done = &st->done;
        GmDev g;
        g.m = m;
        g.H = gm.p;
        g.s = gm.p + (m + 1) * m;
        g.cs = g.s + (m + 1);
        g.sn = g.cs + (m + 1);
        g.y = g.sn + (m + 1);
        auto Vk = [&](int k) { return V.p + (size_t)k * n; };
        auto Zk = [&](int k) { return Z.p + (size_t)k * n; };
        // initial residual: res = b - A x ; left: res = M^-1 res ; beta = ||res||
        spmv<VT, MT>(*c.A, x, res, EpiResid<VT>{st, b}, sl, c.s);
        if (!right) c.M->apply<VT>(res, res, nullptr, c.s);
        vecop(OpGmInit<VT>{n, st, res}, sl, c.s);
        const int quirk = c.quirk;
        auto cycle = [&]() {
            k_gm_cycle_init<<<1, 256, 0, c.s>>>(st, g);
            vecop(OpScaleCopy<VT>{n, st, Vk(0), res, S_GM_INV, 1, (VT)0}, sl, c.s);
            for (int i = 0; i < m; i++) {
                if (right) {
                    c.M->apply<VT>(Vk(i), Zk(i), done, c.s);
                    spmv<VT, MT>(*c.A, Zk(i), w, EpiActive<VT>{st}, sl, c.s);
                } else {
                    spmv<VT, MT>(*c.A, Vk(i), w, EpiActive<VT>{st}, sl, c.s);
                    c.M->apply<VT>(w, w, done, c.s);
                }
                // h_0 = w.V_0
                vecop(OpMgsStep<VT>{n, st, w, nullptr, Vk(0), nullptr, &g.H[0 * m + i], (VT)0}, sl, c.s);
                for (int k = 1; k <= i; k++)
                    vecop(OpMgsStep<VT>{n, st, w, Vk(k - 1), Vk(k), &g.H[(k - 1) * m + i], &g.H[k * m + i], (VT)0}, sl,
                          c.s);
                vecop(OpGmNorm<VT>{n, st, w, Vk(i), &g.H[i * m + i], g, i, quirk, (VT)0}, sl, c.s);
                vecop(OpScaleCopy<VT>{n, st, Vk(i + 1), w, S_GM_INV, 1, (VT)0}, sl, c.s);
            }
            k_gm_backsub<<<1, 32, 0, c.s>>>(st, g);
            k_gm_update<VT><<<geom().sms * 4, 256, 0, c.s>>>(n, st, g.y, right ? Z.p : V.p, (long)n, x);
            // restart residual (skipped once done)
            spmv<VT, MT>(*c.A, x, res, EpiResidActive<VT>{st, b}, sl, c.s);
            if (!right) c.M->apply<VT>(res, res, done, c.s);
        };
        std::vector<const void *> key{b, x, res, w, V.p, Z.p, gm.p, st, c.M, c.A, (const void *)(long)m,
                                      (const void *)(long)right, (const void *)(long)quirk,
                                      (const void *)cfg_key(c)};
        const int maxit = c.W->h_st->maxiter;
        run_graph_loop(c, gc, key, 1, maxit / m + 3, cycle);
    }
};

// ---------------------------------------------------------------- GCR
// multi-dot: alpha[i] = c_i . c_k for i < k, stored in st->sc[S_H + i] (k <= 32)
// or a device array; grid (G, k), partials [i][G]
template <typename VT>
__global__ void __launch_bounds__(256) k_multidot(int n, KState *st, const VT *basis, long stride, const VT *ck, int k,
                                                  double *out, RedSlot slot)
{
    if (st->done) return;
    const int i = blockIdx.y;
    const VT *ci = basis + (long)i * stride;
    double a = 0.0;
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) a += (double)ci[q] * (double)ck[q];
    for (int o = 16; o > 0; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
    __shared__ double sw[32];
    __shared__ bool last;
    if ((threadIdx.x & 31) == 0) sw[threadIdx.x >> 5] = a;
    __syncthreads();
    const int G = gridDim.x;
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) s += sw[w];
        slot.part[(long)i * G + blockIdx.x] = s;
        __threadfence();
        unsigned t = atomicAdd(slot.ticket, 1u);
        last = (t == (unsigned)(G * k) - 1);
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    // last block: each warp sums some of the k dots in block order
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int d = wid; d < k; d += nw) {
        double s = 0.0;
        for (int bb = lane; bb < G; bb += 32) s += __ldcg(slot.part + (long)d * G + bb);
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (lane == 0) out[d] = s;
    }
    __syncthreads();
    if (threadIdx.x == 0) *slot.ticket = 0u;
}

// CGS update: c_k -= sum_i alpha_i c_i ; u_k -= sum_i alpha_i u_i (sequential i)
template <typename VT>
__global__ void k_gcr_cgs_update(int n, const KState *st, const double *alpha, int k, const VT *C, const VT *Ub, long stride,
                                 VT *ck, VT *uk)
{
    if (st->done) return;
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) {
        VT c = ck[q], u = uk[q];
        for (int i = 0; i < k; i++) {
            const VT ma = -(VT)alpha[i];
            c = c + ma * C[(long)i * stride + q];
        }
        for (int i = 0; i < k; i++) {
            const VT ma = -(VT)alpha[i];
            u = u + ma * Ub[(long)i * stride + q];
        }
        ck[q] = c;
        uk[q] = u;
    }
}

// MGS step: c_k -= a c_prev ; u_k -= a u_prev ; acc c_k . c_next
// (prev == null: no update; next == null: acc c_k.c_k and c_k.res -> t0, t1)
template <typename VT>
struct OpGcrMgs {
    static constexpr int K = 2;
    int n;
    KState *st;
    VT *ck, *uk;
    const VT *cprev, *uprev, *cnext, *res;
    const double *aptr;
    double *dst;
    VT a;
    __device__ void load() { a = cprev ? (VT)(*aptr) : (VT)0; }
    __device__ void elem(int q, double (&acc)[2]) const
    {
        VT c = ck[q];
        if (cprev) {
            const VT ma = -a;
            c = c + ma * cprev[q];
            ck[q] = c;
            uk[q] = uk[q] + ma * uprev[q];
        }
        if (cnext) acc[0] += (double)cnext[q] * (double)c;
        else {
            acc[0] += (double)c * (double)c;
            acc[1] += (double)c * (double)res[q];
        }
    }
    __device__ void finalize(const double *t) const
    {
        if (cnext) *dst = t[0];
        else {
            const double t0 = sqrt(t[0]);
            st->sc[S_GCR_T0] = t0;
            st->sc[S_GCR_T1] = t[1];
            st->sc[S_GCR_INV] = 1.0 / (t0 + KSMALL);
            st->sc[S_GCR_COEF] = t[1] / (t0 + KSMALL);
            if (!isfinite(t[0]) || !isfinite(t[1])) { st->err |= DEV_BREAKDOWN; st->done = 3; }
        }
    }
};

// u_k *= inv ; c_k *= inv ; x += coef u_k ; res -= coef c_k ; acc res.res
template <typename VT>
struct OpGcrUpdate {
    static constexpr int K = 1;
    int n;
    KState *st;
    VT *ck, *uk, *x, *res;
    VT inv, coef;
    __device__ void load()
    {
        inv = (VT)st->sc[S_GCR_INV];
        coef = (VT)st->sc[S_GCR_COEF];
    }
    __device__ void elem(int q, double (&a)[1]) const
    {
        const VT u = uk[q] * inv;
        const VT c = ck[q] * inv;
        uk[q] = u;
        ck[q] = c;
        x[q] = x[q] + coef * u;
        const VT mcoef = -coef;
        const VT r = res[q] + mcoef * c;
        res[q] = r;
        a[0] += (double)r * (double)r;
    }
    __device__ void finalize(const double *t) const { record_and_test(st, sqrt(t[0])); }
};

template <typename VT, typename MT>
struct GcrRun {
    VecPool<VT> pool;
    DBuf<VT> U, C;
    DBuf<double> alpha;
    int mcap = 0;
    GraphCache gc;
    // variant 0: left CGS (intel gcr), 1: left MGS (intel igcr), 2: right MGS (hip igcr)
    void run(SolveCtx &c, const VT *b, VT *x, int m, int variant)
    {
        const int n = c.n;
        if (m < 1) m = 1;
        if (mcap != m || U.n != (size_t)m * n) {
            U.alloc((size_t)m * n);
            C.alloc((size_t)m * n);
            alpha.alloc(std::max(m, 1));
            mcap = m;
            gc.reset();
        }
        VT *res = pool.get(0, n);
        KState *st = c.W->st.p;
        RedSlot sl = c.W->slot();
        const int *done = &st->done;
        const bool right = variant == 2;
        auto Uk = [&](int k) { return U.p + (size_t)k * n; };
        auto Ck = [&](int k) { return C.p + (size_t)k * n; };
        spmv<VT, MT>(*c.A, x, res, EpiResid<VT>{st, b}, sl, c.s);
        if (!right) c.M->apply<VT>(res, res, nullptr, c.s);
        vecop(OpGmInit<VT>{n, st, res}, sl, c.s);
        auto cycle = [&]() {
            for (int k = 0; k < m; k++) {
                if (right) {
                    c.M->apply<VT>(res, Uk(k), done, c.s);
                    spmv<VT, MT>(*c.A, Uk(k), Ck(k), EpiActive<VT>{st}, sl, c.s);
                } else {
                    vecop(OpCopy<VT>{n, st, Uk(k), res}, sl, c.s);
                    spmv<VT, MT>(*c.A, Uk(k), Ck(k), EpiActive<VT>{st}, sl, c.s);
                    c.M->apply<VT>(Ck(k), Ck(k), done, c.s);
                }
                if (variant == 0) {
                    if (k > 0) {
                        dim3 grid(std::max(1, geom().red_grid / std::max(k, 1)), k);
                        k_multidot<VT><<<grid, 256, 0, c.s>>>(n, st, C.p, (long)n, Ck(k), k, alpha.p, sl);
                        k_gcr_cgs_update<VT><<<geom().sms * 4, 256, 0, c.s>>>(n, st, alpha.p, k, C.p, U.p, (long)n, Ck(k),
                                                                              Uk(k));
                        check_launch();
                    }
                    vecop(OpGcrMgs<VT>{n, st, Ck(k), Uk(k), nullptr, nullptr, nullptr, res, nullptr, nullptr, (VT)0}, sl,
                          c.s);
                } else {
                    // MGS: alpha_0 = c_0.c_k ; for i: c_k -= alpha_i c_i, alpha_{i+1} = c_{i+1}.c_k
                    if (k > 0) {
                        vecop(OpGcrMgs<VT>{n, st, Ck(k), Uk(k), nullptr, nullptr, Ck(0), res, nullptr, &alpha.p[0], (VT)0},
                              sl, c.s);
                        for (int i = 1; i < k; i++)
                            vecop(OpGcrMgs<VT>{n, st, Ck(k), Uk(k), Ck(i - 1), Uk(i - 1), Ck(i), res, &alpha.p[i - 1],
                                               &alpha.p[i], (VT)0},
                                  sl, c.s);
                        vecop(OpGcrMgs<VT>{n, st, Ck(k), Uk(k), Ck(k - 1), Uk(k - 1), nullptr, res, &alpha.p[k - 1],
                                           nullptr, (VT)0},
                              sl, c.s);
                    } else {
                        vecop(OpGcrMgs<VT>{n, st, Ck(k), Uk(k), nullptr, nullptr, nullptr, res, nullptr, nullptr, (VT)0},
                              sl, c.s);
                    }
                }
                vecop(OpGcrUpdate<VT>{n, st, Ck(k), Uk(k), x, res, (VT)0, (VT)0}, sl, c.s);
            }
        };
        std::vector<const void *> key{b, x, res, U.p, C.p, alpha.p, st, c.M, c.A, (const void *)(long)m,
                                      (const void *)(long)variant,
                                      (const void *)cfg_key(c)};
        run_graph_loop(c, gc, key, 1, c.W->h_st->maxiter / m + 3, cycle);
    }
};

}  // namespace xs
