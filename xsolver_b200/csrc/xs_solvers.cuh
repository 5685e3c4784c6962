// Host drivers of the Krylov methods: initial sequence, one CUDA graph per
// chunk of iterations, pipelined polling of the device done flag.
#pragma once
#include <vector>
#include <cstring>
#include "xs_krylov.cuh"
#include "xs_persist.cuh"

namespace xs {

enum Method {
    KSP_CGM = 1,       // PCG (hip "cg", intel cpu_cgm_solve)
    KSP_CG_LEFT = 2,   // intel cpu_cg_solve (CG on M^-1 A)
    KSP_BICGSTAB = 3,
    KSP_GCR_LEFT = 4,  // intel cpu_gcr_solve (classical GS)
    KSP_IGCR_LEFT = 5, // intel cpu_igcr_solve (modified GS)
    KSP_GCR_RIGHT = 6, // hip Xsolver_igcr (right preconditioned, MGS)
    KSP_GMRES_LEFT = 7,
    KSP_GMRES_RIGHT = 8,
    KSP_ICG = 9,       // intel cpu_icg_solve (single-reduction CG on M^-1 A)
    KSP_ICGM = 10,     // intel cpu_icgm_solve (single-reduction PCG)
    KSP_IBICGSTAB = 11 // intel cpu_ibicgstab_solve (single-reduction, right preconditioned)
};

// vectors owned by a solve, cached across solves of the same size
template <typename VT>
struct VecPool {
    std::vector<DBuf<VT>> v;
    int n = 0;
    VT *get(int idx, int nn)
    {
        if (nn != n) {
            v.clear();
            n = nn;
        }
        while ((int)v.size() <= idx) {
            v.emplace_back();
            v.back().alloc(n);
        }
        return v[idx].p;
    }
};

struct GraphCache {
    size_t nodes = 0;  // kernel nodes in the captured graph
    GraphCache() = default;
    GraphCache(const GraphCache &) = delete;
    GraphCache &operator=(const GraphCache &) = delete;
    cudaGraphExec_t exec = nullptr;
    std::vector<const void *> key;
    // polling resources, created on first use and kept (a pinned allocation
    // per solve would cost more than a short solve)
    int *hflag = nullptr;
    cudaEvent_t ev[2] = {nullptr, nullptr};
    void reset()
    {
        if (exec) cudaGraphExecDestroy(exec);
        exec = nullptr;
        key.clear();
    }
    void ensure_polling()
    {
        if (!hflag) XS_CUDA(cudaMallocHost((void **)&hflag, sizeof(int) * 2));
        for (int q = 0; q < 2; q++)
            if (!ev[q]) XS_CUDA(cudaEventCreateWithFlags(&ev[q], cudaEventDisableTiming));
    }
    ~GraphCache()
    {
        reset();
        if (hflag) cudaFreeHost(hflag);
        for (int q = 0; q < 2; q++)
            if (ev[q]) cudaEventDestroy(ev[q]);
    }
};

struct SolveCtx {
    cudaStream_t s;
    Operator *A;
    PrecondDev *M;
    Workspace *W;
    int n;
    int chunk = 8;
    int quirk = 1;
    long long *launches = nullptr;  // kernels launched (graph nodes), accumulated
};

// configuration that changes the captured kernels
inline long cfg_key(const SolveCtx &c)
{
    return (long)c.M->type * 100000 + (long)c.M->trsv_mode * 100 + c.M->factor_prec * 10 + c.A->format;
}

// Capture `body` `reps` times into a graph and replay until done.
template <class Body>
inline void run_graph_loop(SolveCtx &c, GraphCache &gc, const std::vector<const void *> &key, int reps,
                           int max_launches, Body body)
{
    if (!gc.exec || gc.key != key) {
        Trace tr("graph capture", c.s);
        gc.reset();
        cudaGraph_t g;
        XS_CUDA(cudaStreamBeginCapture(c.s, cudaStreamCaptureModeRelaxed));
        try {
            for (int r = 0; r < reps; r++) body();
        } catch (...) {
            cudaGraph_t junk;
            cudaStreamEndCapture(c.s, &junk);
            if (junk) cudaGraphDestroy(junk);
            throw;
        }
        XS_CUDA(cudaStreamEndCapture(c.s, &g));
        size_t nn = 0;
        cudaGraphGetNodes(g, nullptr, &nn);
        gc.nodes = nn;
        cudaError_t e = cudaGraphInstantiate(&gc.exec, g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) throw Status(XS_ERR_CUDA);
        gc.key = key;
    }
    // pipelined polling: check launch k-1's flag after enqueueing launch k
    gc.ensure_polling();
    int *hflag = gc.hflag;
    cudaEvent_t *ev = gc.ev;
    KState *dst = c.W->st.p;
    bool stop = false;
    for (int l = 0; l < max_launches && !stop; l++) {
        XS_CUDA(cudaGraphLaunch(gc.exec, c.s));
        if (c.launches) *c.launches += (long long)gc.nodes;
        XS_CUDA(cudaMemcpyAsync(&hflag[l & 1], &dst->done, sizeof(int), cudaMemcpyDeviceToHost, c.s));
        XS_CUDA(cudaEventRecord(ev[l & 1], c.s));
        if (l > 0) {
            XS_CUDA(cudaEventSynchronize(ev[(l - 1) & 1]));
            if (hflag[(l - 1) & 1]) stop = true;
        }
    }
    XS_CUDA(cudaStreamSynchronize(c.s));
}

// ---------------------------------------------------------------- PCG (cgm)
template <typename VT, typename MT>
struct PcgRun {
    VecPool<VT> pool;
    GraphCache gc;
    void run(SolveCtx &c, const VT *b, VT *x)
    {
        const int n = c.n;
        VT *r = pool.get(0, n), *z = pool.get(1, n), *p = pool.get(2, n), *Ap = pool.get(3, n);
        KState *st = c.W->st.p;
        RedSlot sl = c.W->slot();
        const int *done = &st->done;
        spmv<VT, MT>(*c.A, x, r, EpiResid<VT>{st, b}, sl, c.s);
        c.M->apply<VT>(r, z, done, c.s);
        vecop(OpCgmInit<VT>{n, st, r, z, p}, sl, c.s);
        auto body = [&]() {
            spmv<VT, MT>(*c.A, p, Ap, EpiDot1<VT>{st, p, 0, M_CGM_SIGMA}, sl, c.s);
            vecop(OpCgmUpdate<VT>{n, st, x, r, p, Ap, (VT)0}, sl, c.s);
            c.M->apply<VT>(r, z, done, c.s);
            vecop(OpDotRZ<VT>{n, st, r, z}, sl, c.s);
            vecop(OpPUpdate<VT>{n, st, p, z, (VT)0}, sl, c.s);
        };
        std::vector<const void *> key{b, x, r, z, p, Ap, st, c.M, c.A, (const void *)cfg_key(c)};
        int maxit = c.W->h_st->maxiter;
        run_graph_loop(c, gc, key, c.chunk, maxit / c.chunk + 3, body);
    }
};

// ---------------------------------------------------------------- left CG (cg)
template <typename VT>
struct OpCgSigma {  // sigma = p.q ; alpha = taoo/(sigma+small)
    static constexpr int K = 1;
    int n;
    KState *st;
    const VT *p, *q;
    __device__ void load() {}
    __device__ void elem(int i, double (&a)[1]) const { a[0] += (double)p[i] * (double)q[i]; }
    __device__ void finalize(const double *t) const
    {
        st->sc[S_SIGMA] = t[0];
        st->sc[S_ALPHA] = st->sc[S_TAOO] / (t[0] + KSMALL);
        if (!isfinite(t[0])) { st->err |= DEV_BREAKDOWN; st->done = 3; }
    }
};

template <typename VT, typename MT>
struct CgLeftRun {
    VecPool<VT> pool;
    GraphCache gc;
    void run(SolveCtx &c, const VT *b, VT *x)
    {
        const int n = c.n;
        VT *r = pool.get(0, n), *q = pool.get(1, n), *p = pool.get(2, n), *Ap = pool.get(3, n);
        KState *st = c.W->st.p;
        RedSlot sl = c.W->slot();
        const int *done = &st->done;
        spmv<VT, MT>(*c.A, x, r, EpiResid<VT>{st, b}, sl, c.s);
        c.M->apply<VT>(r, r, done, c.s);
        vecop(OpCgInit<VT>{n, st, r, p}, sl, c.s);
        auto body = [&]() {
            spmv<VT, MT>(*c.A, p, Ap, EpiActive<VT>{st}, sl, c.s);
            c.M->apply<VT>(Ap, q, done, c.s);
            vecop(OpCgSigma<VT>{n, st, p, q}, sl, c.s);
            vecop(OpCgUpdate<VT>{n, st, x, r, p, q, (VT)0}, sl, c.s);
            vecop(OpCgP<VT>{n, st, p, r, (VT)0}, sl, c.s);
        };
        std::vector<const void *> key{b, x, r, q, p, Ap, st, c.M, c.A, (const void *)cfg_key(c)};
        run_graph_loop(c, gc, key, c.chunk, c.W->h_st->maxiter / c.chunk + 3, body);
    }
};

// ---------------------------------------------------------------- single-reduction CG
// intel/mpisolver-C-v1.cpp:104-191: the initial sequence of CgLeftRun, then
// per iteration SpMV, apply, one pass for the three dot products, one pass
// for the x, r and p updates with the convergence test
template <typename VT, typename MT>
struct IcgRun {
    VecPool<VT> pool;
    GraphCache gc;
    void run(SolveCtx &c, const VT *b, VT *x)
    {
        const int n = c.n;
        VT *r = pool.get(0, n), *q = pool.get(1, n), *p = pool.get(2, n), *Ap = pool.get(3, n);
        KState *st = c.W->st.p;
        RedSlot sl = c.W->slot();
        const int *done = &st->done;
        spmv<VT, MT>(*c.A, x, r, EpiResid<VT>{st, b}, sl, c.s);
        c.M->apply<VT>(r, r, done, c.s);
        vecop(OpCgInit<VT>{n, st, r, p}, sl, c.s);
        auto body = [&]() {
            spmv<VT, MT>(*c.A, p, Ap, EpiActive<VT>{st}, sl, c.s);
            c.M->apply<VT>(Ap, q, done, c.s);
            vecop(OpIcgDots<VT>{n, st, p, r, q}, sl, c.s);
            vecop(OpIcgUpdate<VT>{n, st, x, r, p, q, (VT)0, (VT)0}, sl, c.s);
        };
        std::vector<const void *> key{b, x, r, q, p, Ap, st, c.M, c.A, (const void *)cfg_key(c)};
        run_graph_loop(c, gc, key, c.chunk, c.W->h_st->maxiter / c.chunk + 3, body);
    }
};
// intel/mpisolver-C-v1.cpp:273-363: the initial sequence of PcgRun, then per
// iteration SpMV, apply, one pass for the five dot products, the x and r
// updates with the convergence test, apply, p update
template <typename VT, typename MT>
struct IcgmRun {
    VecPool<VT> pool;
    GraphCache gc;
    void run(SolveCtx &c, const VT *b, VT *x)
    {
        const int n = c.n;
        VT *r = pool.get(0, n), *z = pool.get(1, n), *p = pool.get(2, n), *Ap = pool.get(3, n), *q = pool.get(4, n);
        KState *st = c.W->st.p;
        RedSlot sl = c.W->slot();
        const int *done = &st->done;
        spmv<VT, MT>(*c.A, x, r, EpiResid<VT>{st, b}, sl, c.s);
        c.M->apply<VT>(r, z, done, c.s);
        vecop(OpCgmInit<VT>{n, st, r, z, p}, sl, c.s);
        auto body = [&]() {
            spmv<VT, MT>(*c.A, p, Ap, EpiActive<VT>{st}, sl, c.s);
            c.M->apply<VT>(Ap, q, done, c.s);
            vecop(OpIcgmDots<VT>{n, st, p, r, q, Ap, z}, sl, c.s);
            vecop(OpIcgmUpdate<VT>{n, st, x, r, p, Ap, (VT)0}, sl, c.s);
            c.M->apply<VT>(r, z, done, c.s);
            vecop(OpCgP<VT>{n, st, p, z, (VT)0}, sl, c.s);
        };
        std::vector<const void *> key{b, x, r, z, p, Ap, q, st, c.M, c.A, (const void *)cfg_key(c)};
        run_graph_loop(c, gc, key, c.chunk, c.W->h_st->maxiter / c.chunk + 3, body);
    }
};

// intel/mpisolver-C-v1.cpp:484-683: phi = x0, start-up products, then per
// iteration: vk/sk/zk pass, apply + SpMV (qk), tk pass with five dot
// products, apply + SpMV (pk) with the sixth in its epilogue, res/phi pass
// with the convergence test; finally x = M^-1 phi.  The reference takes
// A M^-1 A phi only for a nonzero phi; for phi = 0 that product is exactly
// zero, so both of its branches are this one sequence.
template <typename VT, typename MT>
struct IbicgRun {
    VecPool<VT> pool;
    GraphCache gc;
    void run(SolveCtx &c, const VT *b, VT *x)
    {
        const int n = c.n;
        VT *res = pool.get(0, n), *reso = pool.get(1, n), *phi = pool.get(2, n), *tk = pool.get(3, n);
        VT *pk = pool.get(4, n), *qk = pool.get(5, n), *zk = pool.get(6, n), *vk = pool.get(7, n);
        VT *sk = pool.get(8, n), *resm = pool.get(9, n);
        KState *st = c.W->st.p;
        RedSlot sl = c.W->slot();
        const int *done = &st->done;
        XS_CUDA(cudaMemcpyAsync(phi, x, sizeof(VT) * n, cudaMemcpyDeviceToDevice, c.s));
        spmv<VT, MT>(*c.A, phi, res, EpiResid<VT>{st, b}, sl, c.s);
        spmv<VT, MT>(*c.A, phi, pk, EpiAx<VT>{}, sl, c.s);
        c.M->apply<VT>(pk, resm, nullptr, c.s);
        spmv<VT, MT>(*c.A, resm, pk, EpiAx<VT>{}, sl, c.s);
        c.M->apply<VT>(res, resm, nullptr, c.s);
        spmv<VT, MT>(*c.A, resm, tk, EpiAx<VT>{}, sl, c.s);
        vecop(OpIbInit<VT>{n, st, res, pk, tk, reso, qk, vk, zk}, sl, c.s);
        auto body = [&]() {
            vecop(OpIbV<VT>{n, st, tk, pk, qk, res, vk, sk, zk}, sl, c.s);
            c.M->apply<VT>(vk, resm, done, c.s);
            spmv<VT, MT>(*c.A, resm, qk, EpiActive<VT>{st}, sl, c.s);
            vecop(OpIbT<VT>{n, st, tk, pk, qk, sk, reso}, sl, c.s);
            c.M->apply<VT>(tk, resm, done, c.s);
            spmv<VT, MT>(*c.A, resm, pk, EpiDot1<VT>{st, reso, 0, M_IBICG_NU}, sl, c.s);
            vecop(OpIbR<VT>{n, st, res, phi, sk, tk, zk}, sl, c.s);
        };
        std::vector<const void *> key{b, x, res, reso, phi, tk, pk, qk, zk, vk, sk, resm, st, c.M, c.A,
                                      (const void *)cfg_key(c)};
        run_graph_loop(c, gc, key, c.chunk, c.W->h_st->maxiter / c.chunk + 3, body);
        c.M->apply<VT>(phi, x, nullptr, c.s);
    }
};

// ---------------------------------------------------------------- BiCGSTAB
template <typename VT, typename MT>
struct BicgRun {
    VecPool<VT> pool;
    GraphCache gc;
    DBuf<unsigned> bar;  // grid barrier of the persistent iteration
    VT *residual(int n) { return pool.get(0, n); }
    VT *shadow(int n) { return pool.get(1, n); }
    // resume: continue the previous run's iteration (same p, u, rhat and
    // scalars; r may have been replaced meanwhile) instead of starting anew
    void run(SolveCtx &c, const VT *b, VT *x, bool resume = false)
    {
        const int n = c.n;
        VT *r = pool.get(0, n), *rhat = pool.get(1, n), *p = pool.get(2, n), *u = pool.get(3, n);
        VT *s = pool.get(4, n), *v = pool.get(5, n), *z1 = pool.get(6, n), *z2 = pool.get(7, n);
        KState *st = c.W->st.p;
        RedSlot sl = c.W->slot();
        const int *done = &st->done;
        // the p and s updates inside the first L pass of the applies that
        // read them when the preconditioner allows it (a launch and a pass
        // over the vector fewer each); p then alternates between two
        // buffers, starting from the first at every graph replay
        const bool fuse = vec_fusion() && c.M->can_fuse_first_pass();
        VT *p2 = fuse ? pool.get(8, n) : p;
        if (!resume) {
            spmv<VT, MT>(*c.A, x, r, EpiResid<VT>{st, b}, sl, c.s);
            vecop(OpBicgInit<VT>{n, st, r, rhat, p, u}, sl, c.s);
        } else if (fuse) {
            k_bicg_p_home<VT><<<geom().sms * 4, 256, 0, c.s>>>(n, st, p, p2);
            k_bicg_p_homed<<<1, 1, 0, c.s>>>(st);
            check_launch();
        }
        const bool fuse_s = fuse;
        int parity = 0;  // iteration index inside the captured chunk
        auto body = [&]() {
            if (fuse) {
                VT *pin = (parity & 1) ? p2 : p, *pout = (parity & 1) ? p : p2;
                c.M->apply_fused<VT>(SrcBicgP<VT>{pin, u, r, pout, st, (VT)0, (VT)0, (parity & 1) ? 0 : 1}, pout, z1,
                                     done, c.s);
                parity++;
            } else {
                vecop(OpBicgP<VT>{n, st, p, r, u, (VT)0, (VT)0}, sl, c.s);
                c.M->apply<VT>(p, z1, done, c.s);
            }
            spmv<VT, MT>(*c.A, z1, u, EpiDot1<VT>{st, rhat, 0, M_BICG_GAMA}, sl, c.s);
            if (fuse_s) {
                c.M->apply_fused<VT>(SrcBicgS<VT>{r, u, s, st, (VT)0}, s, z2, done, c.s);
            } else {
                vecop(OpBicgS<VT>{n, st, s, r, u, (VT)0}, sl, c.s);
                c.M->apply<VT>(s, z2, done, c.s);
            }
            spmv<VT, MT>(*c.A, z2, v, EpiDot2<VT>{st, s, M_BICG_ALPHA}, sl, c.s);
            OpBicgX<VT> ox{n, st, x, r, z1, z2, s, v, rhat, (VT)0, (VT)0};
            ox.vec_ok = aligned16({x, r, z1, z2, s, v, rhat});
            vecop(ox, sl, c.s);
        };
        // the whole iteration as one persistent kernel when it serves this
        // configuration (same vector updates fused into the sweep passes)
        if (fuse && std::is_same<VT, MT>::value) {
            if (!bar.p) bar.alloc(2);
            const PersistVectors<VT> V{x, r, rhat, p, p2, u, s, v, z1, z2};
            if (persist_bicgstab(c, V, c.W->h_st->maxiter + 2, bar.p)) {
                XS_CUDA(cudaStreamSynchronize(c.s));
                return;
            }
        }
        std::vector<const void *> key{b, x, r, rhat, p, p2, u, s, v, z1, z2, st, c.M, c.A, (const void *)cfg_key(c),
                                      (const void *)(long)fuse_s};
        if (fuse && (c.chunk & 1)) throw Status(XS_ERR_INVALID);  // p must be back in its first buffer after a chunk
        run_graph_loop(c, gc, key, c.chunk, c.W->h_st->maxiter / c.chunk + 3, body);
    }
};

}  // namespace xs
