// Kernel-level entry points on device pointers (tests and benchmarks).
// Included at the end of xs_api.cu (uses its Handle and helpers).

struct xs_plan_s {
    std::unique_ptr<Handle> h;
    bool factored = false;
    int factor_kind = -1;
    DBuf<double> l2flush;
    DBuf<double> bx64, by64, bz64;
    DBuf<float> bx32, by32, bz32;
    xs::BatchPrecond bp;  // batched LU solves
    DBuf<int> zero;       // an all-done word that stays 0
};

namespace xs {

// L2 flush between timed repetitions: write the first half of a buffer
// larger than L2, then read the second half, so the timed kernel starts
// with an L2 holding none of its data and no dirty lines still waiting to
// be written back (which would otherwise drain into its own DRAM time)
static __global__ void k_flush(double *p, long m, double v, double *sink)
{
    const long h = m / 2;
    const long stride = (long)gridDim.x * blockDim.x;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < h; i += stride) p[i] = v + (double)i;
    double acc = 0.0;
    for (long i = h + blockIdx.x * (long)blockDim.x + threadIdx.x; i < m; i += stride) acc += p[i];
    if (acc == 1.2345e300) *sink = acc;  // keeps the reads
}
static __global__ void k_fill_rand(int n, double *x, float *x32, unsigned seed)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        unsigned h = (unsigned)i * 2654435761u ^ seed;
        h ^= h >> 13;
        h *= 0x5bd1e995u;
        h ^= h >> 15;
        double v = (double)(h & 0xffffff) / (double)0x1000000 * 2.0 - 1.0;
        x[i] = v;
        if (x32) x32[i] = (float)v;
    }
}

static void plan_lusolve64(Handle &h, const double *x, double *z)
{
    if (!h.M.have_factors) throw Status(XS_ERR_ORDER);
    h.M.apply<double>(x, z, nullptr, h.s);
}
static void plan_lusolve32(Handle &h, const float *x, float *z)
{
    if (!h.M.have_factors || !h.M.U.dinv32.p) throw Status(XS_ERR_ORDER);
    h.M.apply<float>(x, z, nullptr, h.s);
}

}  // namespace xs

extern "C" {

int xs_plan_create(xs_plan_t *p, int n, const int *rp, const int *ci, const double *v)
{
    return guarded([&] {
        if (!p) throw Status(XS_ERR_INVALID);
        check_gpu();
        auto *w = new xs_plan_s;
        w->h.reset(new Handle());
        w->h->all_factor_copies = true;
        try {
            set_matrix(*w->h, n, rp, ci, v, 0);
        } catch (...) {
            delete w;
            throw;
        }
        *p = w;
    });
}
int xs_plan_destroy(xs_plan_t p)
{
    return guarded([&] { delete p; });
}
int xs_plan_build_ell(xs_plan_t p, int *width)
{
    return guarded([&] {
        if (!p) throw Status(XS_ERR_INVALID);
        Handle &h = *p->h;
        operator_build_ell(h.A, h.hrp.data(), h.hci.data(), host_vals(h), 0, h.A.v32.p != nullptr, h.s);
        if (width) *width = h.A.ell_w;
    });
}
int xs_plan_spmv(xs_plan_t p, int format, int precision, const void *x, void *y)
{
    return guarded([&] {
        if (!p || !x || !y) throw Status(XS_ERR_INVALID);
        Handle &h = *p->h;
        if (format == 1 && h.A.ell_w == 0) throw Status(XS_ERR_ORDER);
        int saved = h.A.format;
        h.A.format = format;
        h.W.ensure(64, 1);
        const RedSlot sl = h.W.slot();
        if (precision == 0)
            spmv<double, double>(h.A, (const double *)x, (double *)y, EpiAx<double>{}, sl, h.s);
        else {
            operator_ensure32(h.A, h.hrp.data(), h.s);
            spmv<float, float>(h.A, (const float *)x, (float *)y, EpiAx<float>{}, sl, h.s);
        }
        h.A.format = saved;
    });
}
int xs_plan_spmv_t(xs_plan_t p, const double *x, double *y)
{
    return guarded([&] {
        if (!p || !x || !y) throw Status(XS_ERR_INVALID);
        Handle &h = *p->h;
        if (!h.adj.have_At) {
            std::vector<int> trp, tci;
            std::vector<double> tv;
            host_transpose(h.n, h.hrp.data(), h.hci.data(), host_vals(h), trp, tci, &tv, nullptr);
            h.adj.At = Operator();
            operator_setup(h.adj.At, h.n, trp.data(), tci.data(), tv.data(), 0, false, h.s, h.err.p);
            h.adj.have_At = true;
        }
        h.W.ensure(64, 1);
        spmv<double, double>(h.adj.At, x, y, EpiAx<double>{}, h.W.slot(), h.s);
    });
}
int xs_plan_factor(xs_plan_t p, int kind, int sweeps, double fill, double droptol)
{
    return guarded([&] {
        if (!p) throw Status(XS_ERR_INVALID);
        Handle &h = *p->h;
        if (kind == 0) h.pc_req = PC_ILU0;
        else if (kind == 1) { h.pc_req = PC_PARILU; h.parilu_sweeps = sweeps; }
        else if (kind == 2) { h.pc_req = PC_PARILUT; h.parilut_fill = fill; h.parilut_sweeps = sweeps; h.parilut_droptol = droptol; }
        else if (kind == 3) h.pc_req = PC_IC0;
        else if (kind == 4 || kind == 5) {
            // host threshold factorizations: fill is the entry limit per row part
            if (!(fill >= 0) || !(droptol >= 0) || (kind == 4 && fill < 1) || (kind == 5 && !(droptol > 0)))
                throw Status(XS_ERR_INVALID);
            h.pc_req = kind == 4 ? PC_ILUP : PC_ICT;
            (kind == 4 ? h.ilup_fill : h.ict_fill) = (int)fill;
            (kind == 4 ? h.ilup_tol : h.ict_tol) = droptol;
        } else throw Status(XS_ERR_INVALID);
        h.inner32 = 1;  // keep reduced-precision copies of the factors for the solves
        invalidate_pc(h);
        build_precond(h);
        p->factored = true;
        p->factor_kind = kind;
    });
}
int xs_plan_get_lu_values(xs_plan_t p, double *luv)
{
    return guarded([&] {
        if (!p || !luv) throw Status(XS_ERR_INVALID);
        Handle &h = *p->h;
        if (!p->factored || p->factor_kind == 2 || p->factor_kind >= 4) throw Status(XS_ERR_ORDER);
        h.luv.download(luv, h.nnz, h.s);
        XS_CUDA(cudaStreamSynchronize(h.s));
    });
}
int xs_plan_get_factors(xs_plan_t p, int *nnzL, int *nnzU, int *lrp, int *lci, double *lv, double *dinv, int *urp, int *uci,
                        double *uv)
{
    return guarded([&] {
        if (!p) throw Status(XS_ERR_INVALID);
        Handle &h = *p->h;
        if (!p->factored) throw Status(XS_ERR_ORDER);
        const int n = h.n;
        if (p->factor_kind == 2 || p->factor_kind >= 4) {  // own pattern
            ParilutResult &R = h.ilut;
            if (nnzL) *nnzL = (int)R.nnzL;
            if (nnzU) *nnzU = (int)R.nnzU;
            if (lrp) std::memcpy(lrp, R.hlrp.data(), sizeof(int) * (n + 1));
            if (urp) std::memcpy(urp, R.hurp.data(), sizeof(int) * (n + 1));
            if (lci) std::memcpy(lci, R.hlci.data(), sizeof(int) * R.nnzL);
            if (uci) std::memcpy(uci, R.huci.data(), sizeof(int) * R.nnzU);
            if (lv && R.nnzL) R.lv.download(lv, R.nnzL, h.s);
            if (uv && R.nnzU) R.uv.download(uv, R.nnzU, h.s);
            if (dinv) R.dinv.download(dinv, n, h.s);
            XS_CUDA(cudaStreamSynchronize(h.s));
            return;
        }
        std::vector<double> fv(h.nnz);
        h.fv.download(fv.data(), h.nnz, h.s);
        XS_CUDA(cudaStreamSynchronize(h.s));
        int nl = 0, nu = 0;
        if (lrp) lrp[0] = 0;
        if (urp) urp[0] = 0;
        for (int i = 0; i < n; i++) {
            for (int k = h.hrp[i]; k < h.hrp[i + 1]; k++) {
                int c = h.hci[k];
                if (c < i) {
                    if (lci) lci[nl] = c;
                    if (lv) lv[nl] = fv[k];
                    nl++;
                } else if (c > i) {
                    if (uci) uci[nu] = c;
                    if (uv) uv[nu] = fv[k];
                    nu++;
                } else if (dinv)
                    dinv[i] = fv[k];
            }
            if (lrp) lrp[i + 1] = nl;
            if (urp) urp[i + 1] = nu;
        }
        if (nnzL) *nnzL = nl;
        if (nnzU) *nnzU = nu;
    });
}
int xs_plan_set_factor_precision(xs_plan_t p, int prec)
{
    return guarded([&] {
        if (!p || prec < 0 || prec > 3) throw Status(XS_ERR_INVALID);
        p->h->M.factor_prec = prec;
        p->h->factor_prec = prec;
    });
}
int xs_plan_set_trsv(xs_plan_t p, int mode)
{
    return guarded([&] {
        if (!p || mode < 0 || mode > 1000) throw Status(XS_ERR_INVALID);
        Handle &h = *p->h;
        h.trsv_mode = mode;
        h.M.trsv_mode = mode;
        if (mode > 0) h.M.ensure_sweep_buffers(h.inner32 != 0);
    });
}
int xs_plan_lusolve(xs_plan_t p, int vec_prec, const void *x, void *z)
{
    return guarded([&] {
        if (!p || !x || !z) throw Status(XS_ERR_INVALID);
        Handle &h = *p->h;
        if (vec_prec == 0) plan_lusolve64(h, (const double *)x, (double *)z);
        else plan_lusolve32(h, (const float *)x, (float *)z);
    });
}
int xs_plan_lusolve_batch(xs_plan_t p, int k, const double *x, double *z)
{
    return guarded([&] {
        if (!p || !x || !z || k < 1 || k > BATCH_MAX) throw Status(XS_ERR_INVALID);
        Handle &h = *p->h;
        if (!h.M.have_factors) throw Status(XS_ERR_ORDER);
        if (!batch_precond_ok(h.M)) throw Status(XS_ERR_UNSUPPORTED);
        if (!p->zero.p) p->zero.alloc(1);
        batch_apply(h.M, p->bp, k, x, z, p->zero.p, h.s);
    });
}
int xs_plan_lusolve_t(xs_plan_t p, const double *x, double *z)
{
    return guarded([&] {
        if (!p || !x || !z) throw Status(XS_ERR_INVALID);
        Handle &h = *p->h;
        if (!h.M.have_factors) throw Status(XS_ERR_ORDER);
        adjoint_prepare(h);
        h.adj.Mt.apply<double>(x, z, nullptr, h.s);
    });
}
int xs_plan_debug_break_dependency(xs_plan_t p, int position, int enable)
{
    return guarded([&] {
        if (!p) throw Status(XS_ERR_INVALID);
        Handle &h = *p->h;
        if (!h.M.have_factors) throw Status(XS_ERR_ORDER);
        TriDev &L = h.M.L;
        if (position < 0 || position >= L.n) throw Status(XS_ERR_INVALID);
        XS_CUDA(cudaStreamSynchronize(h.s));
        if (L.tiled) {
            // box layout: the box holding `position` waits for one of its own
            // rows as if it were a halo value; that row is published only
            // after the halo wait, so the wait runs out
            static thread_local int saved_halo = 0, saved_at = -1;
            if (enable) {
                std::vector<int> tp(L.ntiles + 1);
                XS_CUDA(cudaMemcpy(tp.data(), L.t_pos.p, sizeof(int) * tp.size(), cudaMemcpyDeviceToHost));
                const int t = (int)(std::upper_bound(tp.begin(), tp.end(), position) - tp.begin()) - 1;
                int hr[2];
                XS_CUDA(cudaMemcpy(hr, L.t_hptr.p + t, sizeof(int) * 2, cudaMemcpyDeviceToHost));
                if (hr[1] <= hr[0]) throw Status(XS_ERR_INVALID);  // the box reads nothing from earlier boxes
                int row = 0;
                XS_CUDA(cudaMemcpy(&row, L.perm.p + position, sizeof(int), cudaMemcpyDeviceToHost));
                if (saved_at < 0) {
                    XS_CUDA(cudaMemcpy(&saved_halo, L.t_hrow.p + hr[0], sizeof(int), cudaMemcpyDeviceToHost));
                    saved_at = hr[0];
                }
                XS_CUDA(cudaMemcpy(L.t_hrow.p + saved_at, &row, sizeof(int), cudaMemcpyHostToDevice));
            } else if (saved_at >= 0) {
                XS_CUDA(cudaMemcpy(L.t_hrow.p + saved_at, &saved_halo, sizeof(int), cudaMemcpyHostToDevice));
                saved_at = -1;
            }
            return;
        }
        int k[2];
        XS_CUDA(cudaMemcpy(k, L.prp.p + position, sizeof(int) * 2, cudaMemcpyDeviceToHost));
        if (k[1] <= k[0]) throw Status(XS_ERR_INVALID);  // the row has no dependency to break
        int row = 0;
        XS_CUDA(cudaMemcpy(&row, L.perm.p + position, sizeof(int), cudaMemcpyDeviceToHost));
        // the saved entry may be an encoded (negative) chunk-local slot
        static thread_local int saved = 0;
        static thread_local bool have_saved = false;
        if (enable) {
            if (!have_saved) XS_CUDA(cudaMemcpy(&saved, L.pci.p + k[0], sizeof(int), cudaMemcpyDeviceToHost));
            have_saved = true;
            XS_CUDA(cudaMemcpy(L.pci.p + k[0], &row, sizeof(int), cudaMemcpyHostToDevice));  // waits on itself
        } else if (have_saved) {
            XS_CUDA(cudaMemcpy(L.pci.p + k[0], &saved, sizeof(int), cudaMemcpyHostToDevice));
            have_saved = false;
        }
    });
}
int xs_plan_get_stream(xs_plan_t p, void **stream)
{
    return guarded([&] {
        if (!p || !stream) throw Status(XS_ERR_INVALID);
        *stream = (void *)p->h->s;
    });
}
int xs_plan_sync(xs_plan_t p)
{
    return guarded([&] {
        if (!p) throw Status(XS_ERR_INVALID);
        Handle &h = *p->h;
        XS_CUDA(cudaStreamSynchronize(h.s));
        int e = read_dev_err(h);
        if (e) {
            h.M.rearm(h.s);
            clear_dev_err(h);
            XS_CUDA(cudaStreamSynchronize(h.s));
            throw Status(dev_err_to_status(e));
        }
    });
}
int xs_plan_levels(xs_plan_t p, int *lL, int *lU)
{
    return guarded([&] {
        if (!p) throw Status(XS_ERR_INVALID);
        Handle &h = *p->h;
        if (!h.M.have_factors) throw Status(XS_ERR_ORDER);
        if (lL) *lL = h.M.L.nlevels;
        if (lU) *lU = h.M.U.nlevels;
    });
}
int xs_plan_op_bytes(xs_plan_t p, int op, double *bytes)
{
    return guarded([&] {
        if (!p || !bytes) throw Status(XS_ERR_INVALID);
        Handle &h = *p->h;
        const double n = h.n, nnz = (double)h.nnz;
        const double I = 4.0;
        switch (op) {
        case 0: *bytes = (8 + I) * nnz + I * (n + 1) + 8 * n + 8 * n; break;
        // ELL: stored slots (padding included) with the stored column data:
        // a 32- or 16-bit index per slot, or (diagonal slots) no index and
        // one mask per row
        case 1: case 6: {
            const double V = op == 1 ? 8.0 : 4.0;
            const double slot = h.A.ell_dia ? V : V + (h.A.ell16 ? 2.0 : I);
            const double row = h.A.ell_dia ? (h.A.ell_w <= 8 ? 1.0 : 4.0) : 0.0;
            *bytes = slot * h.A.ell_w * n + row * n + 2 * V * n;
            break;
        }
        case 2: *bytes = (4 + I) * nnz + I * (n + 1) + 4 * n + 4 * n; break;
        case 3: case 4: case 5: {
            if (!h.M.have_factors) throw Status(XS_ERR_ORDER);
            const int fp = h.M.factor_prec;
            const double V = fp == 0 ? 8 : (fp == 1 ? 4 : 2);
            const double X = fp == 0 ? 8 : 4;  // vector element
            const int k = h.M.trsv_mode;
            if (k == 0) {
                // exact solve: factor entries + row pointers, rhs read, result written (+ dinv for U)
                const double l = (V + I) * h.M.L.nnz + I * (n + 1) + 2 * X * n;
                const double u = (V + I) * h.M.U.nnz + I * (n + 1) + 3 * X * n;
                *bytes = op == 3 ? l : (op == 4 ? u : l + u);
            } else if (k <= 1) {
                *bytes = 3 * X * n;  // z = dinv * x
            } else {
                // k Jacobi sweeps = k-1 passes per triangle.  Each pass reads
                // the triangle's entries (index width of the copy in use); the
                // first pass reads x (L) or x and dinv (U) and writes its
                // iterate, every later pass also reads the previous iterate.
                auto idx = [&](const TriDev &T) {  // index bytes per entry
                    return T.ell_w > 0 && T.ell_dia ? 0.0 : (T.ell_w > 0 && T.ell16 ? 2.0 : I);
                };
                auto msk = [&](const TriDev &T) {  // mask bytes per row
                    return T.ell_w > 0 && T.ell_dia ? (T.ell_w <= 8 ? 1.0 : 4.0) : 0.0;
                };
                const TriDev &Lt = h.M.L, &Ut = h.M.U;
                // passes over each triangle: k-1, or k-2 when sweeps 2 and 3
                // share one pass (its re-reads of neighbour rows are not
                // compulsory traffic)
                auto fusable = [&](const TriDev &T) {
                    return T.ell_w > 0 && T.ell_dia && T.ell_w <= (fp == 0 ? 3 : 4);
                };
                const bool fused = k >= 3 && fusable(Lt) && fusable(Ut) && trsv_tuning().fuse_sweeps;
                const int P = fused ? k - 2 : k - 1;
                const double l = P * ((V + idx(Lt)) * Lt.nnz + msk(Lt) * n) + 2 * X * n + (P - 1) * 3 * X * n;
                const double u = P * ((V + idx(Ut)) * Ut.nnz + msk(Ut) * n) + 3 * X * n + (P - 1) * 4 * X * n;
                *bytes = op == 3 ? l : (op == 4 ? u : l + u);
            }
            break;
        }
        default: throw Status(XS_ERR_INVALID);
        }
    });
}
int xs_plan_time_op(xs_plan_t p, int op, int reps, int flush_l2, double *ms)
{
    return guarded([&] {
        if (!p || !ms || reps < 1) throw Status(XS_ERR_INVALID);
        Handle &h = *p->h;
        const int n = h.n;
        const bool f32 = (op == 2 || op == 6) || ((op >= 3 && op <= 5) && h.M.factor_prec != FP_F64);
        if (p->bx64.n != (size_t)n) {
            p->bx64.alloc(n); p->by64.alloc(n); p->bz64.alloc(n);
            p->bx32.alloc(n); p->by32.alloc(n); p->bz32.alloc(n);
        }
        k_fill_rand<<<geom().sms * 4, 256, 0, h.s>>>(n, p->bx64.p, p->bx32.p, 12345u);
        check_launch();
        if (flush_l2 && !p->l2flush.p) p->l2flush.alloc((size_t)96 << 20);  // 2 x 384 MB, each > L2
        if (op == 1 || op == 6) {
            if (h.A.ell_w == 0) operator_build_ell(h.A, h.hrp.data(), h.hci.data(), host_vals(h), 0, f32, h.s);
        }
        if (f32) operator_ensure32(h.A, h.hrp.data(), h.s);
        h.W.ensure(64, 1);
        RedSlot sl = h.W.slot();
        auto run = [&]() {
            switch (op) {
            case 0: { int sv = h.A.format; h.A.format = 0; spmv<double, double>(h.A, p->bx64.p, p->by64.p, EpiAx<double>{}, sl, h.s); h.A.format = sv; break; }
            case 1: { int sv = h.A.format; h.A.format = 1; spmv<double, double>(h.A, p->bx64.p, p->by64.p, EpiAx<double>{}, sl, h.s); h.A.format = sv; break; }
            case 2: { int sv = h.A.format; h.A.format = 0; spmv<float, float>(h.A, p->bx32.p, p->by32.p, EpiAx<float>{}, sl, h.s); h.A.format = sv; break; }
            case 6: { int sv = h.A.format; h.A.format = 1; spmv<float, float>(h.A, p->bx32.p, p->by32.p, EpiAx<float>{}, sl, h.s); h.A.format = sv; break; }
            case 3: case 4: case 5: {
                if (!h.M.have_factors) throw Status(XS_ERR_ORDER);
                // op 3: L only (into the L buffer), op 4: U only, op 5: both
                if (!f32) h.M.apply<double>(p->bx64.p, p->bz64.p, nullptr, h.s);
                else h.M.apply<float>(p->bx32.p, p->bz32.p, nullptr, h.s);
                break;
            }
            default: throw Status(XS_ERR_INVALID);
            }
        };
        // warm-up
        run();
        run();
        XS_CUDA(cudaStreamSynchronize(h.s));
        cudaEvent_t a, b;
        XS_CUDA(cudaEventCreate(&a));
        XS_CUDA(cudaEventCreate(&b));
        double total = 0.0;
        const bool half = (op == 3 || op == 4) && h.M.trsv_mode == 0;
        for (int r = 0; r < reps; r++) {
            if (flush_l2)
                k_flush<<<geom().sms * 4, 256, 0, h.s>>>(p->l2flush.p, (long)p->l2flush.n, (double)r, p->l2flush.p);
            if (half && op == 4) {  // U alone needs a fresh L result in the L buffer
                if (!f32) h.M.apply_half<double>(0, p->bx64.p, p->bz64.p, h.s);
                else h.M.apply_half<float>(0, p->bx32.p, p->bz32.p, h.s);
            }
            XS_CUDA(cudaEventRecord(a, h.s));
            if (half) {
                if (!f32) h.M.apply_half<double>(op == 3 ? 0 : 1, p->bx64.p, p->bz64.p, h.s);
                else h.M.apply_half<float>(op == 3 ? 0 : 1, p->bx32.p, p->bz32.p, h.s);
            } else
                run();
            XS_CUDA(cudaEventRecord(b, h.s));
            if (half && op == 3) {  // finish the pair so both buffers are re-armed
                if (!f32) h.M.apply_half<double>(1, p->bx64.p, p->bz64.p, h.s);
                else h.M.apply_half<float>(1, p->bx32.p, p->bz32.p, h.s);
            }
            XS_CUDA(cudaEventSynchronize(b));
            float t = 0;
            cudaEventElapsedTime(&t, a, b);
            total += t;
        }
        cudaEventDestroy(a);
        cudaEventDestroy(b);
        *ms = total / reps;
        int e = read_dev_err(h);
        if (e) {
            h.M.rearm(h.s);
            clear_dev_err(h);
            throw Status(dev_err_to_status(e));
        }
    });
}

}  // extern "C"
