// libxsolver_b200: handle, matrix/preconditioner setup and the C API.
//
// Reference interfaces replaced here (paths relative to the reference root):
//   hip/xsolver_c.cpp:41-333       setter-style API over process globals
//   intel/HostMatrix.h:187-222     cpu_mat_setup / preconditioner setup
//   cuda/DeviceMatrix.h:121-169    gpu_mat_setup / gpu_mat_format / ...
//   cuda/mpicudasolver-C-v1.cu     gpu_*_solve
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "xs_internal.cuh"
#include "xs_spmv.cuh"
#include "xs_trsv.cuh"
#include "xs_factor.cuh"
#include "xs_precond.cuh"
#include "xs_krylov.cuh"
#include "xs_solvers.cuh"
#include "xs_gmres.cuh"
#include "xs_parilut.cuh"
#include "xs_adjoint.cuh"
#include "xs_batch.cuh"
#include "xs_mtx.cuh"
#include "xs_hostilu.h"

namespace xs {

Geom &geom()
{
    static Geom g;
    static bool init = false;
    if (!init) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceProp p;
        if (cudaGetDeviceProperties(&p, dev) == cudaSuccess) {
            g.sms = p.multiProcessorCount;
            // CTAs per SM of the vector-op reductions (environment
            // XS_RED_CTAS_PER_SM, 1-8; default 8: full occupancy)
            int k = 8;
            if (const char *e = getenv("XS_RED_CTAS_PER_SM")) k = std::max(1, std::min(8, atoi(e)));
            g.red_grid = k * g.sms;
        }
        init = true;
    }
    return g;
}

PdlTuning &pdl_tuning()
{
    static PdlTuning t;
    static bool init = false;
    if (!init) {
        if (const char *e = getenv("XS_PDL")) t.enabled = atoi(e) != 0;
        init = true;
    }
    return t;
}

FormatTuning &format_tuning()
{
    static FormatTuning t;
    static bool init = false;
    if (!init) {
        if (const char *e = getenv("XS_ELL_INDEX16")) t.ell_index16 = atoi(e) != 0;
        if (const char *e = getenv("XS_ELL_DIAGONAL")) t.ell_dia = atoi(e) != 0;
        init = true;
    }
    return t;
}

BatchTuning &batch_tuning()
{
    static BatchTuning t = [] {
        BatchTuning b;
        if (const char *e = getenv("XS_BATCH")) b.enabled = atoi(e) != 0;
        return b;
    }();
    return t;
}

PersistTuning &persist_tuning()
{
    static PersistTuning t = [] {
        PersistTuning q;
        if (const char *e = getenv("XS_PERSIST")) q.enabled = atoi(e) != 0;
        return q;
    }();
    return t;
}

bool &vec_fusion_flag()
{
    static bool on = [] {
        const char *e = getenv("XS_VEC_FUSE");
        return !(e && atoi(e) == 0);
    }();
    return on;
}

// box-scheduled exact ILU(0) (1) or the level-ordered lane groups (0,
// default: at 128^3 7-point the box kernel took 10.1 ms against 4.6 ms,
// each internal level paying global-memory latency for the halo rows' upper
// parts and the dependency lookups); environment XS_ILU_TILES at first use
static int &ilu_tiles_flag()
{
    static int f = [] {
        const char *e = getenv("XS_ILU_TILES");
        return e ? (atoi(e) != 0) : 0;
    }();
    return f;
}

TileTuning &tile_tuning()
{
    static TileTuning t;
    static bool init = false;
    if (!init) {
        // XS_TRSV_TILES: "0" keeps the level-ordered solve; "tx,ty,tz" sets the box size
        if (const char *e = getenv("XS_TRSV_TILES")) {
            int a = 0, b = 0, c = 0;
            const int k = sscanf(e, "%d,%d,%d", &a, &b, &c);
            if (k == 1 && a == 0) t.enable = 0;
            else if (k == 3 && a > 0 && b > 0 && c > 0) { t.enable = 1; t.tx = a; t.ty = b; t.tz = c; t.user_box = 1; }
        }
        if (const char *e = getenv("XS_TRSV_TILE_MIN_ROWS")) t.min_rows = std::max(8, atoi(e));
        if (const char *e = getenv("XS_TRSV_TILE_BLOCKS_PER_SM")) t.blocks_per_sm = std::max(1, atoi(e));
        init = true;
    }
    return t;
}

TrsvTuning &trsv_tuning()
{
    static TrsvTuning t;
    static bool init = false;
    if (!init) {
        if (const char *e = getenv("XS_TRSV_BLOCKS_PER_SM")) t.blocks_per_sm = atoi(e);
        if (const char *e = getenv("XS_TRSV_BACKOFF_NS")) t.backoff_ns = std::max(8, atoi(e));
        if (const char *e = getenv("XS_TRSV_CHUNK_ROWS")) t.chunk_rows = std::max(0, atoi(e));
        if (const char *e = getenv("XS_TRSV_BLOCK_ROWS")) t.block_max_rows = std::max(0, atoi(e));
        if (const char *e = getenv("XS_SWEEP_FUSE")) t.fuse_sweeps = atoi(e) != 0;
        if (const char *e = getenv("XS_LU_STAGED")) t.lu_staged = atoi(e) != 0;
        if (const char *e = getenv("XS_SWEEP_BALANCED")) t.balanced_sweep_grid = atoi(e) != 0;
        if (const char *e = getenv("XS_LU_BATCH")) {  // "rows,entries,buffers"
            int r = 0, en = 0, b = 0;
            if (sscanf(e, "%d,%d,%d", &r, &en, &b) == 3 && r >= 32 && en >= 32 && b >= 2 && b <= LUB_MAX_BUFS) {
                t.lub_rows = r;
                t.lub_entries = en;
                t.lub_bufs = b;
                t.lub_auto = 0;
            }
        }
        if (const char *e = getenv("XS_LU_STAGED_THREADS")) {
            const int v = atoi(e);
            t.lu_staged_threads = v >= 32 && v <= LU_BLOCK_THREADS && v % 32 == 0 ? v : 0;
        }
        init = true;
    }
    return t;
}

// ---------------------------------------------------------------- operator setup
__global__ void k_convert_f32(long m, const double *__restrict__ a, float *__restrict__ b)
{
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < m; i += (long)gridDim.x * blockDim.x) b[i] = (float)a[i];
}

void operator_setup(Operator &op, int n, const int *h_rp, const int *h_ci, const double *h_v, int base, bool want32,
                    cudaStream_t s, int *d_err)
{
    op.n = n;
    op.nnz = h_rp[n] - h_rp[0];
    op.err = d_err;
    std::vector<int> rp0(n + 1);
    for (int i = 0; i <= n; i++) rp0[i] = h_rp[i] - base;
    op.rp.alloc(n + 1);
    op.rp.upload(rp0.data(), n + 1, s);
    op.ci.alloc(op.nnz, 8);
    if (base == 0) op.ci.upload(h_ci, op.nnz, s);
    else {
        std::vector<int> c(op.nnz);
        for (long k = 0; k < op.nnz; k++) c[k] = h_ci[k] - base;
        op.ci.upload(c.data(), op.nnz, s);
        XS_CUDA(cudaStreamSynchronize(s));
    }
    op.v.alloc(op.nnz, 8);
    op.v.upload(h_v, op.nnz, s);
    build_tiling(rp0.data(), n, SPMV_THREADS, spmv_cap<double>(), op.tile64, s);
    if (want32) {
        op.v32.alloc(op.nnz, 8);
        k_convert_f32<<<geom().sms * 4, 256, 0, s>>>(op.nnz, op.v.p, op.v32.p);
        check_launch();
        build_tiling(rp0.data(), n, SPMV_THREADS, spmv_cap<float>(), op.tile32, s);
    }
    XS_CUDA(cudaStreamSynchronize(s));
}

void operator_ensure32(Operator &op, const int *rp0, cudaStream_t s)
{
    if (op.v32.p) return;
    op.v32.alloc(op.nnz, 8);
    k_convert_f32<<<geom().sms * 4, 256, 0, s>>>(op.nnz, op.v.p, op.v32.p);
    check_launch();
    build_tiling(rp0, op.n, SPMV_THREADS, spmv_cap<float>(), op.tile32, s);
    if (op.ell_w > 0 && !op.ev32.p) {
        const long m = (long)op.ell_w * ell_ld(op.n);
        op.ev32.alloc(m);
        k_convert_f32<<<geom().sms * 4, 256, 0, s>>>(m, op.ev.p, op.ev32.p);
        check_launch();
    }
}

// Diagonal-slot eligibility of a CSR pattern: the ascending list of distinct
// offsets c - row if there are at most ELL_DIA_MAX of them and the slots
// would hold at most 25% padding; empty otherwise.
std::vector<int> dia_offsets(int n, const int *rp, const int *ci)
{
    if (!format_tuning().ell_dia || n <= 0) return {};
    const long nnz = (long)rp[n] - rp[0];
    // slot count allowed: ELL_DIA_MAX, and slots * n <= nnz + nnz / 4
    const long cap = std::min<long>(ELL_DIA_MAX, (nnz + nnz / 4) / n);
    if (cap <= 0) return {};
    auto add_row = [&](std::vector<int> &offs, long i) {
        for (int q = rp[i]; q < rp[i + 1]; q++) {
            const int o = ci[q] - (int)i;
            auto it = std::lower_bound(offs.begin(), offs.end(), o);
            if (it == offs.end() || *it != o) {
                offs.insert(it, o);
                if ((long)offs.size() > cap) return false;
            }
        }
        return true;
    };
    // a sample of rows: its offsets are a subset of all of them, so a sample
    // over the cap rejects without the full scan
    {
        std::vector<int> offs;
        const long S = std::min(n, 4096);
        for (long t = 0; t < S; t++)
            if (!add_row(offs, (long)n * t / S)) return {};
    }
    // every row, in ranges over host threads; the union of the range sets
    std::vector<std::vector<int>> part(16);
    std::vector<char> ok(16, 1);
    const int T = host_parallel_rows(n, [&](long lo, long hi, int t) {
        for (long i = lo; i < hi; i++)
            if (!add_row(part[t], i)) {
                ok[t] = 0;
                return;
            }
    });
    std::vector<int> offs;
    for (int t = 0; t < T; t++) {
        if (!ok[t]) return {};
        for (int o : part[t]) {
            auto it = std::lower_bound(offs.begin(), offs.end(), o);
            if (it == offs.end() || *it != o) offs.insert(it, o);
        }
        if ((long)offs.size() > cap) return {};
    }
    return offs;
}

// largest |c - row| over a CSR pattern (host threads)
long max_col_offset(int n, const int *rp, const int *ci)
{
    std::vector<long> part(16, 0);
    const int T = host_parallel_rows(n, [&](long lo, long hi, int t) {
        long m = 0;
        for (long i = lo; i < hi; i++)
            for (int q = rp[i]; q < rp[i + 1]; q++) m = std::max(m, std::labs((long)ci[q] - i));
        part[t] = m;
    });
    return *std::max_element(part.begin(), part.begin() + T);
}

void operator_build_ell(Operator &op, const int *rp0, const int *ci0, const double *v, int, bool want32, cudaStream_t s)
{
    int n = op.n, w = 0;
    for (int i = 0; i < n; i++) w = std::max(w, rp0[i + 1] - rp0[i]);
    const long ld = ell_ld(n);
    const std::vector<int> offs = dia_offsets(n, rp0, ci0);
    op.ell_dia = !offs.empty();
    op.eci.free();
    op.eco.free();
    op.emask8.free();
    op.emask32.free();
    op.doff.free();
    if (op.ell_dia) {
        // slot = diagonal; mask bit k = slot k present in the row
        w = (int)offs.size();
        op.ell_w = w;
        op.ell16 = false;
        const size_t m = (size_t)w * ld;
        std::vector<double> vv(m, 0.0);
        std::vector<uint32_t> mask(ld, 0u);
        for (int i = 0; i < n; i++)
            for (int q = rp0[i]; q < rp0[i + 1]; q++) {
                const int k = (int)(std::lower_bound(offs.begin(), offs.end(), ci0[q] - i) - offs.begin());
                vv[(size_t)k * ld + i] = v[q];
                mask[i] |= 1u << k;
            }
        op.doff.alloc(w);
        op.doff.upload(offs.data(), w, s);
        if (w <= 8) {
            std::vector<uint8_t> m8(mask.begin(), mask.end());
            op.emask8.alloc(ld);
            op.emask8.upload(m8.data(), ld, s);
        } else {
            op.emask32.alloc(ld);
            op.emask32.upload(mask.data(), ld, s);
        }
        op.ev.alloc(m);
        op.ev.upload(vv.data(), m, s);
    } else {
        op.ell_w = w;
        const long maxoff = max_col_offset(n, rp0, ci0);
        op.ell16 = format_tuning().ell_index16 && maxoff <= 32767;
        const size_t m = (size_t)w * ld;
        // padding slots of a row point at the row itself (offset 0) with
        // value 0; padding rows n..ld-1 are never gathered
        std::vector<int> c(m, 0);
        std::vector<double> vv(m, 0.0);
        for (int i = 0; i < n; i++) {
            int k = 0;
            for (int q = rp0[i]; q < rp0[i + 1]; q++, k++) {
                c[(size_t)k * ld + i] = ci0[q];
                vv[(size_t)k * ld + i] = v[q];
            }
            for (; k < w; k++) c[(size_t)k * ld + i] = i;
        }
        if (op.ell16) {
            std::vector<short> o(m, 0);
            for (int i = 0; i < n; i++)
                for (int k = 0; k < w; k++) o[(size_t)k * ld + i] = (short)(c[(size_t)k * ld + i] - i);
            op.eco.alloc(m);
            op.eco.upload(o.data(), m, s);
        } else {
            op.eci.alloc(m);
            op.eci.upload(c.data(), m, s);
        }
        op.ev.alloc(m);
        op.ev.upload(vv.data(), m, s);
    }
    if (want32) {
        const long m = (long)op.ell_w * ld;
        op.ev32.alloc(m);
        k_convert_f32<<<geom().sms * 4, 256, 0, s>>>(m, op.ev.p, op.ev32.p);
        check_launch();
    } else {
        op.ev32.free();
    }
    // one wave of resident CTAs (the fused reductions' partial count follows
    // the grid, which is fixed per operator)
    op.ell_grid = (int)std::min<long>((long)geom().sms * ELL_MIN_BLOCKS, (n + 256L * ELL_ROWS - 1) / (256L * ELL_ROWS));
    if (op.ell_grid < 1) op.ell_grid = 1;
    XS_CUDA(cudaStreamSynchronize(s));
}

// new values for an existing ELL copy: slot k of row r is the row's k-th
// CSR entry (0 past the row's end), as operator_build_ell lays it out
// (diagonal slots, doff != null: the entry at column c goes to the slot of
// offset c - r; absent slots keep 0)
__global__ void k_ell_refill(int n, int w, long ld, const int *__restrict__ rp, const int *__restrict__ ci,
                             const double *__restrict__ v, const int *__restrict__ doff, double *ev, float *ev32)
{
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
        const int k0 = rp[r], len = rp[r + 1] - k0;
        if (!doff) {
            for (int k = 0; k < w; k++) {
                const double val = k < len ? v[k0 + k] : 0.0;
                ev[(long)k * ld + r] = val;
                if (ev32) ev32[(long)k * ld + r] = (float)val;
            }
        } else {
            for (int q = 0; q < len; q++) {
                const int off = ci[k0 + q] - r;
                int k = 0;
                while (k < w - 1 && doff[k] != off) k++;
                ev[(long)k * ld + r] = v[k0 + q];
                if (ev32) ev32[(long)k * ld + r] = (float)v[k0 + q];
            }
        }
    }
}

// ---------------------------------------------------------------- handle
struct Handle {
    cudaStream_t s = nullptr;
    DBuf<int> err;
    int n = 0;
    long nnz = 0;
    std::vector<int> hrp, hci;  // 0-based host copy
    std::vector<double> hv;
    // caller entry of each stored entry when set_matrix had to sort a row's
    // columns (empty: stored order = caller order)
    std::vector<long> vperm;
    bool hv_stale = false;  // hv lags the device values (xs_mat_update uploads directly)
    Operator A;
    bool have_matrix = false;
    int format = 0;
    // pattern analysis of A for factorisations
    bool analysed = false;
    std::vector<int> huptr;
    DBuf<int> uptr, rowof, ucp, ucpos, flags;
    DBuf<int> tpos;          // IC(0): position of the transposed entry (-1: none)
    DBuf<double> ic0_tnorm;  // IC(0): droptol * row norms
    int ilu_epoch = 0;
    int max_row_len = -1;  // longest row of the pattern (-1: not yet counted)
    DBuf<unsigned> fticket;
    // box-scheduled exact ILU(0) on the L solve's boxes (k_ilu0_tiles: the
    // arrays of IluTileArgs); built with the pattern analysis when L has
    // boxes whose entries fit in shared memory
    bool ilu_tiles = false, ilu_tiles_built = false;
    size_t ilu_tiles_smem = 0;
    int ilu_max_entries = 0, ilu_max_lower = 0, ilu_max_rows = 0;
    DBuf<int> ilu_ebase, ilu_ent, ilu_roff, ilu_rdiag, ilu_lbase, ilu_loff, ilu_dep;
    TriHostPlan hL, hU;
    DBuf<double> luv, fv, tmpv;
    DBuf<long> udiag_src;
    // preconditioner
    PrecondDev M;
    int pc_req = -1;  // requested type (-1 unset)
    bool pc_ready = false;
    int parilu_sweeps = 20;
    double parilut_fill = 3.0;
    int parilut_sweeps = 10;
    double parilut_droptol = 0.0;
    // host threshold factorizations: Saad ILUT (hip/Precond/precon_ilup.h:
    // 17-24 defaults) and ICT (hip/Precond/precon_ict.h:14-16)
    int ilup_fill = 20;
    double ilup_tol = 1e-5;
    int ict_fill = 100;
    double ict_tol = 1e-8;
    int trsv_mode = 0;
    ParilutResult ilut;  // factors on their own pattern (ParILUT, ILUT, ICT)
    // solver
    int method = 0;
    double tol = 1e-8, abstol = 0.0;
    int maxiter = 1000, restart = 30;
    int *usediter = nullptr;
    double *resvec = nullptr;
    int intel_conv = 0;  // 1: gpu_* conventions
    int quirk = 0;
    // precision
    int inner32 = 0;
    // plans keep every storage precision and layout of the factors (their
    // callers switch precision and triangular-solve mode after factorising);
    // handles build only what their configured solve reads
    bool all_factor_copies = false;
    int factor_prec = FP_F64;
    double inner_rtol = 1e-4;
    int inner_maxiter = 200;
    // mixed BiCGSTAB: refinement steps continue one inner iteration (true
    // residual replaced at each step) instead of restarting it
    int carry_krylov = 1;
    int last_outer = 0;
    // work
    Workspace W;
    RunSet<double> r64;
    RunSet<float> r32;
    VecPool<double> vpool64;
    VecPool<float> vpool32;
    // results
    double setup_ms = 0, solve_ms = 0, final_relres = 0;
    int last_iters = 0;
    long long launches = 0;  // kernels launched by the last solve (graph nodes + direct)
    // adjoint
    AdjointState adj;
    DBuf<OuterState> outer_st;
    bool have_solution = false;
    // several right-hand sides at once (xs_solve_batch, xs_adjoint_batch)
    BatchRuntime batch;

    Handle()
    {
        XS_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
        err.alloc(1);
        fticket.alloc(1);
        M.err = err.p;
    }
    ~Handle()
    {
        cudaStreamSynchronize(s);
        cudaStreamDestroy(s);
    }
};

static int read_dev_err(Handle &h)
{
    int e = 0;
    XS_CUDA(cudaMemcpyAsync(&e, h.err.p, sizeof(int), cudaMemcpyDeviceToHost, h.s));
    XS_CUDA(cudaStreamSynchronize(h.s));
    return e;
}
static void clear_dev_err(Handle &h) { XS_CUDA(cudaMemsetAsync(h.err.p, 0, sizeof(int), h.s)); }

static void invalidate_pc(Handle &h)
{
    h.pc_ready = false;
    h.M.have_factors = false;
    h.adj.have_Mt = false;
}

static void set_matrix(Handle &h, int n, const int *rp, const int *ci, const double *v, int format)
{
    if (n <= 0 || !rp || !ci || !v) throw Status(XS_ERR_INVALID);
    int base = rp[0];
    if (base != 0 && base != 1) throw Status(XS_ERR_INVALID);
    long nnz = (long)rp[n] - base;
    if (nnz < 0 || nnz > 0x7fffffffL - 16) throw Status(XS_ERR_INVALID);
    // Checked and sorted into locals first: a rejected pattern leaves the
    // handle's previous matrix (host copy, device operator, factors) intact.
    std::vector<int> hrp(n + 1), hci(nnz);
    std::vector<double> hv(v, v + nnz);
    std::vector<long> vperm;
    for (int i = 0; i <= n; i++) hrp[i] = rp[i] - base;
    for (int i = 0; i < n; i++) {
        // a row end past rp[n] would read beyond the caller's column array
        if (hrp[i + 1] < hrp[i] || hrp[i + 1] > nnz) throw Status(XS_ERR_INVALID);
        for (int k = hrp[i]; k < hrp[i + 1]; k++) {
            int c = ci[k] - base;
            if (c < 0 || c >= n) throw Status(XS_ERR_INVALID);
            hci[k] = c;
        }
        // columns must be sorted within a row (the reference requires it for
        // its ILU merges; sort here if the caller did not)
        bool sorted = true;
        for (int k = hrp[i] + 1; k < hrp[i + 1]; k++)
            if (hci[k] <= hci[k - 1]) { sorted = false; break; }
        if (!sorted) {
            if (vperm.empty()) {
                vperm.resize(nnz);
                for (long k = 0; k < nnz; k++) vperm[k] = k;
            }
            std::vector<std::pair<int, long>> e;
            for (int k = hrp[i]; k < hrp[i + 1]; k++) e.emplace_back(hci[k], (long)k);
            // stable: entries with the same column keep the caller's order
            std::stable_sort(e.begin(), e.end(), [](auto &a, auto &b) { return a.first < b.first; });
            for (size_t q = 0; q < e.size(); q++) {
                hci[hrp[i] + q] = e[q].first;
                hv[hrp[i] + q] = v[e[q].second];
                vperm[hrp[i] + q] = e[q].second;
            }
        }
    }
    // From here on the handle holds the new pattern; until the device
    // operator is complete it reports no matrix.
    h.have_matrix = false;
    h.analysed = false;
    h.have_solution = false;
    h.adj.reset();
    invalidate_pc(h);
    h.n = n;
    h.nnz = nnz;
    h.hrp.swap(hrp);
    h.hci.swap(hci);
    h.hv.swap(hv);
    h.vperm.swap(vperm);
    h.hv_stale = false;
    h.A = Operator();
    operator_setup(h.A, n, h.hrp.data(), h.hci.data(), h.hv.data(), 0, false, h.s, h.err.p);
    h.format = format;
    if (format == 1) operator_build_ell(h.A, h.hrp.data(), h.hci.data(), h.hv.data(), 0, false, h.s);
    h.A.format = format == 1 ? 1 : 0;
    h.have_matrix = true;
    h.analysed = false;
    h.have_solution = false;
    h.adj.reset();
    invalidate_pc(h);
}

// host copy of A's values (refreshed from the device after xs_mat_update)
static const double *host_vals(Handle &h)
{
    if (h.hv_stale) {
        h.A.v.download(h.hv.data(), h.nnz, h.s);
        XS_CUDA(cudaStreamSynchronize(h.s));
        h.hv_stale = false;
    }
    return h.hv.data();
}

// values changed, same pattern
static void update_values(Handle &h, const double *v)
{
    Trace tr("update_values", h.s);
    if (!h.have_matrix) throw Status(XS_ERR_ORDER);
    if (!v) throw Status(XS_ERR_INVALID);
    if (h.vperm.empty()) {
        // straight from the caller's buffer (a DMA when it is pinned); the
        // host copy is refreshed only if host-side code needs it later
        h.A.v.upload(v, h.nnz, h.s);
        h.hv_stale = true;
    } else {
        for (long k = 0; k < h.nnz; k++) h.hv[k] = v[h.vperm[k]];
        h.A.v.upload(h.hv.data(), h.nnz, h.s);
        h.hv_stale = false;
    }
    if (h.A.v32.p) {
        k_convert_f32<<<geom().sms * 4, 256, 0, h.s>>>(h.nnz, h.A.v.p, h.A.v32.p);
        check_launch();
    }
    if (h.A.ell_w > 0) {
        if (h.A.v32.p && !h.A.ev32.p) h.A.ev32.alloc((size_t)h.A.ell_w * ell_ld(h.n));
        k_ell_refill<<<geom().sms * 4, 256, 0, h.s>>>(h.n, h.A.ell_w, ell_ld(h.n), h.A.rp.p, h.A.ci.p, h.A.v.p,
                                                      h.A.ell_dia ? h.A.doff.p : nullptr, h.A.ev.p,
                                                      h.A.v32.p ? h.A.ev32.p : nullptr);
        check_launch();
    }
    XS_CUDA(cudaStreamSynchronize(h.s));
    h.adj.reset();
    h.have_solution = false;  // the last solution solved the old values
    invalidate_pc(h);
}

// pattern analysis: diagonal positions, triangle plans, ParILU column maps
// the box-scheduled ILU(0)'s arrays (see k_ilu0_tiles) from L's boxes
static void build_ilu_tiles(Handle &h)
{
    h.ilu_tiles = false;
    for (DBuf<int> *b : {&h.ilu_ebase, &h.ilu_ent, &h.ilu_roff, &h.ilu_rdiag, &h.ilu_lbase, &h.ilu_loff, &h.ilu_dep})
        b->free();
    const TriDev &L = h.M.L;
    if (!L.tiled || L.ntiles <= 0) return;
    const int n = h.n, nt = L.ntiles;
    std::vector<int> perm(n), tpos(nt + 1);
    L.perm.download(perm.data(), n, h.s);
    L.t_pos.download(tpos.data(), nt + 1, h.s);
    XS_CUDA(cudaStreamSynchronize(h.s));
    const int *rp = h.hrp.data(), *ci = h.hci.data();
    std::vector<int> ebase(nt + 1, 0), lbase(nt + 1, 0), roff(n), rdiag(n), loff(n), box_of(n), local_of(n);
    int max_e = 0, max_l = 0, max_r = 0;
    for (int t = 0; t < nt; t++) {
        int o = 0, ol = 0;
        for (int p = tpos[t]; p < tpos[t + 1]; p++) {
            const int i = perm[p];
            roff[p] = o;
            rdiag[p] = h.huptr[i] - rp[i];
            loff[p] = ol;
            box_of[i] = t;
            local_of[i] = p - tpos[t];
            o += rp[i + 1] - rp[i];
            ol += h.huptr[i] - rp[i];
        }
        ebase[t + 1] = ebase[t] + o;
        lbase[t + 1] = lbase[t] + ol;
        max_e = std::max(max_e, o);
        max_l = std::max(max_l, ol);
        max_r = std::max(max_r, tpos[t + 1] - tpos[t]);
    }
    if (IluTileSmem::of(max_e, max_l, max_r).total > ILU_TILE_SMEM_MAX) return;
    std::vector<int> ent(std::max<long>(h.nnz, 1)), dep(std::max(lbase[nt], 1), -1);
    for (int t = 0; t < nt; t++)
        for (int p = tpos[t]; p < tpos[t + 1]; p++) {
            const int i = perm[p];
            const int e0 = ebase[t] + roff[p], l0 = lbase[t] + loff[p];
            for (int k = rp[i]; k < rp[i + 1]; k++) {
                ent[e0 + (k - rp[i])] = k;
                if (k < h.huptr[i] && box_of[ci[k]] == t) dep[l0 + (k - rp[i])] = local_of[ci[k]];
            }
        }
    auto up = [&](DBuf<int> &b, const std::vector<int> &v) {
        b.alloc(v.size());
        b.upload(v.data(), v.size(), h.s);
    };
    up(h.ilu_ebase, ebase);
    up(h.ilu_ent, ent);
    up(h.ilu_roff, roff);
    up(h.ilu_rdiag, rdiag);
    up(h.ilu_lbase, lbase);
    up(h.ilu_loff, loff);
    up(h.ilu_dep, dep);
    XS_CUDA(cudaStreamSynchronize(h.s));  // the host arrays go out of scope
    h.ilu_max_entries = max_e;
    h.ilu_max_lower = max_l;
    h.ilu_max_rows = max_r;
    h.ilu_tiles_smem = IluTileSmem::of(max_e, max_l, max_r).total;
    h.ilu_tiles = true;
}

// row of every entry (ParILU, IC(0) split) and, with columns, the U part by
// columns (rows ascending, diagonal last; ParILU) of the analysed pattern
static void ensure_entry_maps(Handle &h, bool columns)
{
    const int n = h.n;
    const int *rp = h.hrp.data(), *ci = h.hci.data();
    std::vector<int> rowof;
    if (!h.rowof.p || (columns && !h.ucp.p)) {
        rowof.resize(h.nnz);
        for (int i = 0; i < n; i++)
            for (int k = rp[i]; k < rp[i + 1]; k++) rowof[k] = i;
    }
    if (!h.rowof.p) {
        h.rowof.alloc(std::max<long>(h.nnz, 1));
        h.rowof.upload(rowof.data(), h.nnz, h.s);
    }
    if (columns && !h.ucp.p) {
        std::vector<int> ucp(n + 1, 0), ucpos;
        for (long k = 0; k < h.nnz; k++)
            if (rowof[k] <= ci[k]) ucp[ci[k] + 1]++;
        for (int j = 0; j < n; j++) ucp[j + 1] += ucp[j];
        ucpos.resize(ucp[n]);
        std::vector<int> pos(ucp.begin(), ucp.end() - 1);
        for (long k = 0; k < h.nnz; k++)
            if (rowof[k] <= ci[k]) ucpos[pos[ci[k]]++] = (int)k;
        h.ucp.alloc(n + 1);
        h.ucp.upload(ucp.data(), n + 1, h.s);
        h.ucpos.alloc(std::max<size_t>(ucpos.size(), 1));
        h.ucpos.upload(ucpos.data(), ucpos.size(), h.s);
    }
    XS_CUDA(cudaStreamSynchronize(h.s));  // the host arrays go out of scope
}

static void analyse_pattern(Handle &h)
{
    if (h.analysed) return;
    h.tpos.free();  // IC(0) transpose map of the previous pattern
    const int n = h.n;
    const int *rp = h.hrp.data(), *ci = h.hci.data();
    // diagonal positions and the strict triangles' row counts (rows in
    // parallel blocks), then the triangles as CSR with source indices into
    // A's value array
    h.huptr.assign(n, -1);
    std::vector<int> lrp(n + 1, 0), urp(n + 1, 0);
    const long RB = 65536;
    host_parallel_for((n + RB - 1) / RB, 1, [&](long b) {
        const int i1 = (int)std::min<long>(n, (b + 1) * RB);
        for (int i = (int)(b * RB); i < i1; i++) {
            int nl = 0, nu = 0;
            for (int k = rp[i]; k < rp[i + 1]; k++) {
                if (ci[k] < i) nl++;
                else if (ci[k] > i) nu++;
                else h.huptr[i] = k;
            }
            lrp[i + 1] = nl;
            urp[i + 1] = nu;
        }
    });
    for (int i = 0; i < n; i++)
        if (h.huptr[i] < 0) throw Status(XS_ERR_NO_DIAG);
    for (int i = 0; i < n; i++) {
        lrp[i + 1] += lrp[i];
        urp[i + 1] += urp[i];
    }
    // written in full by the row blocks below: no serial zero fill
    HostArray<int> lci(lrp[n]), uci(urp[n]);
    HostArray<long> lsrc(lrp[n]), usrc(urp[n]);
    host_parallel_for((n + RB - 1) / RB, 1, [&](long b) {
        const int i1 = (int)std::min<long>(n, (b + 1) * RB);
        for (int i = (int)(b * RB); i < i1; i++) {
            int ol = lrp[i], ou = urp[i];
            for (int k = rp[i]; k < rp[i + 1]; k++) {
                if (ci[k] < i) {
                    lci[ol] = ci[k];
                    lsrc[ol++] = k;
                } else if (ci[k] > i) {
                    uci[ou] = ci[k];
                    usrc[ou++] = k;
                }
            }
        }
    });
    host_both([&] { build_tri_dev(h.M.L, n, lrp, lci, false, [&](int k) { return lsrc[k]; }, h.s); },
              [&] { build_tri_dev(h.M.U, n, urp, uci, true, [&](int k) { return usrc[k]; }, h.s); });
    h.uptr.alloc(n);
    h.uptr.upload(h.huptr.data(), n, h.s);
    h.rowof.free();  // row of each entry and U by columns: built when a factorisation needs them
    h.ucp.free();
    h.ucpos.free();
    std::vector<long> ud(n);
    for (int i = 0; i < n; i++) ud[i] = h.huptr[i];
    h.udiag_src.alloc(n);
    h.udiag_src.upload(ud.data(), n, h.s);
    h.flags.alloc(n);
    h.ilu_epoch = 0;
    h.max_row_len = -1;
    h.ilu_tiles = false;
    h.ilu_tiles_built = false;  // the box ILU(0)'s arrays: built on first use
    XS_CUDA(cudaStreamSynchronize(h.s));
    h.analysed = true;
}

// Which copies of the factor values the configured solve reads: position
// order for the exact solves (trsv_mode 0), the ELL copy for the Jacobi
// sweeps, the natural-order CSR for sweeps on a triangle without an ELL
// copy; FP64 always, and with FP32 inner solves the one reduced precision
// the factors are stored in (red: bit 0 FP32, bit 1 BF16, bit 2 FP16).
struct FactorCopies {
    bool pos = true, ell = true, nat = true;
    unsigned red = 7u;
};
static FactorCopies factor_copies(const Handle &h, bool need32)
{
    FactorCopies c;
    if (!need32) c.red = 0u;
    if (h.all_factor_copies) return c;
    c.pos = h.trsv_mode == 0;
    c.ell = h.trsv_mode > 0;
    c.nat = h.trsv_mode > 0;  // per triangle: only without an ELL copy
    if (need32) c.red = h.factor_prec == FP_BF16 ? 2u : h.factor_prec == FP_F16 ? 4u : 1u;
    return c;
}

// gather factor values (from an array over A's pattern) into the storage
// precisions and layouts of `c`
static void load_tri_values(Handle &h, TriDev &T, const double *vals, const FactorCopies &c)
{
    const int g = geom().sms * 4;
    const long m = std::max<long>(T.nnz, 1);
    const bool pos = c.pos, nat = c.nat && (h.all_factor_copies || T.ell_w == 0);
    auto one = [&](auto &pbuf, auto &nbuf) {
        using FT = std::remove_pointer_t<decltype(pbuf.p)>;
        if (pos) {
            if (pbuf.n != (size_t)m) pbuf.alloc(m, 8);  // padded: the box solve stages whole 4-byte words
            if (T.nnz) k_gather_convert<FT><<<g, 256, 0, h.s>>>(T.nnz, T.src.p, vals, pbuf.p);
        } else {
            pbuf.free();
        }
        if (nat) {
            if (nbuf.n != (size_t)m) nbuf.alloc(m);
            if (T.nnz) k_gather_convert<FT><<<g, 256, 0, h.s>>>(T.nnz, T.src_nat.p, vals, nbuf.p);
        } else {
            nbuf.free();
        }
    };
    one(T.pv64, T.nv64);
    if (c.red & 1u) one(T.pv32, T.nv32); else { T.pv32.free(); T.nv32.free(); }
    if (c.red & 2u) one(T.pvbf, T.nvbf); else { T.pvbf.free(); T.nvbf.free(); }
    if (c.red & 4u) one(T.pvh, T.nvh); else { T.pvh.free(); T.nvh.free(); }
    check_launch();
}

static void load_dinv(Handle &h, const double *vals, const long *diagsrc, bool need32)
{
    const int g = geom().sms * 4;
    TriDev &U = h.M.U;
    if (U.dinv64.n != (size_t)h.n) { U.dinv64.alloc(h.n, 4); U.dinv64_nat.alloc(h.n); }
    k_gather_dinv<double><<<g, 256, 0, h.s>>>(h.n, U.perm.p, diagsrc, vals, U.dinv64.p);
    k_gather_dinv<double><<<g, 256, 0, h.s>>>(h.n, nullptr, diagsrc, vals, U.dinv64_nat.p);
    if (need32) {
        if (U.dinv32.n != (size_t)h.n) { U.dinv32.alloc(h.n, 4); U.dinv32_nat.alloc(h.n); }
        k_gather_dinv<float><<<g, 256, 0, h.s>>>(h.n, U.perm.p, diagsrc, vals, U.dinv32.p);
        k_gather_dinv<float><<<g, 256, 0, h.s>>>(h.n, nullptr, diagsrc, vals, U.dinv32_nat.p);
    }
    check_launch();
}

// IC(0) needs a symmetric pattern: the upper entries take their values from
// the transposed lower ones (the reference's seqic0 builds U as L's
// transpose, which is the upper pattern of A only when A's pattern is
// symmetric)
constexpr double IC0_SMALLNUM = 1e-4, IC0_DROPTOL = 1e-4;  // Precond_ic0 defaults (hip/Precond/precon_ic0.h:14-15)
static void ensure_ic0_maps(Handle &h)
{
    if (h.tpos.n == (size_t)std::max<long>(h.nnz, 1)) return;
    const int n = h.n;
    const int *rp = h.hrp.data(), *ci = h.hci.data();
    std::vector<int> t(std::max<long>(h.nnz, 1), -1);
    for (int r = 0; r < n; r++)
        for (int k = rp[r]; k < rp[r + 1]; k++) {
            const int c = ci[k];
            const int *b = ci + rp[c], *e = ci + rp[c + 1];
            const int *f = std::lower_bound(b, e, r);
            if (f != e && *f == r) t[k] = (int)(f - ci);
            else throw Status(XS_ERR_UNSUPPORTED);  // U is L's transpose: the pattern must be symmetric
        }
    h.tpos.alloc(t.size());
    h.tpos.upload(t.data(), t.size(), h.s);
    h.ic0_tnorm.alloc(n);
}

// IC(0) of A's lower part into h.luv (A's pattern; see k_ic0_rows)
static void factor_ic0(Handle &h)
{
    analyse_pattern(h);
    ensure_ic0_maps(h);
    const int n = h.n;
    h.luv.alloc(std::max<long>(h.nnz, 1));
    XS_CUDA(cudaMemcpyAsync(h.luv.p, h.A.v.p, sizeof(double) * h.nnz, cudaMemcpyDeviceToDevice, h.s));
    k_ic0_tnorm<<<geom().sms * 4, 256, 0, h.s>>>(n, h.A.rp.p, h.A.v.p, IC0_DROPTOL, h.ic0_tnorm.p);
    h.ilu_epoch++;
    if (h.ilu_epoch > 1000000000) {
        XS_CUDA(cudaMemsetAsync(h.flags.p, 0, sizeof(int) * n, h.s));
        h.ilu_epoch = 1;
    }
    const int gl = std::min((n + 127) / 128, geom().sms);
    k_ic0_rows<<<gl, 128, 0, h.s>>>(n, h.A.rp.p, h.A.ci.p, h.uptr.p, h.M.L.level_perm(), h.ic0_tnorm.p, IC0_SMALLNUM,
                                    IC0_DROPTOL, h.luv.p, h.flags.p, h.ilu_epoch, h.err.p, h.fticket.p, 512);
    check_launch();
    int e = 0;
    XS_CUDA(cudaMemcpyAsync(&e, h.err.p, sizeof(int), cudaMemcpyDeviceToHost, h.s));
    XS_CUDA(cudaStreamSynchronize(h.s));
    if (e) throw Status(dev_err_to_status(e));
}

// exact ILU(0) (kind 0) or ParILU (kind 1) into h.luv (A's pattern)
static void factor_ilu(Handle &h, int kind, int sweeps)
{
    analyse_pattern(h);
    const int n = h.n;
    h.luv.alloc(std::max<long>(h.nnz, 1));
    XS_CUDA(cudaMemcpyAsync(h.luv.p, h.A.v.p, sizeof(double) * h.nnz, cudaMemcpyDeviceToDevice, h.s));
    if (kind == 0) {
        h.ilu_epoch++;
        if (h.ilu_epoch > 1000000000) {
            XS_CUDA(cudaMemsetAsync(h.flags.p, 0, sizeof(int) * n, h.s));
            h.ilu_epoch = 1;
        }
        // persistent CTAs per SM: lane-group kernel 4 for groups of <= 8 lanes
        // (128^3 7-point refactorisation 6.9 ms; 7.8 at 8, 7-49 at 16) and 8
        // for wider groups (96^3 27-point 8.7 ms; 10.5 at 4, 13 at 16); the
        // thread-per-row kernel 1 (12 ms at 128^3; 21-45 ms with a CTA per
        // 128 rows)
        static const int ilu_bps_env = [] {
            const char *e = getenv("XS_ILU_BLOCKS_PER_SM");
            return e ? std::max(1, atoi(e)) : 0;
        }();
        static const int ilu_backoff = [] {
            const char *e = getenv("XS_ILU_BACKOFF_NS");
            // longest back-off of a dependency wait: 512 ns measured steadiest
            // (128^3 7-point 6.0 ms, 96^3 27-point 7.3 ms; 64-256 ns gave
            // 6-14 ms with more polling traffic)
            return e ? std::max(32, atoi(e)) : 512;
        }();
        static const int ilu_group = [] {
            const char *e = getenv("XS_ILU_GROUP");
            return e ? atoi(e) : 1;
        }();
        // lanes per row: the longest row rounded up to a power of two (<= 32)
        if (h.max_row_len < 0) {
            int wmax = 0;
            for (int i = 0; i < n; i++) wmax = std::max(wmax, h.hrp[i + 1] - h.hrp[i]);
            h.max_row_len = wmax;
        }
        const int wmax = h.max_row_len;
        int G = 4;
        while (G < wmax && G < 64) G <<= 1;
        if (ilu_tiles_flag() && !h.ilu_tiles_built) {
            build_ilu_tiles(h);
            h.ilu_tiles_built = true;
        }
        if (h.ilu_tiles && ilu_tiles_flag()) {
            // box schedule: CTAs per SM as the staged box area allows
            const TriDev &L = h.M.L;
            const size_t sm = std::max<size_t>(h.ilu_tiles_smem, 16);
            static size_t attr = 0;
            if (sm > attr) {
                XS_CUDA(cudaFuncSetAttribute(k_ilu0_tiles, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
                attr = sm;
            }
            const int per_sm = std::max(1, std::min(4, (int)((size_t)(220 * 1024) / (sm + 1024))));
            const int gl = std::min(L.ntiles, geom().sms * per_sm);
            const IluTileArgs args{L.ntiles, h.A.rp.p, h.A.ci.p, h.uptr.p, h.luv.p, L.t_pos.p, L.t_lvl.p, L.t_lptr.p,
                                   L.perm.p, L.t_hptr.p, L.t_hrow.p, h.ilu_ebase.p, h.ilu_ent.p, h.ilu_roff.p,
                                   h.ilu_rdiag.p, h.ilu_lbase.p, h.ilu_loff.p, h.ilu_dep.p, h.flags.p,
                                   h.ilu_epoch, h.err.p, h.fticket.p};
            k_ilu0_tiles<<<gl, ILU_TILE_THREADS, sm, h.s>>>(args, h.ilu_max_entries, h.ilu_max_lower,
                                                            h.ilu_max_rows);
        } else if (ilu_group && G <= 32) {
            const int rpb = 128 / G;
            const int bps = ilu_bps_env ? ilu_bps_env : (G <= 8 ? 4 : 8);
            const int gl = std::min((n + rpb - 1) / rpb, geom().sms * bps);
            auto go = [&](auto kern) {
                kern<<<gl, 128, 0, h.s>>>(n, h.A.rp.p, h.A.ci.p, h.uptr.p, h.M.L.level_perm(), h.luv.p, h.flags.p,
                                          h.ilu_epoch, h.err.p, h.fticket.p, ilu_backoff);
            };
            if (G == 4) go(k_ilu0_groups<4>);
            else if (G == 8) go(k_ilu0_groups<8>);
            else if (G == 16) go(k_ilu0_groups<16>);
            else go(k_ilu0_groups<32>);
        } else {
            const int gl = std::min((n + 127) / 128, geom().sms * (ilu_bps_env ? ilu_bps_env : 1));
            k_ilu0_rows<<<gl, 128, 0, h.s>>>(n, h.A.rp.p, h.A.ci.p, h.uptr.p, h.M.L.level_perm(), h.luv.p, h.flags.p,
                                             h.ilu_epoch, h.err.p, h.fticket.p, ilu_backoff);
        }
        check_launch();
    } else {
        ensure_entry_maps(h, true);
        h.tmpv.alloc(std::max<long>(h.nnz, 1));
        const int g = geom().sms * 8;
        double *cur = h.luv.p, *nxt = h.tmpv.p;
        for (int sw = 0; sw < sweeps; sw++) {
            k_parilu_sweep<<<g, 256, 0, h.s>>>(h.nnz, h.A.rp.p, h.A.ci.p, h.rowof.p, h.uptr.p, h.ucp.p, h.ucpos.p,
                                               h.A.v.p, cur, nxt);
            std::swap(cur, nxt);
        }
        check_launch();
        if (cur != h.luv.p)
            XS_CUDA(cudaMemcpyAsync(h.luv.p, cur, sizeof(double) * h.nnz, cudaMemcpyDeviceToDevice, h.s));
    }
    int e = read_dev_err(h);
    if (e) throw Status(dev_err_to_status(e));
}

// host-computed factors (L strict, dinv, U' strict) into the device layout
// the threshold factorizations share
static void upload_host_factors(cudaStream_t s, int n, HostTriFactors &F, ParilutResult &R)
{
    R = ParilutResult();
    R.n = n;
    R.nnzL = (long)F.lci.size();
    R.nnzU = (long)F.uci.size();
    R.lrp.alloc(n + 1); R.lrp.upload(F.lrp.data(), n + 1, s);
    R.urp.alloc(n + 1); R.urp.upload(F.urp.data(), n + 1, s);
    R.lci.alloc(std::max<long>(R.nnzL, 1)); R.lv.alloc(std::max<long>(R.nnzL, 1));
    R.uci.alloc(std::max<long>(R.nnzU, 1)); R.uv.alloc(std::max<long>(R.nnzU, 1));
    if (R.nnzL) { R.lci.upload(F.lci.data(), R.nnzL, s); R.lv.upload(F.lv.data(), R.nnzL, s); }
    if (R.nnzU) { R.uci.upload(F.uci.data(), R.nnzU, s); R.uv.upload(F.uv.data(), R.nnzU, s); }
    R.dinv.alloc(std::max(n, 1));
    if (n) R.dinv.upload(F.dinv.data(), n, s);
    std::vector<long> ident(n);
    std::iota(ident.begin(), ident.end(), 0L);
    R.diag_ident.alloc(std::max(n, 1));
    if (n) R.diag_ident.upload(ident.data(), n, s);
    XS_CUDA(cudaStreamSynchronize(s));  // the host arrays are released by the caller
    R.hlrp.assign(F.lrp.begin(), F.lrp.end()); R.hlci.assign(F.lci.begin(), F.lci.end());
    R.hurp.assign(F.urp.begin(), F.urp.end()); R.huci.assign(F.uci.begin(), F.uci.end());
}

// factors out to caller arrays (any of them may be NULL)
static void copy_host_factors(int n, const HostTriFactors &F, int *nnzL, int *nnzU, int *lrp, int *lci, double *lv,
                              double *dinv, int *urp, int *uci, double *uv)
{
    const size_t nl = F.lci.size(), nu = F.uci.size();
    if (nnzL) *nnzL = (int)nl;
    if (nnzU) *nnzU = (int)nu;
    if (lrp) std::memcpy(lrp, F.lrp.data(), sizeof(int) * (n + 1));
    if (urp) std::memcpy(urp, F.urp.data(), sizeof(int) * (n + 1));
    if (lci && nl) std::memcpy(lci, F.lci.data(), sizeof(int) * nl);
    if (lv && nl) std::memcpy(lv, F.lv.data(), sizeof(double) * nl);
    if (uci && nu) std::memcpy(uci, F.uci.data(), sizeof(int) * nu);
    if (uv && nu) std::memcpy(uv, F.uv.data(), sizeof(double) * nu);
    if (dinv && n) std::memcpy(dinv, F.dinv.data(), sizeof(double) * n);
}

static void build_precond(Handle &h)
{
    if (h.pc_ready) return;
    if (!h.have_matrix) throw Status(XS_ERR_ORDER);
    cudaEvent_t e0, e1;
    XS_CUDA(cudaEventCreate(&e0));
    XS_CUDA(cudaEventCreate(&e1));
    XS_CUDA(cudaEventRecord(e0, h.s));
    const int n = h.n;
    PrecondDev &M = h.M;
    M.n = n;
    M.err = h.err.p;
    M.factor_prec = h.factor_prec;
    M.trsv_mode = h.trsv_mode;
    const bool need32 = h.inner32 != 0;
    int type = h.pc_req < 0 ? PC_NONE : h.pc_req;
    M.type = type;
    if (type == PC_JACOBI) {
        analyse_pattern(h);
        M.jdiag64.alloc(n);
        k_jacobi_init<double><<<geom().sms * 4, 256, 0, h.s>>>(n, h.uptr.p, h.A.v.p, M.jdiag64.p);
        M.jdiag32.alloc(n);
        k_jacobi_init<float><<<geom().sms * 4, 256, 0, h.s>>>(n, h.uptr.p, h.A.v.p, M.jdiag32.p);
        check_launch();
    } else if (type == PC_ILU0 || type == PC_PARILU || type == PC_IC0) {
        Trace tr("setup ilu (total)", h.s);
        {
            Trace t1("  analyse_pattern", h.s);
            analyse_pattern(h);
        }
        Trace t2("  numeric factor + loads", h.s);
        if (h.fv.n != (size_t)std::max<long>(h.nnz, 1)) h.fv.alloc(std::max<long>(h.nnz, 1));
        if (type == PC_IC0) {
            factor_ic0(h);
            ensure_entry_maps(h, false);
            k_ic0_split<<<geom().sms * 4, 256, 0, h.s>>>(h.nnz, h.rowof.p, h.A.ci.p, h.uptr.p, h.tpos.p, h.luv.p,
                                                         h.fv.p);
        } else {
            factor_ilu(h, type == PC_ILU0 ? 0 : 1, h.parilu_sweeps);
            k_split_lu<<<geom().sms * 4, 256, 0, h.s>>>(n, h.A.rp.p, h.A.ci.p, h.uptr.p, h.luv.p, h.fv.p);
        }
        check_launch();
        const FactorCopies fc = factor_copies(h, need32);
        load_tri_values(h, M.L, h.fv.p, fc);
        load_tri_values(h, M.U, h.fv.p, fc);
        if (fc.ell) {
            load_tri_ell(M.L, h.fv.p, need32, h.s, fc.red);
            load_tri_ell(M.U, h.fv.p, need32, h.s, fc.red);
        } else {
            for (TriDev *T : {&M.L, &M.U}) { T->ev64.free(); T->ev32.free(); T->evbf.free(); T->evh.free(); }
        }
        load_dinv(h, h.fv.p, h.udiag_src.p, need32);
        M.ensure_buffers64(h.s);
        if (need32) M.ensure_buffers32(h.s);
        if (h.trsv_mode > 0) M.ensure_sweep_buffers(need32);
        M.have_factors = true;
    } else if (pc_own_pattern(type)) {
        Trace tr("setup threshold factor (total)", h.s);
        if (type == PC_PARILUT) {
            parilut_build(h.s, h.err.p, n, h.A, h.parilut_fill, h.parilut_sweeps, h.parilut_droptol, h.ilut);
        } else {
            // sequential row chains: factored by the host, applied on the device
            HostTriFactors F;
            const double *hv = host_vals(h);
            if (type == PC_ILUP) {
                host_ilut(n, h.hrp.data(), h.hci.data(), hv, h.ilup_fill, h.ilup_tol, F);
            } else if (host_ict(n, h.hrp.data(), h.hci.data(), hv, h.ict_fill, h.ict_tol, F) >= 0) {
                throw Status(XS_ERR_NO_DIAG);
            }
            upload_host_factors(h.s, n, F, h.ilut);
        }
        // factors in the seqilu0 layout on their own pattern
        ilut_to_tri(h.s, n, h.ilut, M.L, M.U, need32);
        {
            Trace tr_trim("  scratch pool trim", h.s);
            pool_trim(h.s);
        }
        M.ensure_buffers64(h.s);
        if (need32) M.ensure_buffers32(h.s);
        if (h.trsv_mode > 0) M.ensure_sweep_buffers(need32);
        M.have_factors = true;
    }
    XS_CUDA(cudaEventRecord(e1, h.s));
    XS_CUDA(cudaEventSynchronize(e1));
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    h.setup_ms = ms;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    int e = read_dev_err(h);
    if (e) throw Status(dev_err_to_status(e));
    h.pc_ready = true;
}

// ---------------------------------------------------------------- solves
static void prepare_state(Handle &h, int maxiter, double tol, double abstol, bool rel_hist)
{
    h.W.ensure(64, maxiter);
    KState &s = *h.W.h_st;
    std::memset(&s, 0, sizeof(KState));
    s.tol = tol;
    s.abstol = abstol;
    s.maxiter = maxiter;
    s.hist = h.W.hist.p;
    s.hist_rel = rel_hist ? h.W.hist_rel.p : nullptr;
    XS_CUDA(cudaMemcpyAsync(h.W.st.p, &s, sizeof(KState), cudaMemcpyHostToDevice, h.s));
}

// run a method on device vectors (b, x) of type VT with the given operator
// and preconditioner
template <typename VT>
static void run_method_on(RunSet<VT> &R, Operator &A, PrecondDev &M, Workspace &W, cudaStream_t s, int n, int quirk,
                          int method, const VT *b, VT *x, int restart, long long *launches = nullptr)
{
    SolveCtx c{s, &A, &M, &W, n, 8, quirk, launches};
    if (n < 200000) c.chunk = 16;
    switch (method) {
    case KSP_CGM: R.pcg.run(c, b, x); break;
    case KSP_CG_LEFT: R.cgl.run(c, b, x); break;
    case KSP_ICG: R.icg.run(c, b, x); break;
    case KSP_ICGM: R.icgm.run(c, b, x); break;
    case KSP_IBICGSTAB: R.ibicg.run(c, b, x); break;
    case KSP_BICGSTAB: R.bicg.run(c, b, x); break;
    case KSP_GMRES_LEFT:
    case KSP_GMRES_RIGHT: R.gmres.run(c, b, x, restart, method == KSP_GMRES_RIGHT); break;
    case KSP_GCR_LEFT:
    case KSP_IGCR_LEFT:
    case KSP_GCR_RIGHT:
        R.gcr.run(c, b, x, restart, method == KSP_GCR_LEFT ? 0 : (method == KSP_IGCR_LEFT ? 1 : 2));
        break;
    default: throw Status(XS_ERR_ORDER);
    }
}

template <typename VT>
static void run_method(Handle &h, int method, const VT *b, VT *x, int restart)
{
    if constexpr (std::is_same<VT, double>::value)
        run_method_on<double>(h.r64, h.A, h.M, h.W, h.s, h.n, h.quirk, method, b, x, restart, &h.launches);
    else
        run_method_on<float>(h.r32, h.A, h.M, h.W, h.s, h.n, h.quirk, method, b, x, restart, &h.launches);
}

static int effective_restart(const Handle &h)
{
    int restart = h.restart > 0 ? h.restart : std::min(h.maxiter, 64);
    return std::max(restart, 1);
}

__global__ void k_d2f(int n, const double *__restrict__ a, float *__restrict__ b, const double *scale_inv)
{
    const double s = scale_inv ? *scale_inv : 1.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) b[i] = (float)(a[i] * s);
}
// x += d * scale (FP64 update of the refinement)
__global__ void k_refine_update(int n, double *__restrict__ x, const float *__restrict__ d, const double *scale)
{
    const double s = scale ? *scale : 1.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) x[i] = x[i] + (double)d[i] * s;
}
template <typename VT>
struct EpiOuterResid {
    static constexpr int K = 1;
    OuterState *os;
    const VT *b;
    __device__ bool active() const { return true; }
    __device__ VT out(int r, double ax) const { return (VT)((double)b[r] - ax); }
    __device__ void acc(int, double y, double (&a)[1]) const { a[0] += y * y; }
    __device__ void finalize(const double *t) const
    {
        const double r = sqrt(t[0]);
        os->rnorm = r;
        os->scale = r;
        os->scale_inv = r > 0 ? 1.0 / r : 0.0;
    }
};

// safety factor of the adaptive inner tolerance of the refinement
constexpr double INNER_SAFETY = 0.25;

// Solve with device vectors b (rhs) and x (x0 in, solution out), FP64.
// Writes the conventions requested by the caller into usediter/resvec.
static void solve_device(Handle &h, const double *d_b, double *d_x)
{
    Trace tr("solve_device", h.s);
    if (!h.have_matrix) throw Status(XS_ERR_ORDER);
    if (h.method == 0) throw Status(XS_ERR_ORDER);
    build_precond(h);
    clear_dev_err(h);
    const int n = h.n;
    double *b = h.vpool64.get(0, n), *x = h.vpool64.get(1, n);
    XS_CUDA(cudaMemcpyAsync(b, d_b, sizeof(double) * n, cudaMemcpyDeviceToDevice, h.s));
    XS_CUDA(cudaMemcpyAsync(x, d_x, sizeof(double) * n, cudaMemcpyDeviceToDevice, h.s));
    const int restart = effective_restart(h);
    cudaEvent_t e0, e1;
    XS_CUDA(cudaEventCreate(&e0));
    XS_CUDA(cudaEventCreate(&e1));
    XS_CUDA(cudaEventRecord(e0, h.s));
    int iters = 0;
    std::vector<double> hist;
    int done = 0, devflags = 0;
    h.launches = 4;  // residual SpMV, preconditioner (<= 2 kernels), init reduction
    if (!h.inner32) {
        prepare_state(h, h.maxiter, h.tol, h.abstol, true);
        run_method<double>(h, h.method, b, x, restart);
        XS_CUDA(cudaMemcpyAsync(h.W.h_st, h.W.st.p, sizeof(KState), cudaMemcpyDeviceToHost, h.s));
        XS_CUDA(cudaStreamSynchronize(h.s));
        KState &st = *h.W.h_st;
        iters = st.iter;
        done = st.done;
        devflags = st.err;
        hist.resize(iters + 1);
        XS_CUDA(cudaMemcpyAsync(hist.data(), h.W.hist.p, sizeof(double) * (iters + 1), cudaMemcpyDeviceToHost, h.s));
        std::vector<double> rel(iters);
        if (iters) XS_CUDA(cudaMemcpyAsync(rel.data(), h.W.hist_rel.p, sizeof(double) * iters, cudaMemcpyDeviceToHost, h.s));
        XS_CUDA(cudaStreamSynchronize(h.s));
        h.final_relres = iters ? rel[iters - 1] : (st.res0 > 0 ? 1.0 : 0.0);
        if (h.resvec) {
            if (h.intel_conv) {
                for (int k = 0; k < iters; k++) h.resvec[k] = rel[k];
            } else {
                for (int k = 0; k <= iters; k++) h.resvec[k] = hist[k];
            }
        }
        h.last_outer = 0;
    } else if (h.method == KSP_BICGSTAB && h.carry_krylov) {
        // ---- mixed precision refinement carrying the Krylov iteration
        // One FP32 BiCGSTAB runs across all refinement steps.  A step ends
        // when its recurrence residual has dropped by the inner tolerance;
        // then x += d (FP64), r = b - A x (FP64), the inner residual is
        // replaced by float(r) and beta = (rhat, r) recomputed, and the same
        // iteration continues (p, u, rhat and the scalars are kept) — a
        // restart would throw away the search space it has built.  Vectors
        // stay unscaled (FP32 range covers the 1e10 reduction).
        DBuf<OuterState> &os_buf = h.outer_st;
        if (!os_buf.p) os_buf.alloc(1);
        OuterState *os = os_buf.p;
        double *r = h.vpool64.get(2, n);
        float *r32 = h.vpool32.get(0, n), *d32 = h.vpool32.get(1, n);
        operator_ensure32(h.A, h.hrp.data(), h.s);
        h.W.ensure(64, std::max(h.maxiter, 1) + 8);  // history capacity for the whole solve
        prepare_state(h, std::max(h.inner_maxiter, 1), h.inner_rtol, 0.0, true);
        const RedSlot sl = h.W.slot();
        spmv<double, double>(h.A, x, r, EpiOuterResid<double>{os, b}, sl, h.s);
        OuterState hos;
        XS_CUDA(cudaMemcpyAsync(&hos, os, sizeof(OuterState), cudaMemcpyDeviceToHost, h.s));
        XS_CUDA(cudaStreamSynchronize(h.s));
        const double r0 = hos.rnorm;
        hist.push_back(r0);
        double rn = r0;
        int outer = 0, it_prev = 0;
        const int max_outer = 100;
        done = 0;
        SolveCtx c{h.s, &h.A, &h.M, &h.W, n, 8, h.quirk, &h.launches};
        if (n < 200000) c.chunk = 16;
        BicgRun<float, float> &bi = h.r32.bicg;
        while (true) {
            if (!(rn == rn)) { devflags |= DEV_NAN; done = 3; break; }
            if (rn == 0.0 || rn / (r0 + KSMALL) < h.tol || rn <= h.abstol) { done = 1; break; }
            if (iters >= h.maxiter || outer >= max_outer) { done = 2; break; }
            const double target = std::max(h.tol * (r0 + KSMALL), h.abstol);
            const double irtol = std::min(std::max(h.inner_rtol, INNER_SAFETY * target / rn), 0.5);
            const int more = std::max(1, std::min(h.inner_maxiter, h.maxiter - iters));
            XS_CUDA(cudaMemsetAsync(d32, 0, sizeof(float) * n, h.s));
            if (outer == 0) {
                k_d2f<<<geom().sms * 4, 256, 0, h.s>>>(n, r, r32, nullptr);
                check_launch();
                prepare_state(h, more, irtol, 0.0, true);
                bi.run(c, r32, d32, false);
            } else {
                float *ri = bi.residual(n);
                k_d2f<<<geom().sms * 4, 256, 0, h.s>>>(n, r, ri, nullptr);
                // clear done first: vector ops skip their work while it is set
                k_resume_state<<<1, 1, 0, h.s>>>(h.W.st.p, rn, irtol, more);
                check_launch();
                vecop(OpBicgRho<float>{n, h.W.st.p, bi.shadow(n), ri}, sl, h.s);
                h.W.h_st->maxiter = more;  // iterations this step may add (caps the graph replays)
                bi.run(c, r32, d32, true);
            }
            XS_CUDA(cudaMemcpyAsync(h.W.h_st, h.W.st.p, sizeof(KState), cudaMemcpyDeviceToHost, h.s));
            XS_CUDA(cudaStreamSynchronize(h.s));
            const int it_in = h.W.h_st->iter - it_prev;
            it_prev = h.W.h_st->iter;
            devflags |= h.W.h_st->err;
            if (devflags & (DEV_TRSV_TIMEOUT | DEV_TMA_TIMEOUT)) { done = 3; break; }
            k_refine_update<<<geom().sms * 4, 256, 0, h.s>>>(n, x, d32, nullptr);
            check_launch();
            spmv<double, double>(h.A, x, r, EpiOuterResid<double>{os, b}, sl, h.s);
            XS_CUDA(cudaMemcpyAsync(&hos, os, sizeof(OuterState), cudaMemcpyDeviceToHost, h.s));
            XS_CUDA(cudaStreamSynchronize(h.s));
            iters += std::max(it_in, 1);
            h.launches += 8;  // replacement, rho, resume, refinement update, outer residual
            rn = hos.rnorm;
            hist.push_back(rn);
            outer++;
            if (h.W.h_st->done == 3 && (devflags & (DEV_BREAKDOWN | DEV_NAN))) { done = 3; break; }
        }
        h.last_outer = outer;
        h.final_relres = rn / (r0 + KSMALL);
        if (h.resvec) {
            for (size_t k = 0; k < hist.size(); k++) h.resvec[k] = h.intel_conv ? hist[k] / (r0 + KSMALL) : hist[k];
        }
    } else {
        // ---- mixed precision iterative refinement
        // outer: r = b - A x (FP64), x += d (FP64); inner: FP32 solve of
        // A d = r/||r|| to inner_rtol with FP32 SpMV and BF16/FP16/FP32 factors
        DBuf<OuterState> &os_buf = h.outer_st;
        if (!os_buf.p) os_buf.alloc(1);
        OuterState *os = os_buf.p;
        double *r = h.vpool64.get(2, n);
        float *r32 = h.vpool32.get(0, n), *d32 = h.vpool32.get(1, n);
        operator_ensure32(h.A, h.hrp.data(), h.s);
        prepare_state(h, std::max(h.inner_maxiter, 1), h.inner_rtol, 0.0, true);
        const RedSlot sl = h.W.slot();  // after prepare_state: the workspace exists now
        spmv<double, double>(h.A, x, r, EpiOuterResid<double>{os, b}, sl, h.s);
        OuterState hos;
        XS_CUDA(cudaMemcpyAsync(&hos, os, sizeof(OuterState), cudaMemcpyDeviceToHost, h.s));
        XS_CUDA(cudaStreamSynchronize(h.s));
        const double r0 = hos.rnorm;
        hist.push_back(r0);
        double rn = r0;
        int outer = 0;
        const int max_outer = 100;
        done = 0;
        while (true) {
            if (!(rn == rn)) { devflags |= DEV_NAN; done = 3; break; }
            if (rn == 0.0 || rn / (r0 + KSMALL) < h.tol || rn <= h.abstol) { done = 1; break; }
            if (iters >= h.maxiter || outer >= max_outer) { done = 2; break; }
            // inner rhs r/||r|| in FP32, x0 = 0
            k_d2f<<<geom().sms * 4, 256, 0, h.s>>>(n, r, r32, &os->scale_inv);
            XS_CUDA(cudaMemsetAsync(d32, 0, sizeof(float) * n, h.s));
            check_launch();
            int inner_max = std::min(h.inner_maxiter, h.maxiter - iters);
            // the inner tolerance is loosened (never tightened) to what the
            // outer target still needs, with a safety factor: the last step
            // does not overshoot the target by orders of magnitude
            const double target = std::max(h.tol * (r0 + KSMALL), h.abstol);
            const double need = INNER_SAFETY * target / rn;
            const double irtol = std::min(std::max(h.inner_rtol, need), 0.5);
            prepare_state(h, inner_max, irtol, 0.0, true);
            run_method<float>(h, h.method, r32, d32, restart);
            XS_CUDA(cudaMemcpyAsync(h.W.h_st, h.W.st.p, sizeof(KState), cudaMemcpyDeviceToHost, h.s));
            XS_CUDA(cudaStreamSynchronize(h.s));
            int it_in = h.W.h_st->iter;
            devflags |= h.W.h_st->err;
            if (devflags & (DEV_TRSV_TIMEOUT | DEV_TMA_TIMEOUT)) { done = 3; break; }
            // x += d*||r|| ; r = b - A x
            k_refine_update<<<geom().sms * 4, 256, 0, h.s>>>(n, x, d32, &os->scale);
            check_launch();
            spmv<double, double>(h.A, x, r, EpiOuterResid<double>{os, b}, sl, h.s);
            XS_CUDA(cudaMemcpyAsync(&hos, os, sizeof(OuterState), cudaMemcpyDeviceToHost, h.s));
            XS_CUDA(cudaStreamSynchronize(h.s));
            iters += std::max(it_in, 1);
            h.launches += 7;  // convert, refinement update, outer residual SpMV, inner init
            rn = hos.rnorm;
            hist.push_back(rn);
            outer++;
        }
        h.last_outer = outer;
        h.final_relres = rn / (r0 + KSMALL);
        if (h.resvec) {
            // one entry per outer step: resvec[0] = ||r0||, resvec[k] = ||r|| after step k
            for (size_t k = 0; k < hist.size(); k++) h.resvec[k] = h.intel_conv ? hist[k] / (r0 + KSMALL) : hist[k];
        }
    }
    XS_CUDA(cudaEventRecord(e1, h.s));
    XS_CUDA(cudaEventSynchronize(e1));
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    h.solve_ms = ms;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    h.last_iters = iters;
    if (h.usediter) {
        if (h.intel_conv) {
            bool restarted = (h.method == KSP_GCR_LEFT || h.method == KSP_IGCR_LEFT || h.method == KSP_GMRES_LEFT ||
                              h.method == KSP_GMRES_RIGHT);
            if (done == 1) *h.usediter = std::max(iters - 1, 0);
            else *h.usediter = restarted ? iters : std::max(iters - 1, 0);
        } else {
            *h.usediter = iters;
        }
    }
    XS_CUDA(cudaMemcpyAsync(d_x, x, sizeof(double) * n, cudaMemcpyDeviceToDevice, h.s));
    XS_CUDA(cudaStreamSynchronize(h.s));
    int e = read_dev_err(h) | devflags;
    if (e & (DEV_TRSV_TIMEOUT | DEV_TMA_TIMEOUT | DEV_FACTOR_TIMEOUT)) {
        // an aborted kernel may leave solve buffers and reduction tickets
        // mid-way: re-arm them so the handle stays usable
        h.M.rearm(h.s);
        XS_CUDA(cudaMemsetAsync(h.W.ticket.p, 0, sizeof(unsigned), h.s));
        XS_CUDA(cudaStreamSynchronize(h.s));
    }
    // only a solve that ended without an error is one the adjoint may
    // differentiate through
    if (e) {
        h.have_solution = false;
        throw Status(dev_err_to_status(e));
    }
    h.have_solution = true;
    adjoint_record_solution(h.adj, h.s, n, x);
}

static void solve_host(Handle &h, const double *rhs, double *sol)
{
    if (!rhs || !sol) throw Status(XS_ERR_INVALID);
    const int n = h.n;
    double *b = h.vpool64.get(3, n), *x = h.vpool64.get(4, n);
    XS_CUDA(cudaMemcpyAsync(b, rhs, sizeof(double) * n, cudaMemcpyHostToDevice, h.s));
    XS_CUDA(cudaMemcpyAsync(x, sol, sizeof(double) * n, cudaMemcpyHostToDevice, h.s));
    int status = XS_OK;
    try {
        solve_device(h, b, x);
    } catch (Status &st) {
        status = st.code;
    }
    XS_CUDA(cudaMemcpyAsync(sol, x, sizeof(double) * n, cudaMemcpyDeviceToHost, h.s));
    XS_CUDA(cudaStreamSynchronize(h.s));
    if (status) throw Status(status);
}

// ---------------------------------------------------------------- adjoint
// transposed operator and preconditioner, built on first use
static void adjoint_prepare(Handle &h)
{
    AdjointState &a = h.adj;
    const int n = h.n;
    if (!a.have_At) {
        std::vector<int> trp, tci;
        std::vector<double> tv;
        host_transpose(n, h.hrp.data(), h.hci.data(), host_vals(h), trp, tci, &tv, nullptr);
        a.At = Operator();
        operator_setup(a.At, n, trp.data(), tci.data(), tv.data(), 0, false, h.s, h.err.p);
        if (h.A.format == 1) operator_build_ell(a.At, trp.data(), tci.data(), tv.data(), 0, false, h.s);
        a.At.format = h.A.format;
        a.have_At = true;
    }
    PrecondDev &M = h.M;
    if (a.have_Mt && a.Mt_type == M.type) return;
    PrecondDev &T = a.Mt;
    T = PrecondDev();
    T.n = n;
    T.err = h.err.p;
    T.type = M.type;
    T.trsv_mode = M.trsv_mode;
    T.factor_prec = FP_F64;
    if (M.type == PC_JACOBI) {
        T.jdiag64.alloc(n);
        XS_CUDA(cudaMemcpyAsync(T.jdiag64.p, M.jdiag64.p, sizeof(double) * n, cudaMemcpyDeviceToDevice, h.s));
    } else if (pc_triangular(M.type)) {
        // host patterns of L (strict lower) and U' (strict upper) with their
        // value sources, then the transposed triangles
        std::vector<int> lrp, lci, urp, uci;
        std::vector<long> lsrc, usrc;
        const double *vals;
        const long *diagsrc;
        DBuf<long> ident_diag;
        if (pc_own_pattern(M.type)) {
            ParilutResult &R = h.ilut;
            lrp.assign(R.hlrp.begin(), R.hlrp.end()); lci.assign(R.hlci.begin(), R.hlci.end());
            urp.assign(R.hurp.begin(), R.hurp.end()); uci.assign(R.huci.begin(), R.huci.end());
            lsrc.resize(lci.size()); usrc.resize(uci.size());
            for (size_t k = 0; k < lsrc.size(); k++) lsrc[k] = (long)k;
            for (size_t k = 0; k < usrc.size(); k++) usrc[k] = (long)(lci.size() + k);
            // combined value array: [L values | U' values | dinv]
            h.tmpv.alloc(std::max<size_t>(lci.size() + uci.size() + n, 1));
            if (!lci.empty()) XS_CUDA(cudaMemcpyAsync(h.tmpv.p, R.lv.p, sizeof(double) * lci.size(), cudaMemcpyDeviceToDevice, h.s));
            if (!uci.empty()) XS_CUDA(cudaMemcpyAsync(h.tmpv.p + lci.size(), R.uv.p, sizeof(double) * uci.size(), cudaMemcpyDeviceToDevice, h.s));
            XS_CUDA(cudaMemcpyAsync(h.tmpv.p + lci.size() + uci.size(), R.dinv.p, sizeof(double) * n, cudaMemcpyDeviceToDevice, h.s));
            vals = h.tmpv.p;
            std::vector<long> ds(n);
            for (int i = 0; i < n; i++) ds[i] = (long)(lci.size() + uci.size() + i);
            ident_diag.alloc(n);
            ident_diag.upload(ds.data(), n, h.s);
            diagsrc = ident_diag.p;
        } else {
            lrp.assign(n + 1, 0); urp.assign(n + 1, 0);
            for (int i = 0; i < n; i++) {
                for (int k = h.hrp[i]; k < h.hrp[i + 1]; k++) {
                    if (h.hci[k] < i) { lci.push_back(h.hci[k]); lsrc.push_back(k); }
                    else if (h.hci[k] > i) { uci.push_back(h.hci[k]); usrc.push_back(k); }
                }
                lrp[i + 1] = (int)lci.size();
                urp[i + 1] = (int)uci.size();
            }
            vals = h.fv.p;
            diagsrc = h.udiag_src.p;
        }
        // U'^T: lower triangle; L^T: upper triangle
        std::vector<int> utrp, utci, ltrp, ltci;
        std::vector<long> utsrc_k, ltsrc_k;
        std::vector<double> dummy;
        host_transpose(n, urp.data(), uci.data(), nullptr, utrp, utci, nullptr, &utsrc_k);
        host_transpose(n, lrp.data(), lci.data(), nullptr, ltrp, ltci, nullptr, &ltsrc_k);
        build_tri_dev(T.L, n, utrp, utci, false, [&](int k) { return usrc[utsrc_k[k]]; }, h.s);
        build_tri_dev(T.U, n, ltrp, ltci, true, [&](int k) { return lsrc[ltsrc_k[k]]; }, h.s);
        const int g = geom().sms * 4;
        for (TriDev *D : {&T.L, &T.U}) {
            long m = std::max<long>(D->nnz, 1);
            D->pv64.alloc(m, 8);
            D->nv64.alloc(m);
            if (D->nnz) {
                k_gather_convert<double><<<g, 256, 0, h.s>>>(D->nnz, D->src.p, vals, D->pv64.p);
                k_gather_convert<double><<<g, 256, 0, h.s>>>(D->nnz, D->src_nat.p, vals, D->nv64.p);
            }
        }
        T.U.dinv64.alloc(n, 4);
        T.U.dinv64_nat.alloc(n);
        k_gather_dinv<double><<<g, 256, 0, h.s>>>(n, T.U.perm.p, diagsrc, vals, T.U.dinv64.p);
        k_gather_dinv<double><<<g, 256, 0, h.s>>>(n, nullptr, diagsrc, vals, T.U.dinv64_nat.p);
        check_launch();
        T.ensure_buffers64(h.s);
        load_tri_ell(T.L, vals, false, h.s);
        load_tri_ell(T.U, vals, false, h.s);
        if (T.trsv_mode > 0) T.ensure_sweep_buffers(false);
        XS_CUDA(cudaStreamSynchronize(h.s));
    }
    a.have_Mt = true;
    a.Mt_type = M.type;
}

static void adjoint_solve(Handle &h, const double *dLdx, double *dLdb, double *dLdA)
{
    adjoint_prepare(h);
    AdjointState &a = h.adj;
    const int n = h.n;
    clear_dev_err(h);
    if (a.lam.n != (size_t)n) { a.lam.alloc(n); a.rhs.alloc(n); }
    a.rhs.upload(dLdx, n, h.s);
    XS_CUDA(cudaMemsetAsync(a.lam.p, 0, sizeof(double) * n, h.s));
    // backward solve with the forward method (FP64), transposed operator/preconditioner
    prepare_state(h, h.maxiter, h.tol, h.abstol, true);
    int method = h.method;
    run_method_on<double>(a.runs, a.At, a.Mt, h.W, h.s, n, 0, method, a.rhs.p, a.lam.p, effective_restart(h));
    // gradients
    double *db = nullptr, *dA = nullptr;
    DBuf<double> &gb = a.gb, &gA = a.gA;
    if (dLdb) {
        if (gb.n != (size_t)n) gb.alloc(n);
        db = gb.p;
    }
    if (dLdA) {
        if (gA.n != (size_t)std::max<long>(h.nnz, 1)) gA.alloc(std::max<long>(h.nnz, 1));
        dA = gA.p;
    }
    k_adjoint_grad<<<geom().sms * 4, 256, 0, h.s>>>(n, h.A.rp.p, h.A.ci.p, a.lam.p, a.x_last.p, db, dA);
    check_launch();
    if (dLdb) gb.download(dLdb, n, h.s);
    if (dLdA) {
        if (h.vperm.empty()) gA.download(dLdA, h.nnz, h.s);
        else {
            std::vector<double> t(h.nnz);
            gA.download(t.data(), h.nnz, h.s);
            XS_CUDA(cudaStreamSynchronize(h.s));
            for (long k = 0; k < h.nnz; k++) dLdA[h.vperm[k]] = t[k];
        }
    }
    XS_CUDA(cudaStreamSynchronize(h.s));
    int e = read_dev_err(h) | h.W.h_st->err;
    XS_CUDA(cudaMemcpyAsync(h.W.h_st, h.W.st.p, sizeof(KState), cudaMemcpyDeviceToHost, h.s));
    XS_CUDA(cudaStreamSynchronize(h.s));
    e |= h.W.h_st->err;
    if (e & (DEV_TRSV_TIMEOUT | DEV_TMA_TIMEOUT)) { a.Mt.rearm(h.s); XS_CUDA(cudaStreamSynchronize(h.s)); }
    if (e) throw Status(dev_err_to_status(e));
}

static void adjoint_host(Handle &h, const double *dLdx, double *dLdb, double *dLdA)
{
    if (!h.have_solution) throw Status(XS_ERR_ORDER);
    build_precond(h);
    adjoint_solve(h, dLdx, dLdb, dLdA);
}

// ---------------------------------------------------------------- several right-hand sides
// PCG with an exact (or no / Jacobi) FP64 preconditioner solves k right-hand
// sides together (xs_batch.cuh); anything else solves them one by one.
static bool batch_ok(Handle &h, const PrecondDev &M, int k)
{
    return k >= 2 && k <= BATCH_MAX && h.method == KSP_CGM && !h.inner32 && batch_precond_ok(M) &&
           batch_tuning().enabled;
}

static int batch_errors(Handle &h, BatchRuntime &R, BatchPrecond &bp)
{
    R.S.fetch(h.s);
    int e = read_dev_err(h);
    for (const KState &st : R.S.h) e |= st.err;
    if (e & (DEV_TRSV_TIMEOUT | DEV_TMA_TIMEOUT)) {
        bp.rearm(h.s);
        XS_CUDA(cudaMemsetAsync(R.S.ticket.p, 0, sizeof(unsigned), h.s));
        if (bp.ticket.p) XS_CUDA(cudaMemsetAsync(bp.ticket.p, 0, sizeof(unsigned), h.s));
        XS_CUDA(cudaStreamSynchronize(h.s));
    }
    return e;
}

static void solve_batch(Handle &h, int k, const double *rhs, double *sol)
{
    build_precond(h);
    if (!batch_ok(h, h.M, k)) {
        for (int c = 0; c < k; c++) solve_host(h, rhs + (size_t)c * h.n, sol + (size_t)c * h.n);
        return;
    }
    clear_dev_err(h);
    const int n = h.n;
    const long m = (long)n * k;
    BatchRuntime &R = h.batch;
    if (R.bB.n != (size_t)m) { R.bB.alloc(m); R.bX.alloc(m); R.tmp.alloc(m); }
    const int g = geom().sms * 4;
    R.tmp.upload(rhs, m, h.s);
    k_interleave<<<g, 256, 0, h.s>>>(n, k, R.tmp.p, R.bB.p);
    R.tmp.upload(sol, m, h.s);  // x0 of every column
    k_interleave<<<g, 256, 0, h.s>>>(n, k, R.tmp.p, R.bX.p);
    check_launch();
    R.S.prepare(k, h.maxiter, h.tol, h.abstol, h.s);
    cudaEvent_t e0, e1;
    XS_CUDA(cudaEventCreate(&e0));
    XS_CUDA(cudaEventCreate(&e1));
    XS_CUDA(cudaEventRecord(e0, h.s));
    h.launches = 2;
    const DevCsr A{n, h.nnz, h.A.rp.p, h.A.ci.p, h.A.v.p, nullptr};
    R.pcg.run(h.s, A, h.M, R.bp, R.S, k, R.bB.p, R.bX.p, &h.launches);
    XS_CUDA(cudaEventRecord(e1, h.s));
    k_deinterleave<<<g, 256, 0, h.s>>>(n, k, R.bX.p, R.tmp.p);
    check_launch();
    R.tmp.download(sol, m, h.s);
    XS_CUDA(cudaStreamSynchronize(h.s));
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    h.solve_ms = ms;
    const int e = batch_errors(h, R, R.bp);
    R.iters.assign(k, 0);
    int itmax = 0;
    for (int c = 0; c < k; c++) {
        R.iters[c] = R.S.h[c].iter;
        itmax = std::max(itmax, R.iters[c]);
    }
    h.last_iters = itmax;
    // as for k single solves: usediter / resvec / the adjoint's solution
    // describe the last right-hand side
    const KState &lst = R.S.h[k - 1];
    h.final_relres = lst.iter ? lst.rnorm / (lst.res0 + KSMALL) : (lst.res0 > 0 ? 1.0 : 0.0);
    if (h.usediter) *h.usediter = lst.iter;
    if (h.resvec) XS_CUDA(cudaMemcpy(h.resvec, lst.hist, sizeof(double) * (lst.iter + 1), cudaMemcpyDeviceToHost));
    if (e) {
        h.have_solution = false;
        throw Status(dev_err_to_status(e));
    }
    h.have_solution = true;
    adjoint_record_solution(h.adj, h.s, n, R.tmp.p + (size_t)(k - 1) * n);
    XS_CUDA(cudaStreamSynchronize(h.s));
}

static void adjoint_batch(Handle &h, int k, const double *X, const double *G, double *DB, double *DA)
{
    build_precond(h);
    bool ok = batch_ok(h, h.M, k);
    if (ok) {
        adjoint_prepare(h);
        ok = batch_precond_ok(h.adj.Mt);
    }
    if (!ok) {
        for (int c = 0; c < k; c++) {
            adjoint_set_solution(h.adj, h.s, h.n, X + (size_t)c * h.n);
            h.have_solution = true;
            adjoint_solve(h, G + (size_t)c * h.n, DB ? DB + (size_t)c * h.n : nullptr,
                          DA ? DA + (size_t)c * h.nnz : nullptr);
        }
        return;
    }
    clear_dev_err(h);
    AdjointState &a = h.adj;
    const int n = h.n;
    const long m = (long)n * k;
    BatchRuntime &R = h.batch;
    if (R.bB.n != (size_t)m) { R.bB.alloc(m); R.bX.alloc(m); R.tmp.alloc(m); }
    if (R.bY.n != (size_t)m) R.bY.alloc(m);
    const int g = geom().sms * 4;
    R.tmp.upload(G, m, h.s);
    k_interleave<<<g, 256, 0, h.s>>>(n, k, R.tmp.p, R.bB.p);  // right-hand sides dL/dx
    R.tmp.upload(X, m, h.s);
    k_interleave<<<g, 256, 0, h.s>>>(n, k, R.tmp.p, R.bY.p);  // forward solutions
    check_launch();
    XS_CUDA(cudaMemsetAsync(R.bX.p, 0, sizeof(double) * m, h.s));  // lambda0 = 0
    R.S.prepare(k, h.maxiter, h.tol, h.abstol, h.s);
    cudaEvent_t e0, e1;
    XS_CUDA(cudaEventCreate(&e0));
    XS_CUDA(cudaEventCreate(&e1));
    XS_CUDA(cudaEventRecord(e0, h.s));
    const DevCsr At{n, h.nnz, a.At.rp.p, a.At.ci.p, a.At.v.p, nullptr};
    R.pcg_t.run(h.s, At, a.Mt, R.bpt, R.S, k, R.bB.p, R.bX.p, nullptr);
    // gradients: dL/db = lambda, dL/dA = -lambda_i x_j on A's pattern, per column
    double *db = nullptr, *dA = nullptr;
    if (DB) {
        if (R.gb.n != (size_t)m) R.gb.alloc(m);
        db = R.gb.p;
    }
    if (DA) {
        const size_t mA = (size_t)k * std::max<long>(h.nnz, 1);
        if (R.gA.n != mA) R.gA.alloc(mA);
        dA = R.gA.p;
    }
    k_adjoint_grad_multi<<<g, 256, 0, h.s>>>(n, k, h.nnz, h.A.rp.p, h.A.ci.p, R.bX.p, R.bY.p, db, dA);
    check_launch();
    XS_CUDA(cudaEventRecord(e1, h.s));
    if (DB) R.gb.download(DB, m, h.s);
    if (DA) {
        if (h.vperm.empty()) R.gA.download(DA, (size_t)k * h.nnz, h.s);
        else {
            std::vector<double> t((size_t)k * h.nnz);
            R.gA.download(t.data(), t.size(), h.s);
            XS_CUDA(cudaStreamSynchronize(h.s));
            for (int c = 0; c < k; c++)
                for (long e = 0; e < h.nnz; e++) DA[(size_t)c * h.nnz + h.vperm[e]] = t[(size_t)c * h.nnz + e];
        }
    }
    XS_CUDA(cudaStreamSynchronize(h.s));
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    h.solve_ms = ms;
    const int e = batch_errors(h, R, R.bpt);
    R.iters.assign(k, 0);
    for (int c = 0; c < k; c++) R.iters[c] = R.S.h[c].iter;
    if (e) throw Status(dev_err_to_status(e));
}

// ---------------------------------------------------------------- string helpers
static bool ieq(const char *a, const char *b)
{
    if (!a || !b) return false;
    while (*a && *b) {
        char x = *a >= 'A' && *a <= 'Z' ? *a + 32 : *a;
        char y = *b >= 'A' && *b <= 'Z' ? *b + 32 : *b;
        if (x != y) return false;
        a++;
        b++;
    }
    return *a == 0 && *b == 0;
}

static int parse_ksp(const char *fmt, bool intel)
{
    if (ieq(fmt, "bicgstab")) return KSP_BICGSTAB;
    if (ieq(fmt, "cg")) return intel ? KSP_CG_LEFT : KSP_CGM;
    if (ieq(fmt, "cgm") || ieq(fmt, "pcg")) return KSP_CGM;
    if (ieq(fmt, "icg")) return KSP_ICG;
    if (ieq(fmt, "icgm")) return KSP_ICGM;
    if (ieq(fmt, "ibicgstab")) return KSP_IBICGSTAB;
    if (ieq(fmt, "igcr")) return intel ? KSP_IGCR_LEFT : KSP_GCR_RIGHT;
    if (ieq(fmt, "gcr")) return intel ? KSP_GCR_LEFT : KSP_GCR_RIGHT;
    if (ieq(fmt, "gmres")) return intel ? KSP_GMRES_LEFT : KSP_GMRES_RIGHT;
    if (ieq(fmt, "fgmres")) return KSP_GMRES_RIGHT;
    if (ieq(fmt, "gcr_left")) return KSP_GCR_LEFT;
    if (ieq(fmt, "igcr_left")) return KSP_IGCR_LEFT;
    if (ieq(fmt, "gmres_left")) return KSP_GMRES_LEFT;
    return 0;
}

static int parse_pc(const char *fmt)
{
    if (ieq(fmt, "jacobi")) return PC_JACOBI;
    if (ieq(fmt, "ilu0") || ieq(fmt, "ilu0_mkl")) return PC_ILU0;
    if (ieq(fmt, "parilu")) return PC_PARILU;
    if (ieq(fmt, "ilut") || ieq(fmt, "ilut_mkl") || ieq(fmt, "parilut")) return PC_PARILUT;
    if (ieq(fmt, "none")) return PC_NONE;
    if (ieq(fmt, "ic0")) return PC_IC0;
    if (ieq(fmt, "ict")) return PC_ICT;
    if (ieq(fmt, "ilup") || ieq(fmt, "ilut_saad")) return PC_ILUP;
    return -1;
}

static int parse_fprec(const char *s)
{
    if (ieq(s, "fp64") || ieq(s, "f64") || ieq(s, "double")) return FP_F64;
    if (ieq(s, "fp32") || ieq(s, "f32") || ieq(s, "float")) return FP_F32;
    if (ieq(s, "bf16") || ieq(s, "bfloat16")) return FP_BF16;
    if (ieq(s, "fp16") || ieq(s, "f16") || ieq(s, "half")) return FP_F16;
    return -1;
}

}  // namespace xs

using namespace xs;

// ====================================================================== C API
struct xs_handle_s {
    std::unique_ptr<Handle> h;
};

static thread_local int g_last_error = XS_OK;

template <class F>
static int guarded(F f)
{
    try {
        f();
        g_last_error = XS_OK;
    } catch (Status &s) {
        g_last_error = s.code;
    } catch (std::bad_alloc &) {
        g_last_error = XS_ERR_NOMEM;
    } catch (...) {
        g_last_error = XS_ERR_CUDA;
    }
    return g_last_error;
}

static int check_gpu()
{
    int c = 0;
    if (cudaGetDeviceCount(&c) != cudaSuccess || c <= 0) throw Status(XS_ERR_NO_GPU);
    return c;
}

extern "C" {

const char *xs_version(void) { return "xsolver_b200 1.0 (sm_100a)"; }

int xs_set_launch_overlap(int enable)
{
    return guarded([&] { pdl_tuning().enabled = enable != 0; });
}

int xs_set_sweep_fusion(int enable)
{
    return guarded([&] { trsv_tuning().fuse_sweeps = enable != 0; });
}

int xs_set_trsv_block_rows(int max_rows)
{
    return guarded([&] {
        if (max_rows < 0) throw Status(XS_ERR_INVALID);
        trsv_tuning().block_max_rows = max_rows;
    });
}

int xs_set_ilu_tiles(int enable)
{
    return guarded([&] { ilu_tiles_flag() = enable != 0; });
}

int xs_set_trsv_block_staging(int enable)
{
    return guarded([&] { trsv_tuning().lu_staged = enable != 0; });
}

int xs_set_ell_index_bits(int bits)
{
    return guarded([&] {
        if (bits != 0 && bits != 16 && bits != 32) throw Status(XS_ERR_INVALID);
        format_tuning().ell_dia = bits == 0;
        format_tuning().ell_index16 = bits != 32;
    });
}

int xs_set_trsv_tuning(int blocks_per_sm, int backoff_ns, int chunk_rows)
{
    return guarded([&] {
        if (blocks_per_sm < 0 || blocks_per_sm > 64 || backoff_ns < 8 || backoff_ns > 100000) throw Status(XS_ERR_INVALID);
        if (chunk_rows < 0 || chunk_rows > 24576) throw Status(XS_ERR_INVALID);  // 24576 doubles = 192 KiB shared
        trsv_tuning().blocks_per_sm = blocks_per_sm;
        trsv_tuning().backoff_ns = backoff_ns;
        trsv_tuning().chunk_rows = chunk_rows;
    });
}

int xs_mm_info(const char *path, int *m, int *n, int *nnz, int *symmetric)
{
    return guarded([&] {
        if (!m || !n || !nnz) throw Status(XS_ERR_INVALID);
        MmFile F;
        mm_parse(path, F);
        const long c = mm_csr_nnz(F);
        if (c > 0x7fffffffL) throw Status(XS_ERR_CAPACITY);
        *m = F.m;
        *n = F.n;
        *nnz = (int)c;
        if (symmetric) *symmetric = F.symmetric ? 1 : 0;
    });
}

int xs_mm_read(const char *path, int reference_quirks, int *rowptr, int *colidx, double *val, double *diag)
{
    return guarded([&] {
        if (!rowptr || !colidx || !val) throw Status(XS_ERR_INVALID);
        MmFile F;
        mm_parse(path, F);
        if (mm_csr_nnz(F) > 0x7fffffffL) throw Status(XS_ERR_CAPACITY);
        mm_to_csr(F, reference_quirks != 0, rowptr, colidx, val, diag);
    });
}

int xs_tri_levels(int n, const int *rp, const int *ci, int upper, int *level, int *perm, int *nlevels)
{
    return guarded([&] {
        if (n < 0 || !rp || (!ci && n > 0 && rp[n] > 0)) throw Status(XS_ERR_INVALID);
        TriHostPlan P;
        tri_analyse(n, rp, ci, upper != 0, [](int k) { return (long)k; }, P);
        if (level) std::memcpy(level, P.level.data(), sizeof(int) * n);
        if (perm) std::memcpy(perm, P.perm.data(), sizeof(int) * n);
        if (nlevels) *nlevels = P.nlevels;
    });
}

int xs_tri_tiles(int n, const int *rp, const int *ci, int upper, int tx, int ty, int tz, int *info, int *perm,
                 int *prp, int *pci, int *tile_pos, int *tile_lvl, int *lvl_ptr, int *halo_ptr, int *halo_row)
{
    return guarded([&] {
        if (n < 0 || !rp || !info || (!ci && n > 0 && rp[n] > 0) || tx < 1 || ty < 1 || tz < 1)
            throw Status(XS_ERR_INVALID);
        TileTuning tt;
        tt.tx = tx; tt.ty = ty; tt.tz = tz;
        TileHostPlan P;
        const bool ok = tri_analyse_tiles(n, rp, ci, upper != 0, [](int k) { return (long)k; }, tt, P);
        std::memset(info, 0, sizeof(int) * 12);
        info[0] = ok ? 1 : 0;
        if (!ok) return;
        info[1] = P.nx; info[2] = P.ny; info[3] = P.nz;
        info[4] = P.sa; info[5] = P.sb; info[6] = P.sc;
        info[7] = P.ntiles;
        info[8] = (int)P.lvl_ptr.size() - 1;
        info[9] = (int)P.halo_row.size();
        info[10] = P.max_rows;
        info[11] = P.max_halo;
        auto put = [](int *dst, const auto &v) {
            if (dst && !v.empty()) std::memcpy(dst, v.data(), sizeof(int) * v.size());
        };
        put(perm, P.perm); put(prp, P.prp); put(pci, P.pci); put(tile_pos, P.tile_pos);
        put(tile_lvl, P.tile_lvl); put(lvl_ptr, P.lvl_ptr); put(halo_ptr, P.halo_ptr); put(halo_row, P.halo_row);
    });
}

int xs_set_trsv_tiles(int enable, int tx, int ty, int tz, int min_rows)
{
    return guarded([&] {
        if (enable && (tx < 1 || ty < 1 || tz < 1 || min_rows < 8)) throw Status(XS_ERR_INVALID);
        tile_tuning().enable = enable != 0;
        if (enable) {
            tile_tuning().tx = tx;
            tile_tuning().ty = ty;
            tile_tuning().tz = tz;
            tile_tuning().min_rows = min_rows;
            tile_tuning().user_box = 1;
        }
    });
}

int xs_set_vector_fusion(int enable)
{
    return guarded([&] { vec_fusion_flag() = enable != 0; });
}

int xs_set_persistent_iteration(int enable)
{
    return guarded([&] { persist_tuning().enabled = enable != 0; });
}

int xs_set_batch_kernels(int enable)
{
    return guarded([&] { batch_tuning().enabled = enable != 0; });
}

int xs_device_count(void)
{
    int c = 0;
    if (cudaGetDeviceCount(&c) != cudaSuccess) return 0;
    return c;
}

const char *xsolver_error_string(int s)
{
    switch (s) {
    case XS_OK: return "ok";
    case XS_ERR_INVALID: return "invalid argument";
    case XS_ERR_CUDA: return "CUDA error";
    case XS_ERR_NOMEM: return "out of device memory";
    case XS_ERR_NO_DIAG: return "row without diagonal entry";
    case XS_ERR_TRSV_TIMEOUT: return "sync-free triangular solve timed out";
    case XS_ERR_BREAKDOWN: return "Krylov breakdown";
    case XS_ERR_NAN: return "non-finite value";
    case XS_ERR_ORDER: return "call out of order";
    case XS_ERR_ELL_WIDTH: return "ELL width out of range";
    case XS_ERR_UNSUPPORTED: return "unsupported option";
    case XS_ERR_CAPACITY: return "per-row capacity exceeded";
    case XS_ERR_NO_GPU: return "no CUDA device";
    default: return "unknown";
    }
}

int xsolver_last_error(void) { return g_last_error; }

int xs_create(xs_handle_t *out)
{
    return guarded([&] {
        if (!out) throw Status(XS_ERR_INVALID);
        check_gpu();
        auto *w = new xs_handle_s;
        w->h.reset(new Handle());
        *out = w;
    });
}
int xs_destroy(xs_handle_t h)
{
    return guarded([&] { delete h; });
}

#define HCHK(h) \
    if (!(h) || !(h)->h) throw Status(XS_ERR_INVALID)

int xs_mat_setup(xs_handle_t h, int n, const int *rp, const int *ci, const double *v, int format)
{
    return guarded([&] {
        HCHK(h);
        if (format < 0 || format > 1) throw Status(XS_ERR_UNSUPPORTED);
        set_matrix(*h->h, n, rp, ci, v, format);
    });
}
int xs_ksp_settype(xs_handle_t h, const char *fmt)
{
    return guarded([&] {
        HCHK(h);
        int m = parse_ksp(fmt, h->h->intel_conv != 0);
        if (!m) throw Status(XS_ERR_INVALID);
        h->h->method = m;
    });
}
int xs_ksp_setoption(xs_handle_t h, double tol, int maxiter, int *usediter, double *resvec, int restart)
{
    return guarded([&] {
        HCHK(h);
        if (maxiter < 0 || restart < 0 || !(tol >= 0)) throw Status(XS_ERR_INVALID);
        Handle &H = *h->h;
        H.tol = tol;
        H.maxiter = maxiter;
        H.usediter = usediter;
        H.resvec = resvec;
        H.restart = restart;
    });
}
int xs_ksp_set_absolute_tol(xs_handle_t h, double a)
{
    return guarded([&] {
        HCHK(h);
        h->h->abstol = a;
    });
}
int xs_pc_settype(xs_handle_t h, const char *fmt)
{
    return guarded([&] {
        HCHK(h);
        if (h->h->method == 0) throw Status(XS_ERR_ORDER);
        int t = parse_pc(fmt);
        if (t == -2) throw Status(XS_ERR_UNSUPPORTED);
        if (t < 0) throw Status(XS_ERR_INVALID);
        h->h->pc_req = t;
        invalidate_pc(*h->h);
    });
}
int xs_pc_setilut(xs_handle_t h, double tol, int max_fill)
{
    return guarded([&] {
        HCHK(h);
        if (max_fill < 1 || tol < 0) throw Status(XS_ERR_INVALID);
        h->h->parilut_fill = (double)max_fill;
        h->h->parilut_droptol = tol;
        h->h->ilup_fill = max_fill;
        h->h->ilup_tol = tol;
        invalidate_pc(*h->h);
    });
}
int xs_pc_setict(xs_handle_t h, double tol, int max_fill)
{
    return guarded([&] {
        HCHK(h);
        if (max_fill < 0 || !(tol > 0)) throw Status(XS_ERR_INVALID);
        h->h->ict_fill = max_fill;
        h->h->ict_tol = tol;
        invalidate_pc(*h->h);
    });
}
int xs_host_ilut(int n, const int *rp, const int *ci, const double *v, int lfil, double droptol, int *nnzL, int *nnzU,
                 int *lrp, int *lci, double *lv, double *dinv, int *urp, int *uci, double *uv)
{
    return guarded([&] {
        if (n < 0 || lfil < 1 || droptol < 0 || (n > 0 && (!rp || !ci || !v))) throw Status(XS_ERR_INVALID);
        HostTriFactors F;
        host_ilut(n, rp, ci, v, lfil, droptol, F);
        copy_host_factors(n, F, nnzL, nnzU, lrp, lci, lv, dinv, urp, uci, uv);
    });
}
int xs_host_ict(int n, const int *rp, const int *ci, const double *v, int maxfil, double droptol, int *nnzL, int *nnzU,
                int *lrp, int *lci, double *lv, double *dinv, int *urp, int *uci, double *uv)
{
    return guarded([&] {
        if (n < 0 || maxfil < 0 || !(droptol > 0) || (n > 0 && (!rp || !ci || !v))) throw Status(XS_ERR_INVALID);
        HostTriFactors F;
        if (host_ict(n, rp, ci, v, maxfil, droptol, F) >= 0) throw Status(XS_ERR_NO_DIAG);
        copy_host_factors(n, F, nnzL, nnzU, lrp, lci, lv, dinv, urp, uci, uv);
    });
}
int xs_pc_setparilu(xs_handle_t h, int sweeps)
{
    return guarded([&] {
        HCHK(h);
        if (sweeps < 0) throw Status(XS_ERR_INVALID);
        h->h->parilu_sweeps = sweeps;
        invalidate_pc(*h->h);
    });
}
int xs_pc_setparilut(xs_handle_t h, double fill, int sweeps, double droptol)
{
    return guarded([&] {
        HCHK(h);
        if (!(fill >= 1.0) || sweeps < 1 || droptol < 0) throw Status(XS_ERR_INVALID);
        h->h->parilut_fill = fill;
        h->h->parilut_sweeps = sweeps;
        h->h->parilut_droptol = droptol;
        invalidate_pc(*h->h);
    });
}
int xs_pc_set_trsv(xs_handle_t h, int mode)
{
    return guarded([&] {
        HCHK(h);
        if (mode < 0 || mode > 1000) throw Status(XS_ERR_INVALID);
        h->h->trsv_mode = mode;
        invalidate_pc(*h->h);
    });
}
int xs_set_precision(xs_handle_t h, const char *outer, const char *inner, const char *factor)
{
    return guarded([&] {
        HCHK(h);
        if (parse_fprec(outer) != FP_F64) throw Status(XS_ERR_UNSUPPORTED);
        int in = parse_fprec(inner);
        if (in != FP_F64 && in != FP_F32) throw Status(XS_ERR_UNSUPPORTED);
        int fp = parse_fprec(factor);
        if (fp < 0) throw Status(XS_ERR_INVALID);
        if (in == FP_F64 && fp != FP_F64) throw Status(XS_ERR_UNSUPPORTED);
        Handle &H = *h->h;
        H.inner32 = in == FP_F32;
        H.factor_prec = fp;
        invalidate_pc(H);
    });
}
int xs_set_inner(xs_handle_t h, double rtol, int maxit)
{
    return guarded([&] {
        HCHK(h);
        if (!(rtol > 0) || maxit < 1) throw Status(XS_ERR_INVALID);
        h->h->inner_rtol = rtol;
        h->h->inner_maxiter = maxit;
    });
}
int xs_set_refinement_mode(xs_handle_t h, int carry_krylov)
{
    return guarded([&] {
        HCHK(h);
        h->h->carry_krylov = carry_krylov != 0;
    });
}
int xs_set_compat(xs_handle_t h, int q)
{
    return guarded([&] {
        HCHK(h);
        h->h->quirk = q ? 1 : 0;
    });
}
int xs_solve(xs_handle_t h, const double *rhs, double *sol)
{
    return guarded([&] {
        HCHK(h);
        solve_host(*h->h, rhs, sol);
    });
}
int xs_solve_device(xs_handle_t h, const double *d_rhs, double *d_sol)
{
    return guarded([&] {
        HCHK(h);
        if (!d_rhs || !d_sol) throw Status(XS_ERR_INVALID);
        solve_device(*h->h, d_rhs, d_sol);
    });
}
int xs_solve_batch(xs_handle_t h, int nrhs, const double *rhs, double *sol)
{
    return guarded([&] {
        HCHK(h);
        if (nrhs < 0 || (nrhs > 0 && (!rhs || !sol))) throw Status(XS_ERR_INVALID);
        Handle &H = *h->h;
        if (nrhs == 1) solve_host(H, rhs, sol);
        else if (nrhs > 1) solve_batch(H, nrhs, rhs, sol);
    });
}
int xs_batch_iterations(xs_handle_t h, int nrhs, int *iters)
{
    return guarded([&] {
        HCHK(h);
        Handle &H = *h->h;
        if (!iters || nrhs != (int)H.batch.iters.size()) throw Status(XS_ERR_INVALID);
        for (int c = 0; c < nrhs; c++) iters[c] = H.batch.iters[c];
    });
}
int xs_mat_update(xs_handle_t h, const double *val)
{
    return guarded([&] {
        HCHK(h);
        update_values(*h->h, val);
    });
}
int xs_adjoint(xs_handle_t h, const double *dLdx, double *dLdb, double *dLdA)
{
    return guarded([&] {
        HCHK(h);
        if (!dLdx) throw Status(XS_ERR_INVALID);
        adjoint_host(*h->h, dLdx, dLdb, dLdA);
    });
}
int xs_adjoint_batch(xs_handle_t h, int nrhs, const double *x, const double *dLdx, double *dLdb, double *dLdA)
{
    return guarded([&] {
        HCHK(h);
        if (nrhs < 0 || (nrhs > 0 && (!x || !dLdx))) throw Status(XS_ERR_INVALID);
        Handle &H = *h->h;
        if (nrhs > 0) adjoint_batch(H, nrhs, x, dLdx, dLdb, dLdA);
    });
}
int xs_last_timing(xs_handle_t h, double *setup_ms, double *solve_ms, int *iterations, double *relres)
{
    return guarded([&] {
        HCHK(h);
        Handle &H = *h->h;
        if (setup_ms) *setup_ms = H.setup_ms;
        if (solve_ms) *solve_ms = H.solve_ms;
        if (iterations) *iterations = H.last_iters;
        if (relres) *relres = H.final_relres;
    });
}
int xs_get_stream(xs_handle_t h, void **stream)
{
    return guarded([&] {
        HCHK(h);
        if (!stream) throw Status(XS_ERR_INVALID);
        *stream = (void *)h->h->s;
    });
}
int xs_last_launches(xs_handle_t h, long long *count)
{
    return guarded([&] {
        HCHK(h);
        if (!count) throw Status(XS_ERR_INVALID);
        *count = h->h->launches;
    });
}
int xs_last_outer_steps(xs_handle_t h, int *o)
{
    return guarded([&] {
        HCHK(h);
        if (o) *o = h->h->last_outer;
    });
}

// ---------------------------------------------------------------- reference setter API (global handle)
static std::mutex g_mu;
static xs_handle_t g_h = nullptr;

static Handle &gh()
{
    if (!g_h) {
        if (xs_create(&g_h) != XS_OK) throw Status(g_last_error);
    }
    return *g_h->h;
}

void xsolver_mat_setup(int nInterior, int *rowptr, int *colidx, double *val, int *advanced_pam)
{
    std::lock_guard<std::mutex> lk(g_mu);
    guarded([&] {
        int fmt = 0;
        if (advanced_pam) {
            // MPI distribution (one GPU only here) and CSC input (CPU-only in
            // the reference) are refused before the matrix is taken, so no
            // rank goes on to solve its local block as if it were the system
            if (advanced_pam[0] == 1 || advanced_pam[1] == 2) throw Status(XS_ERR_UNSUPPORTED);
            if (advanced_pam[1] == 1) fmt = 1;
        }
        Handle &H = gh();
        H.intel_conv = 0;
        H.quirk = 0;
        set_matrix(H, nInterior, rowptr, colidx, val, fmt);
    });
}
void xsolver_ksp_settype(char *fmt)
{
    std::lock_guard<std::mutex> lk(g_mu);
    guarded([&] {
        Handle &H = gh();
        int m = parse_ksp(fmt, false);
        if (!m) throw Status(XS_ERR_INVALID);
        H.method = m;
    });
}
void xsolver_ksp_set_absolute_tol(double a)
{
    std::lock_guard<std::mutex> lk(g_mu);
    guarded([&] {
        Handle &H = gh();
        if (H.method == 0) throw Status(XS_ERR_ORDER);
        H.abstol = a;
    });
}
void xsolver_ksp_setoption(double tol, int maxiter, int *usediter, double *resvec, int restart)
{
    std::lock_guard<std::mutex> lk(g_mu);
    guarded([&] {
        Handle &H = gh();
        if (H.method == 0) throw Status(XS_ERR_ORDER);
        if (maxiter < 0 || restart < 0) throw Status(XS_ERR_INVALID);
        H.tol = tol;
        H.maxiter = maxiter;
        H.usediter = usediter;
        H.resvec = resvec;
        H.restart = restart;
    });
}
void xsolver_pc_settype(char *fmt)
{
    std::lock_guard<std::mutex> lk(g_mu);
    guarded([&] {
        Handle &H = gh();
        if (H.method == 0) throw Status(XS_ERR_ORDER);
        int t = parse_pc(fmt);
        if (t == -2) throw Status(XS_ERR_UNSUPPORTED);
        if (t < 0) throw Status(XS_ERR_INVALID);
        H.pc_req = t;
        invalidate_pc(H);
    });
}
void xsolver_pc_setilut(double tol, int max_fill)
{
    std::lock_guard<std::mutex> lk(g_mu);
    guarded([&] {
        Handle &H = gh();
        if (H.pc_req != PC_PARILUT && H.pc_req != PC_ILUP) return;  // ignored otherwise, as in the reference
        if (max_fill < 1 || tol < 0) throw Status(XS_ERR_INVALID);
        if (H.pc_req == PC_PARILUT) {
            H.parilut_fill = (double)max_fill;
            H.parilut_droptol = tol;
        } else {
            H.ilup_fill = max_fill;
            H.ilup_tol = tol;
        }
        invalidate_pc(H);
    });
}
void xsolver_pc_setict(double tol, int max_fill)
{
    std::lock_guard<std::mutex> lk(g_mu);
    guarded([&] {
        Handle &H = gh();
        if (H.pc_req != PC_ICT) return;  // ignored otherwise, as in the reference
        if (max_fill < 0 || !(tol > 0)) throw Status(XS_ERR_INVALID);
        H.ict_fill = max_fill;
        H.ict_tol = tol;
        invalidate_pc(H);
    });
}
void xsolver_solve(double *rhs, double *sol)
{
    std::lock_guard<std::mutex> lk(g_mu);
    guarded([&] { solve_host(gh(), rhs, sol); });
}
void xsolver_free(void)
{
    std::lock_guard<std::mutex> lk(g_mu);
    guarded([&] {
        if (g_h) xs_destroy(g_h);
        g_h = nullptr;
    });
}
void xsolver_set_precision(const char *outer, const char *inner, const char *factor)
{
    std::lock_guard<std::mutex> lk(g_mu);
    xs_handle_t h = nullptr;
    guarded([&] { gh(); h = g_h; });
    if (h) xs_set_precision(h, outer, inner, factor);
}
void xsolver_set_inner(double rtol, int maxit)
{
    std::lock_guard<std::mutex> lk(g_mu);
    xs_handle_t h = nullptr;
    guarded([&] { gh(); h = g_h; });
    if (h) xs_set_inner(h, rtol, maxit);
}
void xsolver_pc_setparilu(int sweeps)
{
    std::lock_guard<std::mutex> lk(g_mu);
    xs_handle_t h = nullptr;
    guarded([&] { gh(); h = g_h; });
    if (h) xs_pc_setparilu(h, sweeps);
}
void xsolver_pc_setparilut(double fill, int sweeps, double droptol)
{
    std::lock_guard<std::mutex> lk(g_mu);
    xs_handle_t h = nullptr;
    guarded([&] { gh(); h = g_h; });
    if (h) xs_pc_setparilut(h, fill, sweeps, droptol);
}
void xsolver_pc_set_trsv(int mode)
{
    std::lock_guard<std::mutex> lk(g_mu);
    xs_handle_t h = nullptr;
    guarded([&] { gh(); h = g_h; });
    if (h) xs_pc_set_trsv(h, mode);
}
void xsolver_set_compat(int q)
{
    std::lock_guard<std::mutex> lk(g_mu);
    guarded([&] { gh().quirk = q ? 1 : 0; });
}
void xsolver_adjoint(double *dLdx, double *dLdb, double *dLdA)
{
    std::lock_guard<std::mutex> lk(g_mu);
    guarded([&] {
        if (!dLdx) throw Status(XS_ERR_INVALID);
        adjoint_host(gh(), dLdx, dLdb, dLdA);
    });
}

// ---------------------------------------------------------------- cuda/ + intel/ Fortran-style API
static struct {
    int n = 0, nhalo = 0, nsizes = 0;
    double *diag = nullptr, *offv = nullptr;
    int *offrp = nullptr, *offci = nullptr;
} g_mc;
static xs_handle_t g_gpu = nullptr;

static void mcsr_to_csr(std::vector<int> &rp, std::vector<int> &ci, std::vector<double> &v)
{
    const int n = g_mc.n;
    rp.assign(n + 1, 0);
    ci.clear();
    v.clear();
    const int base = g_mc.offrp[0];
    if (base != 0 && base != 1) throw Status(XS_ERR_INVALID);
    // row offsets must not run backwards or past the nSizes off-diagonal
    // entries the caller's arrays hold (when it states that count; the
    // reference's device copy takes exactly nSizes entries,
    // cuda/DeviceMatrixCSR.h:60-69)
    for (int i = 0; i < n; i++)
        if (g_mc.offrp[i + 1] < g_mc.offrp[i] || (g_mc.nsizes > 0 && g_mc.offrp[i + 1] - base > g_mc.nsizes))
            throw Status(XS_ERR_INVALID);
    if (g_mc.offrp[n] > base && (!g_mc.offci || !g_mc.offv)) throw Status(XS_ERR_INVALID);
    for (int i = 0; i < n; i++) {
        std::vector<std::pair<int, double>> e;
        for (int k = g_mc.offrp[i] - base; k < g_mc.offrp[i + 1] - base; k++) e.emplace_back(g_mc.offci[k] - base, g_mc.offv[k]);
        e.emplace_back(i, g_mc.diag[i]);
        std::stable_sort(e.begin(), e.end(), [](auto &a, auto &b) { return a.first < b.first; });
        for (auto &q : e) {
            ci.push_back(q.first);
            v.push_back(q.second);
        }
        rp[i + 1] = (int)ci.size();
    }
}

void cpu_mat_setup(int *nInterior, int *nHalo, int *nSizes, double *diag_val, double *offdiag_val, int *offdiag_row_offset,
                   int *offdiag_col_index)
{
    std::lock_guard<std::mutex> lk(g_mu);
    guarded([&] {
        if (!nInterior || !diag_val || !offdiag_row_offset || (!offdiag_val && nSizes && *nSizes > 0))
            throw Status(XS_ERR_INVALID);
        g_mc.n = *nInterior;
        g_mc.nhalo = nHalo ? *nHalo : 0;
        g_mc.nsizes = nSizes ? *nSizes : 0;
        g_mc.diag = diag_val;
        g_mc.offv = offdiag_val;
        g_mc.offrp = offdiag_row_offset;
        g_mc.offci = offdiag_col_index;
        if (g_mc.nhalo != 0) throw Status(XS_ERR_UNSUPPORTED);
    });
}
void cpu_mat_update(double *diag_val, double *offdiag_val)
{
    std::lock_guard<std::mutex> lk(g_mu);
    guarded([&] {
        g_mc.diag = diag_val;
        g_mc.offv = offdiag_val;
    });
}
void gpu_mat_setup(void)
{
    std::lock_guard<std::mutex> lk(g_mu);
    guarded([&] {
        if (g_mc.n <= 0) throw Status(XS_ERR_ORDER);
        if (!g_gpu) {
            if (xs_create(&g_gpu) != XS_OK) throw Status(g_last_error);
        }
        std::vector<int> rp, ci;
        std::vector<double> v;
        mcsr_to_csr(rp, ci, v);
        Handle &H = *g_gpu->h;
        H.intel_conv = 1;
        H.quirk = 1;
        set_matrix(H, g_mc.n, rp.data(), ci.data(), v.data(), 0);
    });
}
void gpu_mat_format(char *fmt, int *num_nz)
{
    std::lock_guard<std::mutex> lk(g_mu);
    guarded([&] {
        if (!g_gpu) throw Status(XS_ERR_ORDER);
        if (!ieq(fmt, "ell")) return;
        if (!num_nz) throw Status(XS_ERR_INVALID);
        // cuda/DeviceMatrix.h:127-144: width rounded to 16 or 32, 1..32 accepted
        if (*num_nz > 0 && *num_nz <= 16) *num_nz = 16;
        else if (*num_nz > 16 && *num_nz <= 32) *num_nz = 32;
        else throw Status(XS_ERR_ELL_WIDTH);
        Handle &H = *g_gpu->h;
        // the reference's limit is on the longest row (its ELL width)
        int wmax = 0;
        for (int i = 0; i < H.n; i++) wmax = std::max(wmax, H.hrp[i + 1] - H.hrp[i]);
        if (wmax > *num_nz) throw Status(XS_ERR_ELL_WIDTH);
        operator_build_ell(H.A, H.hrp.data(), H.hci.data(), host_vals(H), 0, H.A.v32.p != nullptr, H.s);
        H.A.format = 1;
        H.format = 1;
    });
}
void gpu_mat_update(void)
{
    std::lock_guard<std::mutex> lk(g_mu);
    guarded([&] {
        if (!g_gpu) throw Status(XS_ERR_ORDER);
        std::vector<int> rp, ci;
        std::vector<double> v;
        mcsr_to_csr(rp, ci, v);
        update_values(*g_gpu->h, v.data());
    });
}
void gpu_mat_free(void)
{
    std::lock_guard<std::mutex> lk(g_mu);
    guarded([&] {
        if (g_gpu) xs_destroy(g_gpu);
        g_gpu = nullptr;
    });
}
void gpu_preconditioner_setup(char *fmt)
{
    std::lock_guard<std::mutex> lk(g_mu);
    guarded([&] {
        if (!g_gpu) throw Status(XS_ERR_ORDER);
        int t = parse_pc(fmt);
        if (t < 0) throw Status(t == -2 ? XS_ERR_UNSUPPORTED : XS_ERR_INVALID);
        g_gpu->h->pc_req = t;
        invalidate_pc(*g_gpu->h);
        build_precond(*g_gpu->h);
    });
}
void gpu_preconditioner_update(char *fmt)
{
    std::lock_guard<std::mutex> lk(g_mu);
    guarded([&] {
        if (!g_gpu) throw Status(XS_ERR_ORDER);
        (void)fmt;
        invalidate_pc(*g_gpu->h);
        build_precond(*g_gpu->h);
    });
}
void gpu_preconditioner_free(char *)
{
    std::lock_guard<std::mutex> lk(g_mu);
    guarded([&] {
        if (!g_gpu) return;
        g_gpu->h->pc_req = PC_NONE;
        invalidate_pc(*g_gpu->h);
    });
}

static void gpu_solve_common(int method, double *rhs, double *sol, int restart, double tol, int maxiter, double *sol_init,
                             int *usediter, double *resvec)
{
    if (!g_gpu) throw Status(XS_ERR_ORDER);
    Handle &H = *g_gpu->h;
    H.method = method;
    H.tol = tol;
    H.abstol = 0.0;
    H.maxiter = maxiter;
    H.restart = restart;
    H.usediter = usediter;
    H.resvec = resvec;
    H.intel_conv = 1;
    if (sol_init && sol_init != sol) std::memcpy(sol, sol_init, sizeof(double) * H.n);
    solve_host(H, rhs, sol);
}

#define GPU_SOLVE_1(NAME, METHOD)                                                                                   \
    void NAME(double *rhs, double *sol, double *tol, int *maxiter, double *sol_init, int *usediter, double *resvec) \
    {                                                                                                               \
        std::lock_guard<std::mutex> lk(g_mu);                                                                       \
        guarded([&] {                                                                                               \
            if (!tol || !maxiter) throw Status(XS_ERR_INVALID);                                                     \
            gpu_solve_common(METHOD, rhs, sol, 0, *tol, *maxiter, sol_init, usediter, resvec);                      \
        });                                                                                                         \
    }
#define GPU_SOLVE_2(NAME, METHOD)                                                                                   \
    void NAME(double *rhs, double *sol, int *restart, double *tol, int *maxiter, double *sol_init, int *usediter,  \
              double *resvec)                                                                                       \
    {                                                                                                               \
        std::lock_guard<std::mutex> lk(g_mu);                                                                       \
        guarded([&] {                                                                                               \
            if (!tol || !maxiter || !restart || *restart < 1) throw Status(XS_ERR_INVALID);                         \
            gpu_solve_common(METHOD, rhs, sol, *restart, *tol, *maxiter, sol_init, usediter, resvec);               \
        });                                                                                                         \
    }

GPU_SOLVE_1(gpu_cg_solve, KSP_CG_LEFT)
GPU_SOLVE_1(gpu_cgm_solve, KSP_CGM)
GPU_SOLVE_1(gpu_icg_solve, KSP_ICG)
GPU_SOLVE_1(gpu_icgm_solve, KSP_ICGM)
GPU_SOLVE_1(gpu_ibicgstab_solve, KSP_IBICGSTAB)
GPU_SOLVE_1(gpu_bicgstab_solve, KSP_BICGSTAB)
GPU_SOLVE_2(gpu_gcr_solve, KSP_GCR_LEFT)
GPU_SOLVE_2(gpu_igcr_solve, KSP_IGCR_LEFT)
GPU_SOLVE_2(gpu_gmres_solve, KSP_GMRES_LEFT)
GPU_SOLVE_2(gpu_fgmres_solve, KSP_GMRES_RIGHT)

}  // extern "C"

#include "xs_plan_api.cuh"
