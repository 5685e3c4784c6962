// Preconditioner objects on the device (replaces the reference's Precond
// hierarchy, hip/Precond/preconditioner.h:14-30, for the GPU cases: gpujacobi,
// gpuilu0 = ParILU, gpuilut = ParILUT; plus exact ILU(0)).
#pragma once
#include "xs_internal.cuh"
#include "xs_trsv.cuh"

namespace xs {

enum PcType { PC_NONE = 0, PC_JACOBI = 1, PC_ILU0 = 2, PC_PARILU = 3, PC_PARILUT = 4, PC_IC0 = 5, PC_ILUP = 6, PC_ICT = 7 };
// preconditioners applied as z = U'^-1 (dinv * L^-1 x)
inline bool pc_triangular(int t)
{
    return t == PC_ILU0 || t == PC_PARILU || t == PC_PARILUT || t == PC_IC0 || t == PC_ILUP || t == PC_ICT;
}
// ... whose factors have a pattern of their own (threshold factorizations)
inline bool pc_own_pattern(int t) { return t == PC_PARILUT || t == PC_ILUP || t == PC_ICT; }
enum FactorPrec { FP_F64 = 0, FP_F32 = 1, FP_BF16 = 2, FP_F16 = 3 };

template <typename VT>
__global__ void k_copy(int n, const VT *__restrict__ x, VT *__restrict__ y, const int *done_flag)
{
    if (done_flag && *done_flag) return;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) y[i] = x[i];
}
template <typename VT, typename DT>
__global__ void k_diag_scale(int n, const DT *__restrict__ d, const VT *__restrict__ x, VT *__restrict__ y,
                             const int *done_flag)
{
    if (done_flag && *done_flag) return;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) y[i] = (VT)d[i] * x[i];
}

struct PrecondDev {
    int type = PC_NONE;
    int n = 0;
    int factor_prec = FP_F64;
    int trsv_mode = 0;  // 0 exact sync-free; k > 0 Jacobi sweeps
    DBuf<double> jdiag64;
    DBuf<float> jdiag32;
    TriDev L, U;
    DBuf<double> lbuf64, ubuf64, tmp64a, tmp64b, tmp64c;
    DBuf<float> lbuf32, ubuf32, tmp32a, tmp32b, tmp32c;
    int *err = nullptr;
    bool have_factors = false;

    void ensure_buffers64(cudaStream_t s)
    {
        if (lbuf64.n != (size_t)n) {
            lbuf64.alloc(n);
            ubuf64.alloc(n);
            k_fill_sentinel<double><<<256, 256, 0, s>>>(lbuf64, n);
            k_fill_sentinel<double><<<256, 256, 0, s>>>(ubuf64, n);
            check_launch();
        }
    }
    void ensure_buffers32(cudaStream_t s)
    {
        if (lbuf32.n != (size_t)n) {
            lbuf32.alloc(n);
            ubuf32.alloc(n);
            k_fill_sentinel<float><<<256, 256, 0, s>>>(lbuf32, n);
            k_fill_sentinel<float><<<256, 256, 0, s>>>(ubuf32, n);
            check_launch();
        }
    }
    // temporaries of the Jacobi-sweep mode
    void ensure_sweep_buffers(bool need32)
    {
        if (tmp64a.n != (size_t)n) { tmp64a.alloc(n); tmp64b.alloc(n); tmp64c.alloc(n); }
        if (need32 && tmp32a.n != (size_t)n) { tmp32a.alloc(n); tmp32b.alloc(n); tmp32c.alloc(n); }
    }
    // re-arm the sentinel buffers (after an aborted solve)
    void rearm(cudaStream_t s)
    {
        if (lbuf64.n) { k_fill_sentinel<double><<<256, 256, 0, s>>>(lbuf64, n); k_fill_sentinel<double><<<256, 256, 0, s>>>(ubuf64, n); }
        if (lbuf32.n) { k_fill_sentinel<float><<<256, 256, 0, s>>>(lbuf32, n); k_fill_sentinel<float><<<256, 256, 0, s>>>(ubuf32, n); }
        check_launch();
    }

    template <typename VT>
    VT *lbuf() const;
    template <typename VT>
    VT *ubuf() const;

    // z = M^{-1} x on stream s.  x == z allowed.
    template <typename VT>
    void apply(const VT *x, VT *z, const int *done_flag, cudaStream_t s)
    {
        const int g = geom().sms * 4;
        if (type == PC_NONE) {
            if (x != z) k_copy<VT><<<g, 256, 0, s>>>(n, x, z, done_flag);
        } else if (type == PC_JACOBI) {
            if constexpr (std::is_same<VT, double>::value)
                k_diag_scale<double, double><<<g, 256, 0, s>>>(n, jdiag64.p, x, z, done_flag);
            else
                k_diag_scale<float, float><<<g, 256, 0, s>>>(n, jdiag32.p, x, z, done_flag);
        } else {
            if (trsv_mode == 0) {
                if constexpr (std::is_same<VT, double>::value) apply_exact<double, double>(x, z, done_flag, s);
                else {
                    switch (factor_prec) {
                    case FP_BF16: apply_exact<float, __nv_bfloat16>(x, z, done_flag, s); break;
                    case FP_F16: apply_exact<float, __half>(x, z, done_flag, s); break;
                    default: apply_exact<float, float>(x, z, done_flag, s); break;
                    }
                }
            } else {
                if constexpr (std::is_same<VT, double>::value) apply_sweeps<double, double>(x, z, done_flag, s);
                else {
                    switch (factor_prec) {
                    case FP_BF16: apply_sweeps<float, __nv_bfloat16>(x, z, done_flag, s); break;
                    case FP_F16: apply_sweeps<float, __half>(x, z, done_flag, s); break;
                    default: apply_sweeps<float, float>(x, z, done_flag, s); break;
                    }
                }
            }
        }
        check_launch();
    }

    template <typename VT, typename FT>
    void apply_exact(const VT *x, VT *z, const int *done_flag, cudaStream_t s)
    {
        if (!L.vals<FT>() || !U.vals<FT>()) throw Status(XS_ERR_ORDER);  // copies not built for this configuration
        if (lu_block_ok<VT>(L, U)) {
            const VT *dinv;
            if constexpr (std::is_same<VT, double>::value) dinv = U.dinv64.p;
            else dinv = U.dinv32.p;
            launch_lu_block<VT, FT, VT>(L, U, dinv, x, z, done_flag, s);
            return;
        }
        exact_half<VT, FT>(0, x, z, done_flag, s);
        exact_half<VT, FT>(1, x, z, done_flag, s);
    }
    // half 0: L solve x -> L buffer (re-arms the U buffer)
    // half 1: U solve L buffer -> z (re-arms the L buffer)
    template <typename VT, typename FT>
    void exact_half(int half, const VT *x, VT *z, const int *done_flag, cudaStream_t s)
    {
        using DT = VT;
        const DT *dinv;
        if constexpr (std::is_same<VT, double>::value) dinv = U.dinv64.p;
        else dinv = U.dinv32.p;
        VT *lb = lbuf<VT>(), *ub = ubuf<VT>();
        if (half == 0)
            launch_trsv<VT, FT, DT, false>(L, (const DT *)nullptr, x, lb, (VT *)nullptr, ub, done_flag, err, s);
        else
            launch_trsv<VT, FT, DT, true>(U, dinv, lb, ub, z, lb, done_flag, err, s);
    }
    // one half of the exact solve in the configured precision (timing)
    template <typename VT>
    void apply_half(int half, const VT *x, VT *z, cudaStream_t s)
    {
        if constexpr (std::is_same<VT, double>::value) exact_half<double, double>(half, x, z, nullptr, s);
        else {
            switch (factor_prec) {
            case FP_BF16: exact_half<float, __nv_bfloat16>(half, x, z, nullptr, s); break;
            case FP_F16: exact_half<float, __half>(half, x, z, nullptr, s); break;
            default: exact_half<float, float>(half, x, z, nullptr, s); break;
            }
        }
        check_launch();
    }

    template <typename FT>
    const FT *natvals(const TriDev &T) const;

    // A vector update can be fused into the first L pass of an apply when
    // the apply is a Jacobi-sweep solve of at least 2 sweeps whose L copy is
    // an ELL layout (the pass that reads the right-hand side at neighbours)
    bool fused_source_ok(int k) const { return k >= 2 && L.ell_w > 0; }
    bool can_fuse_first_pass() const
    {
        return pc_triangular(type) && trsv_mode >= 2 &&
               fused_source_ok(trsv_mode);
    }

    // z = M^{-1} x where the first L pass forms x from `src` (x is written
    // by that pass; see apply_sweeps).  Only when can_fuse_first_pass().
    template <typename VT, class Src>
    void apply_fused(const Src &src, const VT *x, VT *z, const int *done_flag, cudaStream_t s)
    {
        if (!can_fuse_first_pass()) throw Status(XS_ERR_INVALID);
        if constexpr (std::is_same<VT, double>::value) apply_sweeps<double, double, Src>(x, z, done_flag, s, &src);
        else {
            switch (factor_prec) {
            case FP_BF16: apply_sweeps<float, __nv_bfloat16, Src>(x, z, done_flag, s, &src); break;
            case FP_F16: apply_sweeps<float, __half, Src>(x, z, done_flag, s, &src); break;
            default: apply_sweeps<float, float, Src>(x, z, done_flag, s, &src); break;
            }
        }
        check_launch();
    }

    // srcL (optional): the first L pass reads its right-hand side from this
    // source instead of x (a vector update fused into the pass; the source
    // writes x itself, which the later passes read)
    template <typename VT, typename FT, class SrcL = SrcVec<VT>>
    void apply_sweeps(const VT *x, VT *z, const int *done_flag, cudaStream_t s, const SrcL *srcL = nullptr)
    {
        using DT = VT;
        VT *ta, *tb, *tc;
        const DT *dinv;
        if constexpr (std::is_same<VT, double>::value) { ta = tmp64a.p; tb = tmp64b.p; tc = tmp64c.p; dinv = U.dinv64_nat.p; }
        else { ta = tmp32a.p; tb = tmp32b.p; tc = tmp32c.p; dinv = U.dinv32_nat.p; }
        const int g = std::min(geom().sms * ELL_BLOCKS_PER_SM, (n + 255) / 256);
        const int k = trsv_mode;
        // one sweep pass over triangle T: ELL when available, else CSR
        auto pass = [&](const TriDev &T, bool upper, bool first2, const VT *rhs, const VT *yin, VT *yout,
                        const SrcL *fused = nullptr) {
            if (T.ell_w > 0) {
                const FT *ev = T.evals<FT>();
                if (!ev) throw Status(XS_ERR_ORDER);  // copy not built for this configuration
                const int *doff = T.doff.p;
                // one wave of resident CTAs, grid-stride over the row blocks;
                // balanced: the smallest grid of at most one wave that gives
                // every CTA the same number of row blocks (no partial last round)
                const int rb = (n + 256 * ell_rows_for<FT>() - 1) / (256 * ell_rows_for<FT>());
                const int wave = geom().sms * sweep_min_blocks_for<FT>();
                int gs = std::max(1, std::min(wave, rb));
                if (trsv_tuning().balanced_sweep_grid && rb > wave) {
                    const int per = (rb + wave - 1) / wave;
                    gs = (rb + per - 1) / per;
                }
                auto go = [&](auto cols) {
                    using CT = std::remove_const_t<std::remove_pointer_t<decltype(cols)>>;
                    const DT *dv = upper ? dinv : (const DT *)nullptr;
                    const SrcVec<VT> sv{rhs};
                    if (upper) {
                        if (first2) launch_pdl(k_trsv_sweep_ell<VT, FT, DT, CT, true, true, SrcVec<VT>>, dim3(gs), dim3(256), 0, s, n, T.ell_w, cols, doff, ev, dv, sv, yin, yout, done_flag);
                        else launch_pdl(k_trsv_sweep_ell<VT, FT, DT, CT, true, false, SrcVec<VT>>, dim3(gs), dim3(256), 0, s, n, T.ell_w, cols, doff, ev, dv, sv, yin, yout, done_flag);
                    } else if (fused) {
                        launch_pdl(k_trsv_sweep_ell<VT, FT, DT, CT, false, true, SrcL>, dim3(gs), dim3(256), 0, s, n, T.ell_w, cols, doff, ev, dv, *fused, yin, yout, done_flag);
                    } else {
                        if (first2) launch_pdl(k_trsv_sweep_ell<VT, FT, DT, CT, false, true, SrcVec<VT>>, dim3(gs), dim3(256), 0, s, n, T.ell_w, cols, doff, ev, dv, sv, yin, yout, done_flag);
                        else launch_pdl(k_trsv_sweep_ell<VT, FT, DT, CT, false, false, SrcVec<VT>>, dim3(gs), dim3(256), 0, s, n, T.ell_w, cols, doff, ev, dv, sv, yin, yout, done_flag);
                    }
                };
                if (T.ell_dia && T.ell_w <= 8) go((const uint8_t *)T.emask8.p);
                else if (T.ell_dia) go((const uint32_t *)T.emask32.p);
                else if (T.ell16) go((const short *)T.eco.p);
                else go((const int *)T.eci.p);
            } else {
                if (!natvals<FT>(T)) throw Status(XS_ERR_ORDER);  // copy not built for this configuration
                // CSR: the first sweep is a separate pass (yin = null -> y_1)
                if (first2) {
                    VT *tmp = tc;  // distinct from every buffer the stages read or write
                    if (upper) launch_pdl(k_trsv_sweep<VT, FT, DT, true>, dim3(g), dim3(256), 0, s, n, T.rp_nat, T.ci_nat, natvals<FT>(T), dinv, rhs, (const VT *)nullptr, tmp, 1, done_flag);
                    else launch_pdl(k_trsv_sweep<VT, FT, DT, false>, dim3(g), dim3(256), 0, s, n, T.rp_nat, T.ci_nat, natvals<FT>(T), (const DT *)nullptr, rhs, (const VT *)nullptr, tmp, 1, done_flag);
                    yin = tmp;
                }
                if (upper) launch_pdl(k_trsv_sweep<VT, FT, DT, true>, dim3(g), dim3(256), 0, s, n, T.rp_nat, T.ci_nat, natvals<FT>(T), dinv, rhs, yin, yout, 0, done_flag);
                else launch_pdl(k_trsv_sweep<VT, FT, DT, false>, dim3(g), dim3(256), 0, s, n, T.rp_nat, T.ci_nat, natvals<FT>(T), (const DT *)nullptr, rhs, yin, yout, 0, done_flag);
            }
        };
        if (srcL && !fused_source_ok(k)) throw Status(XS_ERR_INVALID);  // callers check first
        if (k <= 1) {
            // L^-1 x ~ x ; U'^-1 (dinv y) ~ dinv y
            k_diag_scale<VT, DT><<<g, 256, 0, s>>>(n, dinv, x, z, done_flag);
            return;
        }
        // sweeps 2 and 3 of a triangle in one pass (diagonal-slot copies with
        // few slots), further sweeps as single passes
        auto pass23 = [&](const TriDev &T, bool upper, const VT *rhs, VT *yout) {
            const FT *ev = T.evals<FT>();
            if (!ev) throw Status(XS_ERR_ORDER);
            const int gs = std::max(1, std::min(g, (n + 255) / 256));
            const uint8_t *m = T.emask8.p;
            const int *doff = T.doff.p;
            const DT *dv = upper ? dinv : (const DT *)nullptr;
#define XS_SW23(WW)                                                                                                  \
    case WW:                                                                                                         \
        if (upper) k_trsv_sweep23_dia<WW, VT, FT, DT, true><<<gs, 256, 0, s>>>(n, m, doff, ev, dv, rhs, yout, done_flag); \
        else k_trsv_sweep23_dia<WW, VT, FT, DT, false><<<gs, 256, 0, s>>>(n, m, doff, ev, dv, rhs, yout, done_flag);     \
        break;
            switch (T.ell_w) {
                XS_SW23(1) XS_SW23(2) XS_SW23(3) XS_SW23(4)
            default: throw Status(XS_ERR_INVALID);
            }
#undef XS_SW23
        };
        // a row keeps W^2 neighbour values and gathers in registers: at most
        // 4 slots (3 for 8-byte vectors) stay within the register budget
        auto fusable = [](const TriDev &T) {
            return T.ell_w > 0 && T.ell_dia && T.ell_w <= (sizeof(VT) >= 8 ? 3 : 4);
        };
        if (!srcL && k >= 3 && fusable(L) && fusable(U) && trsv_tuning().fuse_sweeps) {
            VT *cur = ta, *other = tb;
            pass23(L, false, x, cur);
            for (int t = 4; t <= k; t++) {
                pass(L, false, false, x, cur, other);
                std::swap(cur, other);
            }
            const VT *yv = cur;
            const int rest = k - 3;  // single U passes after the fused pair
            VT *first = (rest % 2 == 0) ? z : other;
            pass23(U, true, yv, first);
            VT *bufs[2] = {first, first == z ? other : z};
            for (int t = 0; t < rest; t++) pass(U, true, false, yv, bufs[t & 1], bufs[(t + 1) & 1]);
            return;
        }
        // L: passes 2..k, result in `cur` (ta or tb)
        VT *cur = ta, *other = tb;
        pass(L, false, true, x, nullptr, cur, srcL);
        for (int t = 3; t <= k; t++) {
            pass(L, false, false, x, cur, other);
            std::swap(cur, other);
        }
        // U on y = cur: k-1 passes ping-ponging between `other` and z, ending in z
        const VT *yv = cur;
        const int passes = k - 1;
        VT *bufs[2] = {(passes % 2 == 1) ? z : other, (passes % 2 == 1) ? other : z};
        pass(U, true, true, yv, nullptr, bufs[0]);
        for (int t = 1; t < passes; t++) pass(U, true, false, yv, bufs[(t - 1) & 1], bufs[t & 1]);
    }
};

template <>
inline double *PrecondDev::lbuf<double>() const { return lbuf64.p; }
template <>
inline double *PrecondDev::ubuf<double>() const { return ubuf64.p; }
template <>
inline float *PrecondDev::lbuf<float>() const { return lbuf32.p; }
template <>
inline float *PrecondDev::ubuf<float>() const { return ubuf32.p; }
template <>
inline const double *PrecondDev::natvals<double>(const TriDev &T) const { return T.nv64.p; }
template <>
inline const float *PrecondDev::natvals<float>(const TriDev &T) const { return T.nv32.p; }
template <>
inline const __nv_bfloat16 *PrecondDev::natvals<__nv_bfloat16>(const TriDev &T) const { return T.nvbf.p; }
template <>
inline const __half *PrecondDev::natvals<__half>(const TriDev &T) const { return T.nvh.p; }

}  // namespace xs
