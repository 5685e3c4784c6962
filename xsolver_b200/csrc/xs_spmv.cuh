// Sparse matrix-vector products.
//
// CSR (replaces DeviceMatrixCSR::SpMV/bmAx, hip/HostMatrix/DeviceMatrix/
// DeviceMatrixCSR.cpp:59-84, whose kernels map one thread to one row and read
// each row's entries with uncoalesced scalar loads):
//   The rows are cut into row blocks whose entries form one contiguous,
//   16-byte aligned range of at most `cap` entries.  A persistent CTA walks
//   its row blocks (block b, b+G, ...), staging each block's values and column
//   indices into shared memory with two TMA bulk copies (cp.async.bulk,
//   completion on an mbarrier), double-buffered so the copy of the next block
//   overlaps the arithmetic of the current one.  Each thread then sums one row
//   from shared memory in increasing entry order — the same order as the
//   sequential CPU loop — and gathers x through the read-only cache.  An
//   epilogue functor turns the row sum into the stored value (y = Ax,
//   y = b - Ax, ...) and accumulates fused dot products, reduced
//   deterministically across the fixed grid.
//
// ELL (replaces DeviceMatrixELL::SpMV, DeviceMatrixELL.cpp:3-34): column-major
//   val[k*n + row] with the true maximum row width (no fixed width 16); padding
//   entries point at the row itself with value 0.  Consecutive threads read
//   consecutive addresses for every k.
#pragma once
#include <type_traits>
#include "xs_internal.cuh"

namespace xs {

// ---------------------------------------------------------------- PTX helpers
__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_mbar_init()
{
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void fence_proxy_async()
{
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}
// 1D bulk copy global -> shared, completion counted on bar (no multicast)
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar)
{
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// bounded wait; returns false (and records DEV_TMA_TIMEOUT) if the copy never lands
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, uint32_t parity, int *err)
{
    if (mbar_try_wait(bar, parity)) return true;
    const unsigned long long t0 = gtimer();
    for (long it = 1;; it++) {
        if (mbar_try_wait(bar, parity)) return true;
        if ((it & 255) == 0 && gtimer() - t0 > 2 * WAIT_LIMIT_NS) break;
    }
    if (err) atomicOr(err, DEV_TMA_TIMEOUT);
    return false;
}

// ---------------------------------------------------------------- epilogues
// Epilogue interface:
//   static constexpr int K;                   number of fused dot products
//   bool active() const;                      false -> kernel exits (solver done)
//   VT out(int row, double ax);               value stored in y[row]
//   void acc(int row, double stored, double (&a)[K]);   dot contributions
//   void finalize(const double *tot);         last block, thread 0
template <typename VT>
struct EpiAx {
    static constexpr int K = 0;
    __device__ bool active() const { return true; }
    __device__ VT out(int, double ax) const { return (VT)ax; }
    __device__ void acc(int, double, double (&)[K > 0 ? K : 1]) const {}
    __device__ void finalize(const double *) const {}
};

// y = b - A x (bmAx, hip/HostMatrix/DeviceMatrix/DeviceMatrixCSR.cpp:72-84)
template <typename VT>
struct EpiBmAx {
    static constexpr int K = 0;
    const VT *b;
    __device__ bool active() const { return true; }
    __device__ VT out(int r, double ax) const { return (VT)((double)b[r] - ax); }
    __device__ void acc(int, double, double (&)[1]) const {}
    __device__ void finalize(const double *) const {}
};

// ---------------------------------------------------------------- CSR tiled kernel
template <typename MT>
struct CsrTileArgs {
    int n;
    const int *rp;
    const int *ci;
    const MT *v;
    const int *rb;
    const int *longrow;
    int nblocks;
    int cap;
    int *err;
};

constexpr int CSR_CH = 8;  // entries per gather chunk

template <typename VT, typename MT, typename Epi>
__global__ void __launch_bounds__(256) k_csr_spmv_tiled(CsrTileArgs<MT> A, const VT *__restrict__ x, VT *__restrict__ y,
                                                        Epi epi, RedSlot slot)
{
    constexpr int KK = Epi::K > 0 ? Epi::K : 1;
    pdl_trigger();
    pdl_wait();
    if (!epi.active()) return;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    __shared__ __align__(8) uint64_t bars[2];
    __shared__ double tot[KK];
    MT *vbuf[2];
    int *cbuf[2];
    vbuf[0] = (MT *)smem_raw;
    vbuf[1] = vbuf[0] + A.cap;
    cbuf[0] = (int *)(vbuf[1] + A.cap);
    cbuf[1] = cbuf[0] + A.cap;

    double acc[KK];
#pragma unroll
    for (int k = 0; k < KK; k++) acc[k] = 0.0;

    const int G = gridDim.x;
    if (threadIdx.x == 0) {
        mbar_init(&bars[0], 1);
        mbar_init(&bars[1], 1);
        fence_mbar_init();
    }
    __syncthreads();

    auto issue = [&](int b, int slotb) {
        if (A.longrow[b]) {
            // no staging: arrive without transaction bytes so the wait completes
            asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(&bars[slotb])) : "memory");
            return;
        }
        int r0 = A.rb[b], r1 = A.rb[b + 1];
        int e0 = A.rp[r0] & ~3;
        int e1 = (A.rp[r1] + 3) & ~3;
        uint32_t cnt = (uint32_t)(e1 - e0);
        uint32_t vbytes = cnt * (uint32_t)sizeof(MT), cbytes = cnt * 4u;
        if (cnt == 0) {
            asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(&bars[slotb])) : "memory");
            return;
        }
        mbar_expect_tx(&bars[slotb], vbytes + cbytes);
        bulk_g2s(vbuf[slotb], A.v + e0, vbytes, &bars[slotb]);
        bulk_g2s(cbuf[slotb], A.ci + e0, cbytes, &bars[slotb]);
    };

    int it = 0;
    if (threadIdx.x == 0 && blockIdx.x < A.nblocks) issue(blockIdx.x, 0);
    for (int b = blockIdx.x; b < A.nblocks; b += G, it++) {
        const int s = it & 1;
        if (threadIdx.x == 0 && b + G < A.nblocks) {
            fence_proxy_async();
            issue(b + G, s ^ 1);
        }
        if (!mbar_wait_bounded(&bars[s], (uint32_t)((it >> 1) & 1), A.err)) return;
        const int r0 = A.rb[b], r1 = A.rb[b + 1];
        if (!A.longrow[b]) {
            const int e0 = A.rp[r0] & ~3;
            const int r = r0 + (int)threadIdx.x;
            if (r < r1) {
                const int k0 = A.rp[r] - e0, k1 = A.rp[r + 1] - e0;
                const MT *vv = vbuf[s];
                const int *cc = cbuf[s];
                double sum = 0.0;
                // chunks of CSR_CH entries: every gather of x in a chunk is
                // issued before the chunk's (in-order) sum
                for (int kb = k0; kb < k1; kb += CSR_CH) {
                    double xv[CSR_CH];
#pragma unroll
                    for (int j = 0; j < CSR_CH; j++)
                        if (kb + j < k1) xv[j] = (double)__ldg(x + cc[kb + j]);
#pragma unroll
                    for (int j = 0; j < CSR_CH; j++)
                        if (kb + j < k1) {
                            if constexpr (sizeof(MT) <= 4 && sizeof(VT) <= 4)
                                sum = __fma_rn((double)vv[kb + j], xv[j], sum);  // exact product: same bits
                            else
                                sum += (double)vv[kb + j] * xv[j];
                        }
                }
                VT o = epi.out(r, sum);
                y[r] = o;
                if (Epi::K > 0) epi.acc(r, (double)o, acc);
            }
        } else {
            // one row longer than the staging capacity: block-wide reduction
            __shared__ double lsum[32];
            double part = 0.0;
            for (int k = A.rp[r0] + threadIdx.x; k < A.rp[r0 + 1]; k += blockDim.x)
                part += (double)A.v[k] * (double)__ldg(x + A.ci[k]);
            for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(0xffffffffu, part, o);
            if ((threadIdx.x & 31) == 0) lsum[threadIdx.x >> 5] = part;
            __syncthreads();
            if (threadIdx.x == 0) {
                double sum = 0.0;
                for (int w = 0; w < (int)(blockDim.x >> 5); w++) sum += lsum[w];
                VT o = epi.out(r0, sum);
                y[r0] = o;
                if (Epi::K > 0) epi.acc(r0, (double)o, acc);
            }
        }
        __syncthreads();
    }
    if (Epi::K > 0) {
        if (block_reduce_publish<KK>(acc, slot, tot)) {
            if (threadIdx.x == 0) epi.finalize(tot);
        }
    }
}

// ---------------------------------------------------------------- ELL kernel
// Column storage of an ELL copy, chosen per matrix when it is built:
//   CT = int       absolute column per slot
//   CT = short     offset c - row per slot (every |c - row| <= 32767, as for
//                  banded matrices: 2 index bytes per entry instead of 4)
//   CT = uint8_t / uint32_t   diagonal slots: every entry lies on one of at
//                  most 8 / 32 fixed diagonals (stencil matrices), slot k
//                  holds the entry at column row + off[k] (offsets ascending,
//                  so slot order is entry order) and the per-row bit mask in
//                  ci says which slots are present.  No per-entry index is
//                  stored and a gather address is known before any load.
template <typename CT>
struct EllDiag {
    static constexpr bool value = std::is_same<CT, uint8_t>::value || std::is_same<CT, uint32_t>::value;
};
constexpr int ELL_DIA_MAX = 32;

template <typename CT>
__device__ __forceinline__ int ell_col(CT c, int row)
{
    if constexpr (sizeof(CT) == 2) return row + (int)c;
    else return (int)c;
}

// ELL layout: slot k of row r at [k * ld + r], ld = n rounded up to
// ELL_LD_ALIGN (rows n..ld-1 are padding and never gathered), so R
// consecutive rows of one slot form one aligned vector of R elements.
constexpr int ELL_LD_ALIGN = 8;
__host__ __device__ inline long ell_ld(int n) { return ((long)n + ELL_LD_ALIGN - 1) / ELL_LD_ALIGN * ELL_LD_ALIGN; }

template <typename MT, typename CT>
struct EllArgs {
    int n, w;
    long ld;
    const CT *ci;     // columns / offsets per slot, or the per-row masks (diagonal slots)
    const MT *v;
    const int *doff;  // diagonal slots: the w offsets
};

// the diagonal offsets of a launch, staged in shared memory (slot index is
// not a compile-time constant inside the chunk loop)
template <typename CT>
__device__ __forceinline__ void ell_stage_offsets(const int *doff, int w, int *s_off)
{
    if constexpr (EllDiag<CT>::value) {
        if (threadIdx.x < (unsigned)w) s_off[threadIdx.x] = doff[threadIdx.x];
        __syncthreads();
    }
}

// Launch shape of the ELL kernels (SpMV and the Jacobi-sweep triangle
// kernels): CTAs of 256 threads, ELL_MIN_BLOCKS of them resident per SM;
// each thread takes ELL_ROWS consecutive rows (vector loads of the slot
// data) and walks the entries in chunks of ELL_CHUNK, issuing every load of
// a chunk before its gathers.  These kernels are bound by the latency of the
// dependent index -> gather loads, so the shape trades registers (rows x
// chunk in flight) against resident warps.  Default (5 CTAs of 256
// resident, 51 registers, 2 rows x 8 slots per thread) was the fastest of
// nine shapes timed on B200 for the 128^3 7-point ELL SpMV (FP32/FP64) and
// the BF16/FP32/FP64 Jacobi-sweep passes.  The grids are one wave of
// resident CTAs with a grid-stride loop: the SpMV 5 CTAs per SM, each sweep
// pass sweep_min_blocks_for<FT>() per SM (a second partial wave of CTAs cost
// 4 us of the 44 us BF16 apply and 1.8 ms of the 27 ms mixed solve at 128^3).
// ELL_BLOCKS_PER_SM sizes the grids of the CSR sweep and vector kernels.
#ifndef XS_ELL_MIN_BLOCKS
#define XS_ELL_MIN_BLOCKS 5
#endif
#ifndef XS_ELL_BLOCKS_PER_SM
#define XS_ELL_BLOCKS_PER_SM 10
#endif
#ifndef XS_ELL_ROWS
#define XS_ELL_ROWS 2
#endif
#ifndef XS_ELL_CHUNK
#define XS_ELL_CHUNK 8
#endif
constexpr int ELL_MIN_BLOCKS = XS_ELL_MIN_BLOCKS;
constexpr int ELL_BLOCKS_PER_SM = XS_ELL_BLOCKS_PER_SM;
constexpr int ELL_ROWS = XS_ELL_ROWS;
constexpr int ELL_CHUNK = XS_ELL_CHUNK;
static_assert(ELL_ROWS == 1 || ELL_ROWS == 2 || ELL_ROWS == 4 || ELL_ROWS == 8, "rows per thread");
static_assert(ELL_LD_ALIGN % ELL_ROWS == 0, "row vectors must stay aligned");
// rows per thread and slots per chunk for values of type MT (8-byte values
// have their own pair: their chunks take twice the registers)
#ifndef XS_ELL_ROWS64
#define XS_ELL_ROWS64 2
#endif
#ifndef XS_ELL_CHUNK64
#define XS_ELL_CHUNK64 4
#endif
static_assert(XS_ELL_ROWS64 == 1 || XS_ELL_ROWS64 == 2 || XS_ELL_ROWS64 == 4, "rows per thread (8-byte values)");
template <typename MT>
__host__ __device__ constexpr int ell_rows_for()
{
    return sizeof(MT) >= 8 ? XS_ELL_ROWS64 : ELL_ROWS;
}
template <typename MT>
__host__ __device__ constexpr int ell_chunk_for()
{
    return sizeof(MT) >= 8 ? XS_ELL_CHUNK64 : ELL_CHUNK;
}
// resident CTAs per SM the register budget is sized for, by value type:
// the SpMV keeps 5 for every type; the Jacobi-sweep passes with 2- and
// 4-byte factor values run fastest at full occupancy (8 CTAs, 32 registers:
// 46.3 against 49.7 us for the BF16 apply at 128^3), the FP32 SpMV at 5
// (26.7 against 34.8 us at 8)
#ifndef XS_SWEEP_MIN_BLOCKS_NARROW
#define XS_SWEEP_MIN_BLOCKS_NARROW 8
#endif
template <typename MT>
__host__ __device__ constexpr int ell_min_blocks_for()
{
    return ELL_MIN_BLOCKS;
}
template <typename FT>
__host__ __device__ constexpr int sweep_min_blocks_for()
{
    return sizeof(FT) >= 8 ? ELL_MIN_BLOCKS : XS_SWEEP_MIN_BLOCKS_NARROW;
}

// R consecutive elements starting at an R-aligned index, one vector load
// (two for 32 bytes) through the read-only path
template <int R, typename T>
__device__ __forceinline__ void ld_vec(const T *p, T (&o)[R])
{
    constexpr int B = R * (int)sizeof(T);
    if constexpr (B == 1) {
        unsigned char u = __ldg((const unsigned char *)p);
        memcpy(o, &u, 1);
    } else if constexpr (B == 2) {
        unsigned short u = __ldg((const unsigned short *)p);
        memcpy(o, &u, 2);
    } else if constexpr (B == 4) {
        unsigned u = __ldg((const unsigned *)p);
        memcpy(o, &u, 4);
    } else if constexpr (B == 8) {
        uint2 u = __ldg((const uint2 *)p);
        memcpy(o, &u, 8);
    } else if constexpr (B == 16) {
        uint4 u = __ldg((const uint4 *)p);
        memcpy(o, &u, 16);
    } else {
        static_assert(B % 16 == 0, "vector size");
#pragma unroll
        for (int q = 0; q < B / 16; q++) {
            uint4 u = __ldg((const uint4 *)p + q);
            memcpy((char *)o + 16 * q, &u, 16);
        }
    }
}

// C consecutive slots (k0 .. k0+C-1) of rows r0..r0+R-1: slot loads, then
// the gathers of x, then the per-row sums in slot order (each row's sum stays
// in entry order; a slot absent from a row adds nothing).
// Row sums accumulate in FP64 for every value type (an FP32 accumulator in
// the inner solve of the mixed-precision refinement measurably raised its
// iteration count on the 128^3 benchmark: 183 against 162 inner iterations).
#ifndef XS_ELL_ACC32
#define XS_ELL_ACC32 0
#endif
template <typename VT, typename MT>
using EllAcc = typename std::conditional<XS_ELL_ACC32 && std::is_same<VT, float>::value &&
                                             std::is_same<MT, float>::value,
                                         float, double>::type;

// sum + v * x in the accumulator type.  With FP64 sums of values and
// vector entries of at most 4 bytes the FP64 product is exact (two mantissas
// of <= 24 bits), so one fused multiply-add gives the bits of the multiply
// followed by the add with one instruction fewer; FP64 operands keep the
// separate multiply and add of the CPU order.
template <typename AT, typename MT, typename VT>
__device__ __forceinline__ AT ell_madd(AT sum, MT v, VT x)
{
    if constexpr (std::is_same<AT, double>::value && sizeof(MT) <= 4 && sizeof(VT) <= 4)
        return __fma_rn((double)v, (double)x, sum);
    else
        return sum + (AT)v * (AT)x;
}

template <int C, int R, typename VT, typename MT, typename CT, typename AT>
__device__ __forceinline__ void ell_chunk(const CT *&cp, const MT *&vp, long ld, const VT *__restrict__ x, int r0,
                                          int n, int k0, const CT (&mask)[R], const int *s_off, AT (&sum)[R])
{
    MT v[C][R];
    VT xv[C][R];
    if constexpr (EllDiag<CT>::value) {
        // gathers do not wait for the mask: every slot's column is clamped
        // into [0, n) and loaded, and the mask decides what is summed
#pragma unroll
        for (int j = 0; j < C; j++) {
            ld_vec<R>(vp, v[j]);
            vp += ld;
        }
#pragma unroll
        for (int j = 0; j < C; j++) {
            const int off = s_off[k0 + j];
#pragma unroll
            for (int q = 0; q < R; q++) xv[j][q] = XS_VLD(x + min(max(r0 + q + off, 0), n - 1));
        }
#pragma unroll
        for (int j = 0; j < C; j++)
#pragma unroll
            for (int q = 0; q < R; q++)
                if ((mask[q] >> (k0 + j)) & 1u) sum[q] = ell_madd<AT>(sum[q], v[j][q], xv[j][q]);
    } else {
        CT c[C][R];
#pragma unroll
        for (int j = 0; j < C; j++) {
            ld_vec<R>(cp, c[j]);
            ld_vec<R>(vp, v[j]);
            cp += ld;
            vp += ld;
        }
#pragma unroll
        for (int j = 0; j < C; j++)
#pragma unroll
            for (int q = 0; q < R; q++)
                xv[j][q] = (R == 1 || r0 + q < n) ? XS_VLD(x + ell_col<CT>(c[j][q], r0 + q)) : (VT)0;
#pragma unroll
        for (int j = 0; j < C; j++)
#pragma unroll
            for (int q = 0; q < R; q++) sum[q] = ell_madd<AT>(sum[q], v[j][q], xv[j][q]);
    }
}

template <int R, typename VT, typename MT, typename CT, typename AT>
__device__ __forceinline__ void ell_rows(const CT *cp, const MT *vp, int w, long ld, const VT *__restrict__ x, int r0,
                                         int n, const int *s_off, AT (&sum)[R])
{
    constexpr int CH = ell_chunk_for<MT>();
    CT mask[R];
    if constexpr (EllDiag<CT>::value) {
        ld_vec<R>(cp, mask);  // cp points at the row's mask (padding rows: 0)
    }
    for (int k0 = 0; k0 < w; k0 += CH) {
        const int m = min(CH, w - k0);  // warp-uniform
#define XS_ELL_CHUNK_CALL(CC) ell_chunk<CC, R>(cp, vp, ld, x, r0, n, k0, mask, s_off, sum)
        if (m == CH) XS_ELL_CHUNK_CALL(CH);
        else if (CH > 7 && m == 7) XS_ELL_CHUNK_CALL(7);
        else if (CH > 6 && m == 6) XS_ELL_CHUNK_CALL(6);
        else if (CH > 5 && m == 5) XS_ELL_CHUNK_CALL(5);
        else if (CH > 4 && m == 4) XS_ELL_CHUNK_CALL(4);
        else if (CH > 3 && m == 3) XS_ELL_CHUNK_CALL(3);
        else if (CH > 2 && m == 2) XS_ELL_CHUNK_CALL(2);
        else XS_ELL_CHUNK_CALL(1);
#undef XS_ELL_CHUNK_CALL
    }
}

template <typename VT, typename MT, typename CT, typename Epi>
__global__ void __launch_bounds__(256, ell_min_blocks_for<MT>()) k_ell_spmv(EllArgs<MT, CT> A, const VT *__restrict__ x,
                                                                   VT *__restrict__ y, Epi epi, RedSlot slot)
{
    constexpr int KK = Epi::K > 0 ? Epi::K : 1;
    constexpr int R = ell_rows_for<MT>();
    __shared__ double tot[KK];
    __shared__ int s_off[ELL_DIA_MAX];
    ell_stage_offsets<CT>(A.doff, A.w, s_off);  // constant data: before the dependency wait
    pdl_trigger();
    pdl_wait();
    if (!epi.active()) return;
    double acc[KK];
#pragma unroll
    for (int k = 0; k < KK; k++) acc[k] = 0.0;
    const int n = A.n;
    using AT = EllAcc<VT, MT>;
    for (int r0 = (blockIdx.x * blockDim.x + threadIdx.x) * R; r0 < n; r0 += gridDim.x * blockDim.x * R) {
        AT sum[R];
#pragma unroll
        for (int q = 0; q < R; q++) sum[q] = (AT)0;
        ell_rows<R, VT, MT, CT, AT>(A.ci + r0, A.v + r0, A.w, A.ld, x, r0, n, s_off, sum);
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

// ---------------------------------------------------------------- host side
// The matrix operator the solvers call: CSR (tiled) or ELL, FP64 or FP32 values.
struct Operator {
    int n = 0;
    long nnz = 0;
    int format = 0;  // 0 CSR, 1 ELL
    // CSR (device, padded by 8 entries for aligned bulk copies)
    DBuf<int> rp, ci;
    DBuf<double> v;
    DBuf<float> v32;
    SpmvTiling tile64, tile32;
    int grid64 = 0, grid32 = 0;  // persistent grid sizes
    // ELL: columns in eci, 16-bit row offsets in eco (ell16), or diagonal
    // slots (ell_dia: offsets in doff, per-row masks in emask8 / emask32)
    int ell_w = 0;
    bool ell16 = false;
    bool ell_dia = false;
    DBuf<int> eci;
    DBuf<short> eco;
    DBuf<int> doff;
    DBuf<uint8_t> emask8;
    DBuf<uint32_t> emask32;
    DBuf<double> ev;
    DBuf<float> ev32;
    int ell_grid = 0;
    int *err = nullptr;  // device status word

    CsrTileArgs<double> csr64() const
    {
        return CsrTileArgs<double>{n, rp.p, ci.p, v.p, tile64.rb.p, tile64.longrow.p, tile64.nblocks, tile64.cap, err};
    }
    CsrTileArgs<float> csr32() const
    {
        return CsrTileArgs<float>{n, rp.p, ci.p, v32.p, tile32.rb.p, tile32.longrow.p, tile32.nblocks, tile32.cap, err};
    }
    template <typename MT, typename CT>
    EllArgs<MT, CT> ell() const
    {
        const MT *vals;
        if constexpr (std::is_same<MT, double>::value) vals = ev.p;
        else vals = ev32.p;
        const CT *c;
        if constexpr (std::is_same<CT, uint8_t>::value) c = emask8.p;
        else if constexpr (std::is_same<CT, uint32_t>::value) c = emask32.p;
        else if constexpr (sizeof(CT) == 2) c = eco.p;
        else c = eci.p;
        return EllArgs<MT, CT>{n, ell_w, ell_ld(n), c, vals, doff.p};
    }
};

// Cut rows into blocks: at most max_rows rows, and the 4-aligned entry range
// [rp[r0] & ~3, (rp[r1] + 3) & ~3) at most cap entries.  A single row whose
// range exceeds cap becomes its own "long row" block.
inline void build_tiling(const int *h_rp, int n, int max_rows, int cap, SpmvTiling &t, cudaStream_t s)
{
    std::vector<int> rb;
    std::vector<int> lr;
    rb.reserve(n / 64 + 2);
    int r0 = 0;
    while (r0 < n) {
        int r1 = r0;
        auto span = [&](int a, int b) { return (long)(((h_rp[b] + 3) & ~3) - (h_rp[a] & ~3)); };
        if (span(r0, r0 + 1) > cap) {
            rb.push_back(r0);
            lr.push_back(1);
            r0 = r0 + 1;
            continue;
        }
        // grow while within limits (binary search would be faster; this is setup)
        int lo = r0 + 1, hi = std::min(n, r0 + max_rows);
        // largest r1 in [lo, hi] with span(r0, r1) <= cap (span is monotone in r1)
        while (lo < hi) {
            int mid = (lo + hi + 1) / 2;
            if (span(r0, mid) <= cap) lo = mid;
            else hi = mid - 1;
        }
        r1 = lo;
        rb.push_back(r0);
        lr.push_back(0);
        r0 = r1;
    }
    rb.push_back(n);
    t.nblocks = (int)lr.size();
    t.max_rows = max_rows;
    // shared-memory stage = the largest staged range actually needed (so
    // short rows leave room for more resident blocks), rounded to 64 entries
    long need = 4;
    for (size_t b = 0; b < lr.size(); b++)
        if (!lr[b]) need = std::max(need, (long)(((h_rp[rb[b + 1]] + 3) & ~3) - (h_rp[rb[b]] & ~3)));
    t.cap = (int)std::min<long>(cap, (need + 63) & ~63L);
    t.rb.alloc(rb.size());
    t.rb.upload(rb.data(), rb.size(), s);
    t.longrow.alloc(std::max<size_t>(lr.size(), 1));
    if (!lr.empty()) t.longrow.upload(lr.data(), lr.size(), s);
    XS_CUDA(cudaStreamSynchronize(s));
}

constexpr int SPMV_THREADS = 256;
constexpr int SPMV_BYTES_PER_BUF = 48 * 1024;

template <typename MT>
inline int spmv_cap()
{
    return SPMV_BYTES_PER_BUF / (int)(sizeof(MT) + sizeof(int)) & ~3;
}
template <typename MT>
inline size_t spmv_smem(int cap)
{
    return (size_t)2 * cap * (sizeof(MT) + sizeof(int));
}

template <typename VT, typename MT, typename Epi>
inline int spmv_grid(int nblocks, int cap)
{
    static int cached_cap = -1;
    static int per_sm = 1;
    static bool attr = false;
    if (!attr) {
        XS_CUDA(cudaFuncSetAttribute(k_csr_spmv_tiled<VT, MT, Epi>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)spmv_smem<MT>(spmv_cap<MT>())));
        attr = true;
    }
    if (cap != cached_cap) {
        int occ = 0;
        XS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_csr_spmv_tiled<VT, MT, Epi>, SPMV_THREADS,
                                                              spmv_smem<MT>(cap)));
        per_sm = occ > 0 ? occ : 1;
        cached_cap = cap;
    }
    long g = (long)per_sm * geom().sms;
    if (g > nblocks) g = nblocks;
    return (int)(g > 0 ? g : 1);
}

// Launch y = epi(A x) on the CSR tiled kernel (FP64 values if MT = double).
template <typename VT, typename MT, typename Epi>
inline void launch_csr(const Operator &op, const VT *x, VT *y, Epi epi, RedSlot slot, cudaStream_t s, int grid = 0)
{
    const SpmvTiling &t = std::is_same<MT, double>::value ? op.tile64 : op.tile32;
    CsrTileArgs<MT> a;
    if constexpr (std::is_same<MT, double>::value) a = op.csr64();
    else a = op.csr32();
    int g = grid > 0 ? grid : spmv_grid<VT, MT, Epi>(t.nblocks, t.cap);
    size_t sm = spmv_smem<MT>(t.cap);
    launch_pdl(k_csr_spmv_tiled<VT, MT, Epi>, dim3(g), dim3(SPMV_THREADS), sm, s, a, x, y, epi, slot);
}

// ELL SpMV on a grid whose CTAs all take the same number of row blocks
// (environment XS_ELL_BALANCED=1) instead of one full wave (default)
inline bool ell_balanced_grid()
{
    static const bool b = [] {
        const char *e = getenv("XS_ELL_BALANCED");
        return e && atoi(e) != 0;
    }();
    return b;
}

template <typename VT, typename MT, typename Epi>
inline void launch_ell(const Operator &op, const VT *x, VT *y, Epi epi, RedSlot slot, cudaStream_t s)
{
    // the grid covers the rows at ell_rows_for<MT>() rows per thread;
    // balanced: every CTA takes the same number of row blocks
    const long rb = (op.n + 256L * ell_rows_for<MT>() - 1) / (256L * ell_rows_for<MT>());
    const long wave = (long)op.ell_grid * ELL_ROWS / ell_rows_for<MT>();
    int g = (int)std::min<long>(wave, rb);
    if (ell_balanced_grid() && rb > wave) {
        const long per = (rb + wave - 1) / wave;
        g = (int)((rb + per - 1) / per);
    }
    if (op.ell_dia && op.ell_w <= 8)
        launch_pdl(k_ell_spmv<VT, MT, uint8_t, Epi>, dim3(g), dim3(256), 0, s, op.ell<MT, uint8_t>(), x, y, epi, slot);
    else if (op.ell_dia)
        launch_pdl(k_ell_spmv<VT, MT, uint32_t, Epi>, dim3(g), dim3(256), 0, s, op.ell<MT, uint32_t>(), x, y, epi, slot);
    else if (op.ell16)
        launch_pdl(k_ell_spmv<VT, MT, short, Epi>, dim3(g), dim3(256), 0, s, op.ell<MT, short>(), x, y, epi, slot);
    else
        launch_pdl(k_ell_spmv<VT, MT, int, Epi>, dim3(g), dim3(256), 0, s, op.ell<MT, int>(), x, y, epi, slot);
}

// Dispatch on the operator's format.  The grid of each path is fixed per
// operator so the fused reductions are deterministic.
template <typename VT, typename MT, typename Epi>
inline void spmv(const Operator &op, const VT *x, VT *y, Epi epi, RedSlot slot, cudaStream_t s)
{
    if (op.format == 1) launch_ell<VT, MT, Epi>(op, x, y, epi, slot, s);
    else launch_csr<VT, MT, Epi>(op, x, y, epi, slot, s);
}

// Build the operator's device CSR, tilings and (optionally) ELL from host CSR.
void operator_setup(Operator &op, int n, const int *h_rp, const int *h_ci, const double *h_v, int base,
                    bool want32, cudaStream_t s, int *d_err);
void operator_build_ell(Operator &op, const int *h_rp, const int *h_ci, const double *h_v, int base, bool want32,
                        cudaStream_t s);

}  // namespace xs
