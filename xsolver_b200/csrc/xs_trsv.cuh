// Sync-free sparse triangular solves.
//
// Replaces the reference's triangular solves of the ILU preconditioners:
//   * Lcsr_trsv_sync_free / Ucsc_trsv_sync_free (hip/Precond/gpuparilu.cpp:
//     257-364): warp per row, unbounded spin on an int flag array, per-call
//     hipMalloc, not on the default path;
//   * Lsolve_iter / Usolve_iter (DeviceMatrixCSR.cpp:281-304): the default
//     path, an approximate solve by k Jacobi sweeps (kept here as an option).
//
// Design
//   Rows are renumbered into "positions" sorted by dependency level (rows of
//   level 0 first), so every dependency of a position lies at a smaller
//   position.  Blocks take consecutive position ranges through a ticket
//   counter (atomicAdd at block start), so a block only ever waits on blocks
//   that are already running or finished: no deadlock whatever order the
//   hardware schedules blocks in.  One thread solves one row; its entries are
//   stored contiguously per position, in exactly the order the CPU reference
//   accumulates them (L: increasing column; U: decreasing column), with
//   separate multiply and subtract, so the FP64 result is bitwise identical
//   to hip/HostMatrix/HostMatrixCSR.cpp:385-409 (LUsolve).
//
//   Readiness is carried by the value itself: the solve buffer is pre-filled
//   with a NaN bit pattern that arithmetic never produces, and a row is
//   ready when its value differs from it.  A waiting thread issues the loads
//   of up to 8 dependencies at once and re-polls only the pending ones, so a
//   dependency hop costs one L2 round trip.  The L solve re-arms the U
//   buffer and the U solve re-arms the L buffer, so no separate reset pass is
//   needed.  Each spin is bounded (DEV_TRSV_TIMEOUT recorded, kernel returns),
//   and any thread seeing the error word set stops waiting.
#pragma once
#include <exception>
#include <vector>
#include <algorithm>
#include "xs_internal.cuh"
#include "xs_spmv.cuh"  // ELL column storage and launch shape

namespace xs {

constexpr int TRSV_THREADS = 128;
constexpr int TRSV_CHUNK = 8;
// single-CTA LU solve: the solution vector in shared memory (at most this
// many bytes); the staged form also holds up to LUB_MAX_BUFS level batches
// (sizes in TrsvTuning), all within LU_SMEM_LIMIT
constexpr size_t LU_BLOCK_SMEM_MAX = 200 * 1024;
constexpr int LUB_MAX_BUFS = 4;
constexpr size_t LU_SMEM_LIMIT = 227 * 1024;

// one batch buffer, filled with 16-byte copies of 16-byte aligned ranges: a
// header (the batch's code, last level + 1, first position, first entry,
// and the element shift of each copied range inside its region), the level
// starts (at most R+1), rows (R), entry offsets (R+1), U's dinv (R),
// columns (E) and values (E); each region has 16 bytes of slack for the
// rounding of its range
template <typename FT, typename DT>
struct LuBatchSmem {
    size_t hdr, lvl, row, eptr, in, pci, pv, bytes;
    static __host__ __device__ LuBatchSmem of(int R, int E)
    {
        auto al = [](size_t b) { return (b + 16 + 15) & ~(size_t)15; };
        LuBatchSmem m;
        m.hdr = 0;
        m.lvl = 64;
        m.row = m.lvl + al((size_t)(R + 1) * sizeof(int));
        m.eptr = m.row + al((size_t)R * sizeof(int));
        m.in = m.eptr + al((size_t)(R + 1) * sizeof(int));
        m.pci = m.in + al((size_t)R * sizeof(DT));
        m.pv = m.pci + al((size_t)E * sizeof(int));
        m.bytes = m.pv + al((size_t)E * sizeof(FT));
        return m;
    }
};

template <typename FT>
struct TrsvArgs {
    int n;
    const int *perm;
    const int *prp;
    const int *pci;
    const FT *pv;
};

template <typename VT>
struct CalcT {
    using T = VT;
};

// acc - y*v in the vector type; FP64: separate multiply and subtract (the
// library is compiled without FMA contraction), FP32: fused.
__device__ __forceinline__ double msub(double acc, double y, double v) { return acc - y * v; }
__device__ __forceinline__ float msub(float acc, float y, float v) { return __fmaf_rn(-y, v, acc); }
}  // namespace xs

#include "xs_trsv_tiles.cuh"  // box-scheduled exact solves (uses msub)

namespace xs {

// Launch tuning of the sync-free solves (host side, process-wide):
//   blocks_per_sm  persistent blocks per SM (0: one block per 128 positions,
//                  no persistence)
//   backoff_ns     upper bound of the exponential back-off between polls of a
//                  pending dependency (0: spin without sleeping)
// ELL column storage: diagonal slots when the pattern lies on few diagonals
// (ell_dia), else 16-bit row offsets whenever they fit (ell_index16), else
// 32-bit columns.  Applies to ELL copies built afterwards.
struct FormatTuning {
    int ell_index16 = 1;
    int ell_dia = 1;  // diagonal slots when the pattern has few diagonals
};
FormatTuning &format_tuning();
// ascending distinct diagonal offsets of a CSR pattern if it qualifies for
// diagonal ELL slots (at most ELL_DIA_MAX, at most 25% padding), else empty
std::vector<int> dia_offsets(int n, const int *rp, const int *ci);
long max_col_offset(int n, const int *rp, const int *ci);

struct TrsvTuning {
    int blocks_per_sm = 2;
    int backoff_ns = 128;
    int chunk_rows = 0;  // chunked kernel: rows per CTA chunk (0: level-ordered kernel)
    // single-CTA solve (k_lu_block) for systems of at most this many rows
    // whose solution fits in shared memory; 0 disables it
    int block_max_rows = 1 << 30;
    // Jacobi-sweep mode: sweeps 2 and 3 of a triangle in one pass (1) or
    // as two passes (0, default: on B200 at 128^3 the fused pass measured
    // 54 us against 55 us (BF16) and 94 against 87 us (FP64) — the neighbour
    // re-reads from L2 cost what the saved DRAM traffic gained)
    int fuse_sweeps = 0;
    // single-CTA solve with its level batches staged in shared memory (1) or
    // its row data loaded one level ahead from global memory (0)
    int lu_staged = 1;
    // walker threads of the staged single-CTA solve (multiple of 32, at most
    // 512; 0: the widest level's rows rounded to whole warps)
    int lu_staged_threads = 0;
    // its level batches: at most lub_rows rows and lub_entries entries, in
    // lub_bufs shared-memory buffers (copied up to lub_bufs - 1 batches
    // ahead); lub_auto sizes two buffers to fill the shared memory the
    // solution vector leaves (fewer, larger batches measured faster: 2D
    // 128^2 231 us with 768-row batches against 234 at 512 and 260-311 with
    // 3-4 smaller buffers)
    int lub_rows = 512, lub_entries = 2048, lub_bufs = 2, lub_auto = 1;
    // Jacobi-sweep passes on a grid whose CTAs all take the same number of
    // row blocks (1) or on one full wave of CTAs (0)
    int balanced_sweep_grid = 0;
};
TrsvTuning &trsv_tuning();

template <typename VT, typename FT, typename DT, bool UPPER>
__device__ __forceinline__ bool trsv_row(const TrsvArgs<FT> &P, const DT *__restrict__ dinv, const VT *rhs, VT *self,
                                         VT *out_user, VT *reset_other, int *err, int p, int backoff_ns)
{
    const int row = __ldg(P.perm + p);
    VT acc;
    if (!UPPER) {
        acc = rhs[row];
    } else {
        const VT yv = rhs[row];
        acc = yv * (VT)__ldg(dinv + p);
    }
    if (reset_other) reset_other[row] = Sentinel<VT>::value();
    const int k0 = __ldg(P.prp + p), k1 = __ldg(P.prp + p + 1);
    for (int base = k0; base < k1; base += TRSV_CHUNK) {
        const int cnt = min(TRSV_CHUNK, k1 - base);
        int c[TRSV_CHUNK];
        VT yv[TRSV_CHUNK];
        VT fv[TRSV_CHUNK];
        unsigned pending = 0;
#pragma unroll
        for (int j = 0; j < TRSV_CHUNK; j++) {
            if (j < cnt) {
                c[j] = __ldg(P.pci + base + j);
                fv[j] = (VT)FVal<FT>::ld(P.pv, base + j);
            }
        }
#pragma unroll
        for (int j = 0; j < TRSV_CHUNK; j++) {
            if (j < cnt) {
                yv[j] = ld_poll(self + c[j]);
                if (Sentinel<VT>::is(yv[j])) pending |= 1u << j;
            }
        }
        if (pending) {
            const unsigned long long t0 = gtimer();
            unsigned ns = 8;
            long spins = 0;
            while (pending) {
                // the sleep is also the yield point that lets a producer lane
                // of the same warp run: a spin without it can starve the lane
                // it waits for
                __nanosleep(ns);
                if (ns < (unsigned)backoff_ns) ns <<= 1;
#pragma unroll
                for (int j = 0; j < TRSV_CHUNK; j++) {
                    if (pending & (1u << j)) {
                        yv[j] = ld_poll(self + c[j]);
                        if (!Sentinel<VT>::is(yv[j])) pending &= ~(1u << j);
                    }
                }
                if (pending && ((++spins & 63) == 0)) {
                    if (gtimer() - t0 > WAIT_LIMIT_NS) {
                        atomicOr(err, DEV_TRSV_TIMEOUT);
                        return false;
                    }
                    if (*(volatile int *)err) return false;
                }
            }
        }
#pragma unroll
        for (int j = 0; j < TRSV_CHUNK; j++)
            if (j < cnt) acc = msub(acc, yv[j], fv[j]);
    }
    st_publish(self + row, acc);
    if (out_user) out_user[row] = acc;
    return true;
}

// Blocks take position ranges of TRSV_THREADS rows through a ticket counter
// (so a block only waits on ranges taken earlier, by running blocks).  With a
// persistent grid every block keeps taking tickets until the work runs out;
// the block that draws the last ticket (work + grid - 1) resets the counter.
template <typename VT, typename FT, typename DT, bool UPPER>
__global__ void __launch_bounds__(TRSV_THREADS) k_trsv_syncfree(TrsvArgs<FT> P, const DT *__restrict__ dinv,
                                                               const VT *rhs, VT *self, VT *out_user, VT *reset_other,
                                                               const int *done_flag, int *err, unsigned *ticket,
                                                               int backoff_ns)
{
    if (done_flag && *done_flag) return;
    __shared__ int s_blk;
    const unsigned work = (unsigned)((P.n + TRSV_THREADS - 1) / TRSV_THREADS);
    const unsigned last = work + gridDim.x - 1;
    bool ok = true;
    while (true) {
        __syncthreads();
        if (threadIdx.x == 0) {
            const unsigned t = atomicAdd(ticket, 1u);
            if (t == last) *ticket = 0u;  // every block has drawn its final ticket
            s_blk = (int)t;
        }
        __syncthreads();
        const int b = s_blk;
        if ((unsigned)b >= work) break;
        const int p = b * TRSV_THREADS + (int)threadIdx.x;
        if (ok && p < P.n) ok = trsv_row<VT, FT, DT, UPPER>(P, dinv, rhs, self, out_user, reset_other, err, p, backoff_ns);
    }
}

inline int trsv_grid(int n)
{
    const int work = (n + TRSV_THREADS - 1) / TRSV_THREADS;
    const TrsvTuning &t = trsv_tuning();
    if (t.blocks_per_sm <= 0) return work;
    long g = (long)t.blocks_per_sm * geom().sms;
    if (g > work) g = work;
    return (int)(g > 0 ? g : 1);
}

// ---------------------------------------------------------------- chunked variant
// Rows are taken in "logical" order (L: row order; U: reverse row order, so a
// dependency always has a smaller logical index) and cut into contiguous
// chunks of at most CH rows, one CTA per chunk (chunks claimed through a
// ticket in order).  Inside a chunk, rows are sorted by their local
// dependency level (levels counted over dependencies inside the chunk only);
// the CTA walks the local levels with __syncthreads between them and keeps
// every result of the chunk in shared memory, so a dependency inside the
// chunk is one shared-memory load.  A dependency on an earlier chunk is read
// from the global solve buffer with the same sentinel polling as above; the
// encoded dependency index carries the distinction (high bit set: local
// shared-memory slot).  Each thread prefetches the row data of its row in the
// next local level while it works on the current one.  The entry order and
// arithmetic per row are those of the level-ordered kernel, so results are
// bitwise identical.
template <typename FT>
struct ChunkArgs {
    int n, nchunks, ch;
    const int *lvl_off;  // per chunk: first level index (nchunks+1)
    const int *lvl_ptr;  // per level: first position (total levels + 1)
    const int *perm;
    const int *prp;
    const int *pci;      // encoded: >= 0 global row, < 0 local slot | 0x80000000
    const FT *pv;
};

constexpr int CH_THREADS = 256;
constexpr int CH_PF = 8;  // entries prefetched per row

template <typename VT, typename FT, typename DT, bool UPPER>
struct ChunkRow {
    int p = -1, row = 0, k0 = 0, k1 = 0;
    VT rhsv = 0;
    DT dv = 0;
    int c[CH_PF];
    VT f[CH_PF];
    __device__ __forceinline__ void load(const ChunkArgs<FT> &P, const DT *dinv, const VT *rhs, int pos)
    {
        p = pos;
        row = __ldg(P.perm + pos);
        k0 = __ldg(P.prp + pos);
        k1 = __ldg(P.prp + pos + 1);
        rhsv = rhs[row];
        if (UPPER) dv = __ldg(dinv + pos);
#pragma unroll
        for (int j = 0; j < CH_PF; j++)
            if (k0 + j < k1) {
                c[j] = __ldg(P.pci + k0 + j);
                f[j] = (VT)FVal<FT>::ld(P.pv, k0 + j);
            }
    }
};

template <typename VT>
__device__ __forceinline__ bool chunk_dep(int enc, const VT *ysh, const VT *self, int *err, int backoff_ns, VT &y)
{
    if (enc < 0) {
        y = ysh[enc & 0x7fffffff];
        return true;
    }
    y = ld_poll(self + enc);
    if (!Sentinel<VT>::is(y)) return true;
    const unsigned long long t0 = gtimer();
    unsigned ns = 8;
    long spins = 0;
    while (Sentinel<VT>::is(y)) {
        __nanosleep(ns);
        if (ns < (unsigned)backoff_ns) ns <<= 1;
        y = ld_poll(self + enc);
        if ((++spins & 63) == 0) {
            if (gtimer() - t0 > WAIT_LIMIT_NS) {
                atomicOr(err, DEV_TRSV_TIMEOUT);
                return false;
            }
            if (*(volatile int *)err) return false;
        }
    }
    return true;
}

template <typename VT, typename FT, typename DT, bool UPPER>
__global__ void __launch_bounds__(CH_THREADS) k_trsv_chunked(ChunkArgs<FT> P, const DT *__restrict__ dinv, const VT *rhs,
                                                             VT *self, VT *out_user, VT *reset_other,
                                                             const int *done_flag, int *err, unsigned *ticket,
                                                             int backoff_ns)
{
    if (done_flag && *done_flag) return;
    extern __shared__ __align__(16) unsigned char ch_smem[];
    VT *ysh = (VT *)ch_smem;
    __shared__ int s_chunk;
    const unsigned last = (unsigned)P.nchunks + gridDim.x - 1;
    bool ok = true;
    while (true) {
        __syncthreads();
        if (threadIdx.x == 0) {
            const unsigned t = atomicAdd(ticket, 1u);
            if (t == last) *ticket = 0u;
            s_chunk = (int)t;
        }
        __syncthreads();
        const int c = s_chunk;
        if (c >= P.nchunks) break;
        const int c0 = c * P.ch;
        const int l0 = P.lvl_off[c], l1 = P.lvl_off[c + 1];
        ChunkRow<VT, FT, DT, UPPER> cur, nxt;
        {
            const int pos = P.lvl_ptr[l0] + (int)threadIdx.x;
            if (pos < P.lvl_ptr[l0 + 1]) cur.load(P, dinv, rhs, pos);
        }
        for (int l = l0; l < l1; l++) {
            const int pa = P.lvl_ptr[l], pb = P.lvl_ptr[l + 1];
            // prefetch this thread's first row of the next level
            nxt.p = -1;
            if (l + 1 < l1) {
                const int pos = pb + (int)threadIdx.x;
                if (pos < P.lvl_ptr[l + 2]) nxt.load(P, dinv, rhs, pos);
            }
            for (int pos = pa + (int)threadIdx.x; pos < pb; pos += CH_THREADS) {
                ChunkRow<VT, FT, DT, UPPER> r;
                if (pos == cur.p) r = cur;
                else r.load(P, dinv, rhs, pos);
                if (!ok) continue;
                VT acc = UPPER ? (VT)(r.rhsv * (VT)r.dv) : r.rhsv;
                if (reset_other) reset_other[r.row] = Sentinel<VT>::value();
                for (int k = r.k0; k < r.k1 && ok; k++) {
                    const int j = k - r.k0;
                    int enc;
                    VT fv;
                    if (j < CH_PF) { enc = r.c[j]; fv = r.f[j]; }
                    else { enc = __ldg(P.pci + k); fv = (VT)FVal<FT>::ld(P.pv, k); }
                    VT y;
                    ok = chunk_dep<VT>(enc, ysh, self, err, backoff_ns, y);
                    if (ok) acc = msub(acc, y, fv);
                }
                if (!ok) continue;
                const int q = UPPER ? P.n - 1 - r.row : r.row;
                ysh[q - c0] = acc;
                st_publish(self + r.row, acc);
                if (out_user) out_user[r.row] = acc;
            }
            cur = nxt;
            __syncthreads();
        }
    }
}

// Re-arm a solve buffer (used at setup and after an aborted solve).
template <typename VT>
__global__ void k_fill_sentinel(VT *b, int n)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) b[i] = Sentinel<VT>::value();
}

// ---------------------------------------------------------------- Jacobi-sweep mode
// Reference GPU path (DeviceMatrixCSR.cpp:14-58, 281-304): y = 0, then k times
// y = x - L_off y   (L) / y = dinv*x - U' y  (U, row-scaled form).
// Each sweep reads the previous iterate and writes the next (double buffer).
template <typename VT, typename FT, typename DT, bool UPPER>
__global__ void k_trsv_sweep(int n, const int *__restrict__ rp, const int *__restrict__ ci, const FT *__restrict__ v,
                             const DT *__restrict__ dinv_row, const VT *__restrict__ x, const VT *__restrict__ yin,
                             VT *__restrict__ yout, int first, const int *done_flag)
{
    pdl_trigger();
    pdl_wait();
    if (done_flag && *done_flag) return;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        VT acc = UPPER ? (VT)(x[i] * (VT)dinv_row[i]) : x[i];
        if (!first) {
            for (int k = rp[i]; k < rp[i + 1]; k++) acc = msub(acc, yin[ci[k]], (VT)FVal<FT>::ld(v, k));
        }
        yout[i] = acc;
    }
}

// Source of a sweep pass's right-hand side x: a vector (SrcVec), or a value
// formed on the fly from other vectors (a fused vector update, which also
// stores the value of each row it owns through put()).
template <typename VT>
struct SrcVec {
    const VT *x;
    __device__ void load() {}
    __device__ VT at(int c) const { return XS_VLD(x + c); }
    __device__ void put(int, VT) const {}
};

// C consecutive slots of rows i0..i0+R-1 of a sweep pass: acc -= v * y(c),
// with y(c) = x[c] (L, first pass), dinv[c]*x[c] (U, first pass) or yin[c].
template <int C, int R, typename VT, typename FT, typename DT, typename CT, bool UPPER, bool FIRST2, class Src>
__device__ __forceinline__ void sweep_chunk(const CT *&cp, const FT *&vp, long ld, int i0, int n, int k0,
                                            const CT (&mask)[R], const int *s_off, const DT *__restrict__ dinv,
                                            const Src &x, const VT *__restrict__ yin, VT (&acc)[R])
{
    FT v[C][R];
    VT y[C][R];
    bool pr[C][R];
    int col[C][R];
    if constexpr (EllDiag<CT>::value) {
        // gathers do not wait for the mask: columns clamped into [0, n),
        // the mask decides what is subtracted
#pragma unroll
        for (int j = 0; j < C; j++) {
            ld_vec<R>(vp, v[j]);
            vp += ld;
            const int off = s_off[k0 + j];
#pragma unroll
            for (int q = 0; q < R; q++) {
                pr[j][q] = (mask[q] >> (k0 + j)) & 1u;
                col[j][q] = min(max(i0 + q + off, 0), n - 1);
            }
        }
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
            for (int q = 0; q < R; q++) {
                pr[j][q] = R == 1 || i0 + q < n;
                col[j][q] = ell_col<CT>(c[j][q], i0 + q);
            }
    }
#pragma unroll
    for (int j = 0; j < C; j++)
#pragma unroll
        for (int q = 0; q < R; q++) {
            if (EllDiag<CT>::value || pr[j][q]) {
                const int cc = col[j][q];
                if (FIRST2) y[j][q] = UPPER ? (VT)(x.at(cc) * (VT)__ldg(dinv + cc)) : x.at(cc);
                else y[j][q] = XS_VLD(yin + cc);
            } else {
                y[j][q] = (VT)0;
            }
        }
#pragma unroll
    for (int j = 0; j < C; j++)
#pragma unroll
        for (int q = 0; q < R; q++)
            if (!EllDiag<CT>::value || pr[j][q]) acc[q] = msub(acc[q], y[j][q], (VT)FVal<FT>::cvt(v[j][q]));
}

// Jacobi sweeps on a column-major ELL copy of the triangle (natural order,
// padding slot = the row itself with value 0): every slot load is coalesced.
// FIRST2 folds the first sweep into the second: the previous iterate of the
// first sweep is x itself (L) or dinv*x (U), so k sweeps cost k-1 passes.
// Launch shape as the ELL SpMV (ELL_ROWS rows per thread, ELL_CHUNK slots
// per load chunk, warp-uniform chunk lengths).
template <typename VT, typename FT, typename DT, typename CT, bool UPPER, bool FIRST2, class Src>
__global__ void __launch_bounds__(256, sweep_min_blocks_for<FT>()) k_trsv_sweep_ell(int n, int w, const CT *__restrict__ eci,
                                                                         const int *__restrict__ doff,
                                                                         const FT *__restrict__ ev,
                                                                         const DT *__restrict__ dinv,
                                                                         Src x,
                                                                         const VT *__restrict__ yin,
                                                                         VT *__restrict__ yout, const int *done_flag)
{
    constexpr int R = ell_rows_for<FT>();
    __shared__ int s_off[ELL_DIA_MAX];
    ell_stage_offsets<CT>(doff, w, s_off);  // constant data: before the dependency wait
    pdl_trigger();
    pdl_wait();
    if (done_flag && *done_flag) return;
    x.load();  // scalars the source needs (after the wait: an earlier kernel computes them)
    const long ld = ell_ld(n);
    for (int i0 = (blockIdx.x * blockDim.x + threadIdx.x) * R; i0 < n; i0 += gridDim.x * blockDim.x * R) {
        VT acc[R];
#pragma unroll
        for (int q = 0; q < R; q++) {
            const int i = i0 + q;
            if (R == 1 || i < n) {
                const VT xi = x.at(i);
                x.put(i, xi);
                acc[q] = UPPER ? (VT)(xi * (VT)dinv[i]) : xi;
            } else {
                acc[q] = (VT)0;
            }
        }
        const CT *cp = eci + i0;
        const FT *vp = ev + i0;
        CT mask[R];
        if constexpr (EllDiag<CT>::value) ld_vec<R>(cp, mask);
        constexpr int CH = ell_chunk_for<FT>();
        for (int k0 = 0; k0 < w; k0 += CH) {
            const int m = min(CH, w - k0);  // warp-uniform
#define XS_SWEEP_CHUNK(CC) \
    sweep_chunk<CC, R, VT, FT, DT, CT, UPPER, FIRST2, Src>(cp, vp, ld, i0, n, k0, mask, s_off, dinv, x, yin, acc)
            if (m == CH) XS_SWEEP_CHUNK(CH);
            else if (CH > 7 && m == 7) XS_SWEEP_CHUNK(7);
            else if (CH > 6 && m == 6) XS_SWEEP_CHUNK(6);
            else if (CH > 5 && m == 5) XS_SWEEP_CHUNK(5);
            else if (CH > 4 && m == 4) XS_SWEEP_CHUNK(4);
            else if (CH > 3 && m == 3) XS_SWEEP_CHUNK(3);
            else if (CH > 2 && m == 2) XS_SWEEP_CHUNK(2);
            else XS_SWEEP_CHUNK(1);
#undef XS_SWEEP_CHUNK
        }
#pragma unroll
        for (int q = 0; q < R; q++)
            if (R == 1 || i0 + q < n) yout[i0 + q] = acc[q];
    }
}

// Sweeps 2 and 3 in one pass (the first sweep folded in as in FIRST2), for
// diagonal-slot copies with W <= 4 slots (W a compile-time constant):
//   L: y3_i = x_i - sum_j L_ij y2_j,  y2_j = x_j - sum_k L_jk x_k
//   U: w3_i = d_i - sum_j U_ij w2_j,  w2_j = d_j - sum_k U_jk d_k,  d = dinv*y
// Each row recomputes y2 / w2 at its W neighbours instead of reading them
// from a grid-wide first pass.  With diagonal slots every address is known
// from the row index alone, so all loads of a row — its mask and values, its
// neighbours' masks and values, and the gathers of x (and dinv) — issue in
// one round; the neighbours' slot data comes mostly from L2 (rows being swept
// at the same time).  The first pass's write and read of y2 and its second
// read of the factor disappear: about half the DRAM traffic of two passes,
// one launch instead of two.  y2_j / w2_j are computed with the operations
// and order of the separate pass, so the result is identical.
template <int W, typename VT, typename FT, typename DT, bool UPPER>
__global__ void __launch_bounds__(256, ELL_MIN_BLOCKS) k_trsv_sweep23_dia(int n, const uint8_t *__restrict__ mask,
                                                                           const int *__restrict__ doff,
                                                                           const FT *__restrict__ ev,
                                                                           const DT *__restrict__ dinv,
                                                                           const VT *__restrict__ x,
                                                                           VT *__restrict__ yout, const int *done_flag)
{
    if (done_flag && *done_flag) return;
    int off[W];
#pragma unroll
    for (int a = 0; a < W; a++) off[a] = __ldg(doff + a);
    const long ld = ell_ld(n);
    auto xin = [&](int c) -> VT { return UPPER ? (VT)(__ldg(x + c) * (VT)__ldg(dinv + c)) : __ldg(x + c); };
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const unsigned mi = __ldg(mask + i);
        int j[W];
        VT vi[W];
        unsigned mj[W];
        VT xj[W];
        VT vj[W][W], xk[W][W];
#pragma unroll
        for (int a = 0; a < W; a++) {
            j[a] = min(max(i + off[a], 0), n - 1);
            vi[a] = (VT)FVal<FT>::ld(ev, (long)a * ld + i);
            mj[a] = __ldg(mask + j[a]);
            xj[a] = xin(j[a]);
#pragma unroll
            for (int b = 0; b < W; b++) {
                vj[a][b] = (VT)FVal<FT>::ld(ev, (long)b * ld + j[a]);
                xk[a][b] = xin(min(max(j[a] + off[b], 0), n - 1));
            }
        }
        VT acc = xin(i);
#pragma unroll
        for (int a = 0; a < W; a++) {
            if (!((mi >> a) & 1u)) continue;
            VT y2 = xj[a];
#pragma unroll
            for (int b = 0; b < W; b++)
                if ((mj[a] >> b) & 1u) y2 = msub(y2, xk[a][b], vj[a][b]);
            acc = msub(acc, y2, vi[a]);
        }
        yout[i] = acc;
    }
}

// dst[q] = src >= 0 ? (FT) vals[src[q]] : 0
template <typename FT>
__global__ void k_gather_convert_pad(long m, const long *__restrict__ src, const double *__restrict__ vals, FT *dst)
{
    for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < m; q += (long)gridDim.x * blockDim.x) {
        const long s = src[q];
        const double v = s >= 0 ? vals[s] : 0.0;
        if constexpr (std::is_same<FT, double>::value) dst[q] = v;
        else if constexpr (std::is_same<FT, float>::value) dst[q] = (float)v;
        else if constexpr (std::is_same<FT, __nv_bfloat16>::value) dst[q] = __double2bfloat16(v);
        else dst[q] = __double2half(v);
    }
}

// ELL copy of a triangle from its natural CSR: slot k of row i at k*ld + i
// (column, or the 16-bit offset col - i when CT = short) and the source index
// of its value (-1: padding; padding slots point at the row itself, padding
// rows n..ld-1 are never read by the solves)
template <typename CT>
__global__ void k_tri_ell_build(int n, int w, long ld, const int *__restrict__ rp, const int *__restrict__ ci,
                                const long *__restrict__ src, CT *ecol, long *esrc)
{
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < ld; i += (long)gridDim.x * blockDim.x) {
        const int k0 = i < n ? rp[i] : 0;
        const int len = i < n ? rp[i + 1] - k0 : 0;
        for (int k = 0; k < w; k++) {
            int c = (int)(i < n ? i : 0);
            long es = -1;
            if (k < len) {
                c = ci[k0 + k];
                es = src[k0 + k];
            }
            if constexpr (sizeof(CT) == 2) ecol[(long)k * ld + i] = (CT)(i < n ? c - (int)i : 0);
            else ecol[(long)k * ld + i] = (CT)c;
            esrc[(long)k * ld + i] = es;
        }
    }
}

// diagonal-slot copy of a triangle: per-row slot mask and the source index
// of each slot's value (-1: absent; padding rows have mask 0)
template <typename MaskT>
__global__ void k_tri_dia_build(int n, int D, long ld, const int *__restrict__ rp, const int *__restrict__ ci,
                                const long *__restrict__ src, const int *__restrict__ doff, MaskT *mask, long *esrc)
{
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < ld; i += (long)gridDim.x * blockDim.x) {
        for (int k = 0; k < D; k++) esrc[(long)k * ld + i] = -1;
        uint32_t m = 0;
        if (i < n) {
            for (int q = rp[i]; q < rp[i + 1]; q++) {
                const int off = ci[q] - (int)i;
                int k = 0;
                while (k < D - 1 && doff[k] != off) k++;
                esrc[(long)k * ld + i] = src[q];
                m |= 1u << k;
            }
        }
        mask[i] = (MaskT)m;
    }
}

// level-ordered entry arrays from the natural CSR: position p holds row
// perm[p]; its entries in increasing column order (L) or decreasing (U)
static __global__ void k_pos_entries(int n, bool upper, const int *__restrict__ perm, const int *__restrict__ prp,
                              const int *__restrict__ rp, const int *__restrict__ ci, const long *__restrict__ src_nat,
                              int *pci, long *src)
{
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
        const int row = perm[p], o = prp[p], len = prp[p + 1] - o;
        for (int k = 0; k < len; k++) {
            const int q = upper ? rp[row + 1] - 1 - k : rp[row] + k;
            pci[o + k] = ci[q];
            src[o + k] = src_nat ? src_nat[q] : (long)q;
        }
    }
}
static __global__ void k_iota_long(long m, long *a)
{
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < m; i += (long)gridDim.x * blockDim.x) a[i] = i;
}

// ---------------------------------------------------------------- host plan building
// Host-side analysis of a triangular pattern.
struct TriHostPlan {
    int n = 0;
    int nlevels = 0;
    std::vector<int> perm;  // position -> row
    std::vector<int> prp;   // position rowptr
    std::vector<int> pci;   // dependency row per entry
    std::vector<long> src;  // source index of each entry in the value array
    std::vector<int> level; // per row
    std::vector<int> lstart;  // first position of each level (nlevels + 1)
};

// rp/ci: CSR of the strict triangle (0-based); src_of(k) maps entry k of the
// triangle's CSR to its index in the value array the values will be gathered
// from.  upper: dependencies on larger rows, entries summed in decreasing
// column order.
template <typename SrcF>
inline void tri_analyse(int n, const int *rp, const int *ci, bool upper, SrcF src_of, TriHostPlan &h,
                        bool entries = true)
{
    h.n = n;
    h.level.assign(n, 0);
    int maxl = 0;
    if (!upper) {
        for (int i = 0; i < n; i++) {
            int l = 0;
            for (int k = rp[i]; k < rp[i + 1]; k++) l = std::max(l, h.level[ci[k]] + 1);
            h.level[i] = l;
            maxl = std::max(maxl, l);
        }
    } else {
        for (int i = n - 1; i >= 0; i--) {
            int l = 0;
            for (int k = rp[i]; k < rp[i + 1]; k++) l = std::max(l, h.level[ci[k]] + 1);
            h.level[i] = l;
            maxl = std::max(maxl, l);
        }
    }
    h.nlevels = n > 0 ? maxl + 1 : 0;
    // counting sort by level; inside a level rows follow the solve direction
    // (L ascending, U descending), so the first rows of a level depend on the
    // first rows of the level before and can start while its tail still runs
    std::vector<int> cnt(h.nlevels + 1, 0);
    for (int i = 0; i < n; i++) cnt[h.level[i] + 1]++;
    for (int l = 0; l < h.nlevels; l++) cnt[l + 1] += cnt[l];
    h.lstart.assign(cnt.begin(), cnt.end());
    h.perm.assign(n, 0);
    if (!upper)
        for (int i = 0; i < n; i++) h.perm[cnt[h.level[i]]++] = i;
    else
        for (int i = n - 1; i >= 0; i--) h.perm[cnt[h.level[i]]++] = i;
    h.prp.assign(n + 1, 0);
    for (int p = 0; p < n; p++) {
        int r = h.perm[p];
        h.prp[p + 1] = h.prp[p] + (rp[r + 1] - rp[r]);
    }
    if (!entries) return;  // pci/src are built on the device (k_pos_entries)
    long nnz = h.prp[n];
    h.pci.assign(nnz, 0);
    h.src.assign(nnz, 0);
    for (int p = 0; p < n; p++) {
        int r = h.perm[p];
        int q = h.prp[p];
        if (!upper) {
            for (int k = rp[r]; k < rp[r + 1]; k++, q++) { h.pci[q] = ci[k]; h.src[q] = src_of(k); }
        } else {
            for (int k = rp[r + 1] - 1; k >= rp[r]; k--, q++) { h.pci[q] = ci[k]; h.src[q] = src_of(k); }
        }
    }
}

// Chunked layout (see k_trsv_chunked).  Produces perm/prp/src as
// tri_analyse does plus the encoded dependency array, chunk level offsets
// and level position pointers.
struct TriChunkPlan {
    int n = 0, ch = 0, nchunks = 0, maxlevels = 0;
    std::vector<int> perm, prp, pci_enc, lvl_off, lvl_ptr;
    std::vector<long> src;
};

template <typename SrcF>
inline void tri_analyse_chunked(int n, const int *rp, const int *ci, bool upper, SrcF src_of, int ch, TriChunkPlan &h)
{
    h.n = n;
    h.ch = ch;
    h.nchunks = (n + ch - 1) / ch;
    h.perm.assign(n, 0);
    h.prp.assign(n + 1, 0);
    h.lvl_off.assign(h.nchunks + 1, 0);
    h.lvl_ptr.clear();
    std::vector<int> lev(n, 0);  // by logical index
    auto row_of = [&](int q) { return upper ? n - 1 - q : q; };
    auto logical = [&](int r) { return upper ? n - 1 - r : r; };
    int pos = 0;
    for (int c = 0; c < h.nchunks; c++) {
        const int c0 = c * ch, c1 = std::min(n, c0 + ch);
        int maxl = 0;
        for (int q = c0; q < c1; q++) {
            const int r = row_of(q);
            int l = 0;
            for (int k = rp[r]; k < rp[r + 1]; k++) {
                const int qd = logical(ci[k]);
                if (qd >= c0) l = std::max(l, lev[qd] + 1);
            }
            lev[q] = l;
            maxl = std::max(maxl, l);
        }
        const int nl = maxl + 1;
        std::vector<int> cnt(nl + 1, 0);
        for (int q = c0; q < c1; q++) cnt[lev[q] + 1]++;
        for (int l = 0; l < nl; l++) cnt[l + 1] += cnt[l];
        h.lvl_off[c] = (int)h.lvl_ptr.size();
        for (int l = 0; l < nl; l++) h.lvl_ptr.push_back(pos + cnt[l]);
        std::vector<int> fillp(cnt.begin(), cnt.end() - 1);
        for (int q = c0; q < c1; q++) h.perm[pos + fillp[lev[q]]++] = row_of(q);
        pos += c1 - c0;
        h.maxlevels = std::max(h.maxlevels, nl);
    }
    h.lvl_off[h.nchunks] = (int)h.lvl_ptr.size();
    h.lvl_ptr.push_back(n);
    for (int p = 0; p < n; p++) {
        const int r = h.perm[p];
        h.prp[p + 1] = h.prp[p] + (rp[r + 1] - rp[r]);
    }
    const long nnz = h.prp[n];
    h.pci_enc.assign(nnz, 0);
    h.src.assign(nnz, 0);
    for (int p = 0; p < n; p++) {
        const int r = h.perm[p];
        const int c0 = (logical(r) / ch) * ch;
        int q = h.prp[p];
        auto put = [&](int k) {
            const int d = ci[k];
            const int qd = logical(d);
            h.pci_enc[q] = qd >= c0 ? (int)(0x80000000u | (unsigned)(qd - c0)) : d;
            h.src[q] = src_of(k);
            q++;
        };
        if (!upper)
            for (int k = rp[r]; k < rp[r + 1]; k++) put(k);
        else
            for (int k = rp[r + 1] - 1; k >= rp[r]; k--) put(k);
    }
}

// Device copy of a triangle prepared for the sync-free solve.  Values are
// gathered on the device from a value array (so re-factorisation or a change
// of storage precision does not repeat the host analysis).
struct TriDev {
    int n = 0;
    long nnz = 0;
    int nlevels = 0;
    bool upper = false;
    DBuf<int> perm, prp, pci;
    DBuf<long> src;
    DBuf<int> lstart;            // level-ordered layout: first position of each level
    DBuf<int> rp_nat, ci_nat;    // natural-order CSR of the triangle (Jacobi-sweep mode)
    DBuf<long> src_nat;
    DBuf<double> pv64, nv64;     // position-order and natural-order values (FP64)
    DBuf<float> pv32, nv32;
    DBuf<__nv_bfloat16> pvbf, nvbf;
    DBuf<__half> pvh, nvh;
    DBuf<double> dinv64;         // U: per position; also natural order for sweeps
    DBuf<float> dinv32;
    DBuf<double> dinv64_nat;
    DBuf<float> dinv32_nat;
    DBuf<unsigned> ticket;
    // natural-order ELL copy for the Jacobi-sweep mode (ell_w = 0: none)
    int ell_w = 0;
    bool ell16 = false;    // columns as 16-bit row offsets in eco
    bool ell_dia = false;  // diagonal slots: offsets in doff, per-row masks in emask8 / emask32
    DBuf<int> eci;
    DBuf<short> eco;
    DBuf<int> doff;
    DBuf<uint8_t> emask8;
    DBuf<uint32_t> emask32;
    DBuf<long> esrc;
    DBuf<double> ev64;
    DBuf<float> ev32;
    DBuf<__nv_bfloat16> evbf;
    DBuf<__half> evh;
    template <typename FT>
    const FT *evals() const;
    // chunked layout (perm/prp/pci then hold the chunk-major order, pci encoded)
    bool chunked = false;
    int nchunks = 0, ch = 0;
    DBuf<int> lvl_off, lvl_ptr;
    // tile layout (perm/prp/pci then hold the box-major order, pci = shared-
    // memory slots); lvperm keeps the dependency-level order for the
    // factorisation kernels, which take rows in level order
    // single-CTA staged solve (small systems): consecutive whole levels in
    // batches of at most TrsvTuning::lub_rows rows and lub_entries entries; lub[b] is
    // batch b's first level (nlub + 1 values), or -1 - level for a level too
    // large to stage (solved from global memory)
    int nlub = 0;
    int lub_rows = 0, lub_entries = 0;  // batch limits the list was built with
    int max_level_rows = 0;  // widest dependency level (level layout)
    DBuf<int> lub;
    bool tiled = false;
    int ntiles = 0, tile_elems = 0;  // tile_elems: shared-memory values per box (rows + halo)
    int t_max_rows = 0, t_max_halo = 0, t_max_entries = 0;
    DBuf<int> t_pos, t_lvl, t_lptr, t_hptr, t_hrow, lvperm;
    const int *level_perm() const { return tiled ? lvperm.p : perm.p; }
    template <typename FT>
    TileArgs<FT> targs() const
    {
        return TileArgs<FT>{n,       ntiles, t_pos.p, t_lvl.p, t_lptr.p,   t_hptr.p,   t_hrow.p,
                            perm.p,  prp.p,  pci.p,   vals<FT>(), t_max_rows, t_max_halo, t_max_entries};
    }

    template <typename FT>
    TrsvArgs<FT> args() const;
    template <typename FT>
    ChunkArgs<FT> cargs() const
    {
        return ChunkArgs<FT>{n, nchunks, ch, lvl_off.p, lvl_ptr.p, perm.p, prp.p, pci.p, vals<FT>()};
    }
    template <typename FT>
    const FT *vals() const;
};
template <>
inline const double *TriDev::evals<double>() const { return ev64.p; }
template <>
inline const float *TriDev::evals<float>() const { return ev32.p; }
template <>
inline const __nv_bfloat16 *TriDev::evals<__nv_bfloat16>() const { return evbf.p; }
template <>
inline const __half *TriDev::evals<__half>() const { return evh.p; }
template <>
inline const double *TriDev::vals<double>() const { return pv64.p; }
template <>
inline const float *TriDev::vals<float>() const { return pv32.p; }
template <>
inline const __nv_bfloat16 *TriDev::vals<__nv_bfloat16>() const { return pvbf.p; }
template <>
inline const __half *TriDev::vals<__half>() const { return pvh.p; }

template <>
inline TrsvArgs<double> TriDev::args<double>() const { return TrsvArgs<double>{n, perm.p, prp.p, pci.p, pv64.p}; }
template <>
inline TrsvArgs<float> TriDev::args<float>() const { return TrsvArgs<float>{n, perm.p, prp.p, pci.p, pv32.p}; }
template <>
inline TrsvArgs<__nv_bfloat16> TriDev::args<__nv_bfloat16>() const
{
    return TrsvArgs<__nv_bfloat16>{n, perm.p, prp.p, pci.p, pvbf.p};
}
template <>
inline TrsvArgs<__half> TriDev::args<__half>() const { return TrsvArgs<__half>{n, perm.p, prp.p, pci.p, pvh.p}; }

// gather + convert: dst[q] = (FT) src_vals[src[q]]
template <typename FT>
__global__ void k_gather_convert(long m, const long *__restrict__ src, const double *__restrict__ vals, FT *dst)
{
    for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < m; q += (long)gridDim.x * blockDim.x) {
        double v = vals[src[q]];
        if constexpr (std::is_same<FT, double>::value) dst[q] = v;
        else if constexpr (std::is_same<FT, float>::value) dst[q] = (float)v;
        else if constexpr (std::is_same<FT, __nv_bfloat16>::value) dst[q] = __double2bfloat16(v);
        else dst[q] = __double2half(v);
    }
}
// dinv per position: dst[p] = vals[diagpos[perm[p]]]
template <typename DT>
__global__ void k_gather_dinv(int n, const int *__restrict__ perm, const long *__restrict__ diagsrc,
                              const double *__restrict__ vals, DT *dst)
{
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
        int r = perm ? perm[p] : p;
        dst[p] = (DT)vals[diagsrc[r]];
    }
}

}  // namespace xs

namespace xs {

// a() on this host thread and b() on a second one, returning when both are
// done; the second thread takes the caller's current device, and the first
// exception either throws is rethrown.  Used to analyse a factor's two
// triangles at once (independent host work, uploads on one stream).
template <typename A, typename B>
inline void host_both(A a, B b)
{
    int dev = 0;
    XS_CUDA(cudaGetDevice(&dev));
    (void)geom();  // lazily initialised process-wide settings: set before the second thread reads them
    (void)trsv_tuning();
    (void)tile_tuning();
    std::exception_ptr ea, eb;
    std::thread t([&] {
        try {
            XS_CUDA(cudaSetDevice(dev));
            b();
        } catch (...) {
            eb = std::current_exception();
        }
    });
    try {
        a();
    } catch (...) {
        ea = std::current_exception();
    }
    t.join();
    if (ea) std::rethrow_exception(ea);
    if (eb) std::rethrow_exception(eb);
}

// Build the device plan of a strict triangle (natural CSR rp/ci, src_of maps
// an entry to its index in the value array) in the layout the tuning selects,
// plus the natural-order copy used by the Jacobi-sweep mode.
template <typename SrcF, typename RV, typename CV>
// rp/ci: std::vector<int> or HostArray<int>
// identity_src: entry k's value is vals[k] (src_of is not called)
// d_rp/d_ci: the same pattern already on the device (copied instead of uploaded)
// need_levels: keep the level order of a triangle that gets boxes (the
// level-ordered ILU(0)/IC(0) kernels read it); without it a boxed
// triangle skips the level analysis (nlevels = -1)
inline void build_tri_dev(TriDev &T, int n, const RV &rp, const CV &ci, bool upper, SrcF src_of,
                          cudaStream_t s, bool identity_src = false, const int *d_rp = nullptr,
                          const int *d_ci = nullptr, bool need_levels = true)
{
    TriHostPlan P;  // level analysis (also gives the level count)
    const int chr = trsv_tuning().chunk_rows;
    T.chunked = chr > 0;
    auto level_analysis = [&]() {
        Trace tr_an("    level analysis", s);
        tri_analyse(n, rp.data(), ci.data(), upper, src_of, P, /*entries=*/false);
    };
    Trace tr_up("    upload + positions", s);
    Trace tr_nat("      natural CSR + sources", s);
    T.n = n;
    T.nnz = rp[n];
    T.nlevels = -1;
    T.upper = upper;
    const long m = std::max<long>(T.nnz, 1);
    const int g = geom().sms * 4;
    // natural CSR and the source index of each entry's value
    T.rp_nat.alloc(n + 1);
    T.ci_nat.alloc(m);
    if (d_rp && d_ci) {
        XS_CUDA(cudaMemcpyAsync(T.rp_nat.p, d_rp, sizeof(int) * (n + 1), cudaMemcpyDeviceToDevice, s));
        if (T.nnz) XS_CUDA(cudaMemcpyAsync(T.ci_nat.p, d_ci, sizeof(int) * T.nnz, cudaMemcpyDeviceToDevice, s));
    } else {
        T.rp_nat.upload(rp.data(), n + 1, s);
        if (T.nnz) T.ci_nat.upload(ci.data(), T.nnz, s);
    }
    T.src_nat.alloc(m);
    if (identity_src) {
        k_iota_long<<<g, 256, 0, s>>>(T.nnz, T.src_nat.p);
    } else {
        HostArray<long> ns(T.nnz);  // written in full below
        host_parallel_for((T.nnz + 65535) / 65536, 1, [&](long b) {
            const long k1 = std::min<long>(T.nnz, (b + 1) * 65536);
            for (long k = b * 65536; k < k1; k++) ns[k] = src_of((int)k);
        });
        if (T.nnz) T.src_nat.upload(ns.data(), T.nnz, s);
    }
    tr_nat.stop();
    // box layout for patterns on a structured grid (large triangles only);
    // boxes shrink until the rows and halo of one fit in shared memory
    TileHostPlan TP;
    T.tiled = false;
    T.t_pos.free(); T.t_lvl.free(); T.t_lptr.free(); T.t_hptr.free(); T.t_hrow.free(); T.lvperm.free();
    if (!T.chunked && tile_tuning().enable && n >= tile_tuning().min_rows) {
        Trace tr_tile("    box analysis", s);
        TileTuning tt = tile_tuning();
        TileGrid G;
        Trace tr_det("      grid detection", s);
        const bool on_grid = tile_detect(n, rp.data(), ci.data(), upper, G);
        tr_det.stop();
        if (on_grid) {
            auto shrink = [&]() {
                int &big = tt.tx >= tt.ty && tt.tx >= tt.tz ? tt.tx : (tt.ty >= tt.tz ? tt.ty : tt.tz);
                if (big <= 2) return false;
                big /= 2;
                return true;
            };
            // first guess from the mean entries per row (a box of mean rows,
            // its halo a quarter of its rows: the smallest box the layout
            // could accept), then the layout's own sizes decide
            const double per_row = (double)T.nnz / n;
            if (!tt.user_box && per_row >= TILE_DENSE_ROW) {
                tt.tx = TILE_DENSE_BOX[0];
                tt.ty = TILE_DENSE_BOX[1];
                tt.tz = TILE_DENSE_BOX[2];
            }
            for (;;) {
                const int rows = tt.tx * tt.ty * tt.tz;
                if (TileSmem::of<double, double, double>(rows, rows / 4, (int)(rows * per_row)).total <=
                        TILE_SMEM_MAX ||
                    !shrink())
                    break;
            }
            for (int attempt = 0; attempt < 6; attempt++) {
                TP = TileHostPlan();
                Trace tr_lay("      box layout", s);
                if (!tile_layout(n, rp.data(), ci.data(), upper, src_of, G, tt, TP, /*entries=*/false)) break;
                tr_lay.stop();
                if (TileSmem::of<double, double, double>(TP.max_rows, TP.max_halo, TP.max_entries).total <=
                    TILE_SMEM_MAX) {
                    T.tiled = true;
                    break;
                }
                if (!shrink()) break;
            }
        }
    }
    if (T.tiled) {
        Trace tr_bu("      box uploads", s);
        T.ntiles = TP.ntiles;
        T.tile_elems = TP.max_rows + TP.max_halo;
        T.t_max_rows = TP.max_rows;
        T.t_max_halo = TP.max_halo;
        T.t_max_entries = TP.max_entries;
        T.perm.alloc(n); T.perm.upload(TP.perm.data(), n, s);
        T.prp.alloc(n + 1); T.prp.upload(TP.prp.data(), n + 1, s);
        T.t_pos.alloc(TP.tile_pos.size()); T.t_pos.upload(TP.tile_pos.data(), TP.tile_pos.size(), s);
        T.t_lvl.alloc(TP.tile_lvl.size()); T.t_lvl.upload(TP.tile_lvl.data(), TP.tile_lvl.size(), s);
        T.t_lptr.alloc(TP.lvl_ptr.size()); T.t_lptr.upload(TP.lvl_ptr.data(), TP.lvl_ptr.size(), s);
        T.t_hptr.alloc(TP.halo_ptr.size()); T.t_hptr.upload(TP.halo_ptr.data(), TP.halo_ptr.size(), s);
        T.t_hrow.alloc(std::max<size_t>(TP.halo_row.size(), 1));
        if (!TP.halo_row.empty()) T.t_hrow.upload(TP.halo_row.data(), TP.halo_row.size(), s);
        // the entries (slot and value source of each) written on the device
        // from the rows' boxes and positions
        T.pci.alloc(m);
        T.src.alloc(m);
        if (T.nnz) {
            DBuf<int> d_tile_of, d_pos_of;
            d_tile_of.alloc(n); d_tile_of.upload(TP.tile_of.data(), n, s);
            d_pos_of.alloc(n); d_pos_of.upload(TP.pos_of.data(), n, s);
            auto kern = upper ? k_tile_entries<true> : k_tile_entries<false>;
            kern<<<g, 256, 0, s>>>(n, T.perm.p, T.prp.p, T.rp_nat.p, T.ci_nat.p, T.src_nat.p, d_tile_of.p, d_pos_of.p,
                                   T.t_pos.p, T.t_hptr.p, T.t_hrow.p, T.pci.p, T.src.p);
            check_launch();
            XS_CUDA(cudaStreamSynchronize(s));  // before the temporaries are freed
        }
        tr_bu.stop();
        if (need_levels) {
            level_analysis();
            T.nlevels = P.nlevels;
            T.lvperm.alloc(n); T.lvperm.upload(P.perm.data(), n, s);
        }
        T.lstart.free();
        XS_CUDA(cudaStreamSynchronize(s));  // the host plans go out of scope
    } else if (!T.chunked) {
        level_analysis();
        T.nlevels = P.nlevels;
        // padded: the staged single-CTA solve copies 16-byte aligned ranges
        T.perm.alloc(n, 4); T.perm.upload(P.perm.data(), n, s);
        T.prp.alloc(n + 1, 4); T.prp.upload(P.prp.data(), n + 1, s);
        T.pci.alloc(m, 4);
        T.src.alloc(m);
        k_pos_entries<<<g, 256, 0, s>>>(n, upper, T.perm.p, T.prp.p, T.rp_nat.p, T.ci_nat.p, T.src_nat.p, T.pci.p,
                                        T.src.p);
        check_launch();
        T.lstart.alloc(P.nlevels + 1, 4); T.lstart.upload(P.lstart.data(), P.nlevels + 1, s);
        T.max_level_rows = 0;
        for (int l = 0; l < P.nlevels; l++) T.max_level_rows = std::max(T.max_level_rows, P.lstart[l + 1] - P.lstart[l]);
        // level batches of the staged single-CTA solve (systems it serves only)
        T.nlub = 0;
        T.lub.free();
        if ((size_t)n * sizeof(double) <= LU_BLOCK_SMEM_MAX) {
            const TrsvTuning &tu = trsv_tuning();
            int brows = tu.lub_rows, bents = tu.lub_entries;
            if (tu.lub_auto) {
                // two buffers in what the FP64 solution vector leaves
                const size_t ysb = ((size_t)n * sizeof(double) + 15) & ~(size_t)15;
                const double epr = std::max(1.0, (double)T.nnz / std::max(n, 1));
                brows = (int)((double)((LU_SMEM_LIMIT - ysb) / 2) / (16.0 + 12.0 * epr));
                for (; brows > 32; brows -= 16) {
                    bents = (int)std::ceil(brows * epr) + 32;
                    if (ysb + 2 * LuBatchSmem<double, double>::of(brows, bents).bytes <= LU_SMEM_LIMIT) break;
                }
                brows = std::max(brows, 32);
            }
            T.lub_rows = brows;
            T.lub_entries = bents;
            std::vector<int> b;
            int l = 0;
            while (l < P.nlevels) {
                const int p0 = P.lstart[l];
                int l1 = l, rows = 0;
                long ents = 0;
                while (l1 < P.nlevels) {
                    const int r = P.lstart[l1 + 1] - P.lstart[l1];
                    const long e = (long)P.prp[P.lstart[l1 + 1]] - P.prp[P.lstart[l1]];
                    if (rows + r > brows || ents + e > bents) break;
                    rows += r;
                    ents += e;
                    l1++;
                }
                (void)p0;
                if (l1 == l) {  // one level larger than a batch: solved unstaged
                    b.push_back(-1 - l);
                    l++;
                } else {
                    b.push_back(l);
                    l = l1;
                }
            }
            b.push_back(P.nlevels);
            T.nlub = (int)b.size() - 1;
            T.lub.alloc(b.size());
            T.lub.upload(b.data(), b.size(), s);
        }
    } else {
        level_analysis();
        T.nlevels = P.nlevels;
        TriChunkPlan C;
        tri_analyse_chunked(n, rp.data(), ci.data(), upper, src_of, chr, C);
        T.nchunks = C.nchunks;
        T.ch = C.ch;
        T.perm.alloc(n); T.perm.upload(C.perm.data(), n, s);
        T.prp.alloc(n + 1); T.prp.upload(C.prp.data(), n + 1, s);
        T.pci.alloc(m); if (T.nnz) T.pci.upload(C.pci_enc.data(), T.nnz, s);
        T.src.alloc(m); if (T.nnz) T.src.upload(C.src.data(), T.nnz, s);
        T.lvl_off.alloc(C.lvl_off.size()); T.lvl_off.upload(C.lvl_off.data(), C.lvl_off.size(), s);
        T.lvl_ptr.alloc(C.lvl_ptr.size()); T.lvl_ptr.upload(C.lvl_ptr.data(), C.lvl_ptr.size(), s);
    }
    tr_up.stop();
    Trace tr_ell("    ELL copy", s);
    // ELL copy when the rows are nearly uniform (padding at most 2x)
    int w = 0;
    for (int i = 0; i < n; i++) w = std::max(w, rp[i + 1] - rp[i]);
    T.ell_w = 0;
    const std::vector<int> offs = w > 0 ? dia_offsets(n, rp.data(), ci.data()) : std::vector<int>();
    T.ell_dia = !offs.empty();
    if (T.ell_dia) {
        // diagonal slots, built on the device from the natural CSR
        const int D = (int)offs.size();
        const long ld = ell_ld(n);
        T.ell_w = D;
        T.ell16 = false;
        T.doff.alloc(D); T.doff.upload(offs.data(), D, s);
        T.esrc.alloc((size_t)D * ld);
        const int g = geom().sms * 4;
        if (D <= 8) {
            T.emask8.alloc(ld);
            k_tri_dia_build<uint8_t><<<g, 256, 0, s>>>(n, D, ld, T.rp_nat.p, T.ci_nat.p, T.src_nat.p, T.doff.p,
                                                       T.emask8.p, T.esrc.p);
        } else {
            T.emask32.alloc(ld);
            k_tri_dia_build<uint32_t><<<g, 256, 0, s>>>(n, D, ld, T.rp_nat.p, T.ci_nat.p, T.src_nat.p, T.doff.p,
                                                        T.emask32.p, T.esrc.p);
        }
        check_launch();
    } else if (w > 0 && w <= 64 && (long)w * n <= 2 * std::max<long>(T.nnz, 1)) {
        // layout of the operator's ELL copy, built on the device from the
        // natural CSR just uploaded
        const long maxoff = max_col_offset(n, rp.data(), ci.data());
        T.ell_w = w;
        T.ell16 = format_tuning().ell_index16 && maxoff <= 32767;
        const long ld = ell_ld(n);
        const size_t m = (size_t)w * ld;
        T.esrc.alloc(m);
        const int g = geom().sms * 4;
        if (T.ell16) {
            T.eco.alloc(m);
            T.eci.free();
            k_tri_ell_build<short><<<g, 256, 0, s>>>(n, w, ld, T.rp_nat.p, T.ci_nat.p, T.src_nat.p, T.eco.p, T.esrc.p);
        } else {
            T.eci.alloc(m);
            T.eco.free();
            k_tri_ell_build<int><<<g, 256, 0, s>>>(n, w, ld, T.rp_nat.p, T.ci_nat.p, T.src_nat.p, T.eci.p, T.esrc.p);
        }
        check_launch();
    }
    T.ticket.alloc(1);
    XS_CUDA(cudaStreamSynchronize(s));
}

// gather the ELL copy's values (FP64 always, reduced precisions on request)
// red: reduced precisions built with need32 (bit 0 FP32, bit 1 BF16, bit 2 FP16)
inline void load_tri_ell(TriDev &T, const double *vals, bool need32, cudaStream_t s, unsigned red = 7u)
{
    if (T.ell_w == 0) return;
    const long m = (long)T.ell_w * ell_ld(T.n);
    const int g = geom().sms * 4;
    if (T.ev64.n != (size_t)m) T.ev64.alloc(m);
    k_gather_convert_pad<double><<<g, 256, 0, s>>>(m, T.esrc.p, vals, T.ev64.p);
    auto one = [&](auto &buf, bool want) {
        using FT = std::remove_pointer_t<decltype(buf.p)>;
        if (!want) {
            buf.free();
            return;
        }
        if (buf.n != (size_t)m) buf.alloc(m);
        k_gather_convert_pad<FT><<<g, 256, 0, s>>>(m, T.esrc.p, vals, buf.p);
    };
    one(T.ev32, need32 && (red & 1u));
    one(T.evbf, need32 && (red & 2u));
    one(T.evh, need32 && (red & 4u));
    check_launch();
}

// ---------------------------------------------------------------- single-CTA LU solve
// For small systems the cross-SM hand-off of the sync-free solve (a store
// becoming visible in L2, then a poll) costs more per dependency level than
// the level's work.  One CTA walks the levels instead: z = U'^-1 (dinv *
// L^-1 x) with the whole solution vector in shared memory, a __syncthreads
// between levels, the L result overwritten in place by the U result (a row's
// own y value is read only by that row; its dependencies hold final z values
// from earlier levels).  Row arithmetic and entry order are those of
// trsv_row, so results are bitwise identical to the sync-free solve.  The
// sync-free solve buffers are not touched (they stay armed).
constexpr int LU_BLOCK_THREADS = 1024;

// One thread's row of a level, loaded ahead: the row, its entry range, the
// first LU_PF entries and the row's scalar input (x[row] for L, dinv for U).
constexpr int LU_PF = 4;
template <typename VT, typename FT>
struct LuRow {
    int row, k0, len;
    int c[LU_PF];
    FT v[LU_PF];
    VT in;
};

template <typename VT, typename FT, typename DT, bool UPPER>
__device__ __forceinline__ void lu_row_load(const TrsvArgs<FT> &P, int p, const VT *__restrict__ x,
                                            const DT *__restrict__ dinv, LuRow<VT, FT> &r)
{
    r.row = __ldg(P.perm + p);
    r.k0 = __ldg(P.prp + p);
    r.len = __ldg(P.prp + p + 1) - r.k0;
#pragma unroll
    for (int j = 0; j < LU_PF; j++) {
        if (j < r.len) {
            r.c[j] = __ldg(P.pci + r.k0 + j);
            r.v[j] = P.pv[r.k0 + j];
        }
    }
    if (UPPER) r.in = (VT)__ldg(dinv + p);
    else r.in = x[r.row];
}

template <typename VT, typename FT, bool UPPER>
__device__ __forceinline__ void lu_row_solve(const TrsvArgs<FT> &P, const LuRow<VT, FT> &r, VT *ys)
{
    VT acc = UPPER ? ys[r.row] * r.in : r.in;
#pragma unroll
    for (int j = 0; j < LU_PF; j++)
        if (j < r.len) acc = msub(acc, ys[r.c[j]], (VT)FVal<FT>::cvt(r.v[j]));
    for (int k = r.k0 + LU_PF; k < r.k0 + r.len; k++) acc = msub(acc, ys[__ldg(P.pci + k)], (VT)FVal<FT>::ld(P.pv, k));
    ys[r.row] = acc;
}

// walk the levels of one triangle; the row a thread takes in level l+1 is
// loaded before the barrier that ends level l, so its global loads overlap
// the barrier instead of starting after it
template <typename VT, typename FT, typename DT, bool UPPER>
__device__ __forceinline__ void lu_block_phase(const TrsvArgs<FT> &P, const int *__restrict__ ls, int nl,
                                               const VT *__restrict__ x, const DT *__restrict__ dinv, VT *ys)
{
    LuRow<VT, FT> nxt;
    bool have = nl > 0 && __ldg(ls) + (int)threadIdx.x < __ldg(ls + 1);
    if (have) lu_row_load<VT, FT, DT, UPPER>(P, __ldg(ls) + threadIdx.x, x, dinv, nxt);
    for (int l = 0; l < nl; l++) {
        const int p0 = __ldg(ls + l), p1 = __ldg(ls + l + 1);
        if (have) {
            const LuRow<VT, FT> cur = nxt;
            lu_row_solve<VT, FT, UPPER>(P, cur, ys);
        }
        // rows beyond the first blockDim.x of a wide level, without look-ahead
        for (int p = p0 + (int)threadIdx.x + (int)blockDim.x; p < p1; p += blockDim.x) {
            LuRow<VT, FT> r;
            lu_row_load<VT, FT, DT, UPPER>(P, p, x, dinv, r);
            lu_row_solve<VT, FT, UPPER>(P, r, ys);
        }
        have = false;
        if (l + 1 < nl) {
            const int q = p1 + (int)threadIdx.x;
            if (q < __ldg(ls + l + 2)) {
                lu_row_load<VT, FT, DT, UPPER>(P, q, x, dinv, nxt);
                have = true;
            }
        }
        __syncthreads();
    }
}

template <typename VT, typename FT, typename DT>
__global__ void __launch_bounds__(LU_BLOCK_THREADS) k_lu_block(TrsvArgs<FT> L, const int *__restrict__ lstart, int nlL,
                                                                TrsvArgs<FT> U, const int *__restrict__ ustart, int nlU,
                                                                const DT *__restrict__ dinv, const VT *__restrict__ x,
                                                                VT *__restrict__ z, const int *done_flag)
{
    extern __shared__ __align__(16) unsigned char lu_smem[];
    VT *ys = (VT *)lu_smem;
    if (done_flag && *done_flag) return;
    lu_block_phase<VT, FT, DT, false>(L, lstart, nlL, x, dinv, ys);
    lu_block_phase<VT, FT, DT, true>(U, ustart, nlU, x, dinv, ys);
    for (int i = threadIdx.x; i < L.n; i += blockDim.x) z[i] = ys[i];
}

// ---- staged single-CTA solve: the level batches of each triangle are
// copied into shared memory by asynchronous copies one batch ahead, so a
// level reads only shared memory (the row data of the plain form above
// arrives from global memory one level ahead, a memory latency per level).
// The solution vector starts as x (its own slot is a row's right-hand side
// in the L phase) and is overwritten level by level; row arithmetic and
// entry order are those of trsv_row, so results are bitwise the same.

__device__ __forceinline__ void named_sync(int id, int count)
{
    asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(count) : "memory");
}
__device__ __forceinline__ void named_arrive(int id, int count)
{
    asm volatile("bar.arrive %0, %1;" ::"r"(id), "r"(count) : "memory");
}

// first level of batch b of a triangle's batch list
__device__ __forceinline__ int lub_first_level(const int *__restrict__ lub, int b)
{
    const int v = __ldg(lub + b);
    return v < 0 ? -1 - v : v;
}

// copy batch b (level starts, rows, entry offsets, columns, values, U's
// dinv) into buf with 16-byte copies, threads tid of T: each array range is
// rounded out to 16-byte boundaries (the arrays are allocated with at least
// 16 bytes of padding) and the element shift of its start goes into the
// header; a level too large to stage only gets its code
template <typename FT, typename DT, bool UPPER>
__device__ __forceinline__ void lu_stage_batch(const TrsvArgs<FT> &P, const int *__restrict__ ls,
                                               const int *__restrict__ lub, int b, const DT *__restrict__ dinv,
                                               unsigned char *buf, const LuBatchSmem<FT, DT> &B, int tid, int T)
{
    int *hdr = (int *)(buf + B.hdr);
    const int code = __ldg(lub + b);
    if (code < 0) {
        if (tid == 0) hdr[0] = code;
        return;
    }
    const int l0 = code, l1 = lub_first_level(lub, b + 1);
    const int pa = __ldg(ls + l0), pb = __ldg(ls + l1);
    const int ea = __ldg(P.prp + pa), eb = __ldg(P.prp + pb);
    if (tid == 0) {
        hdr[0] = l0;
        hdr[1] = l1;
        hdr[2] = pa;
        hdr[3] = ea;
    }
    auto copy = [&](const void *base, long first, long count, int esz, size_t dst, int slot) {
        const uintptr_t a0 = (uintptr_t)base + (uintptr_t)(first * esz);
        const uintptr_t b0 = a0 & ~(uintptr_t)15;
        const uintptr_t b1 = (a0 + (uintptr_t)(count * esz) + 15) & ~(uintptr_t)15;
        if (tid == 0) hdr[4 + slot] = (int)((a0 - b0) / (uintptr_t)esz);
        const long chunks = (long)((b1 - b0) >> 4);
        for (long c = tid; c < chunks; c += T) cp_async16(buf + dst + 16 * c, (const void *)(b0 + 16 * c));
    };
    copy(ls, l0, l1 - l0 + 1, 4, B.lvl, 0);
    copy(P.perm, pa, pb - pa, 4, B.row, 1);
    copy(P.prp, pa, pb - pa + 1, 4, B.eptr, 2);
    copy(P.pci, ea, eb - ea, 4, B.pci, 3);
    copy(P.pv, ea, eb - ea, (int)sizeof(FT), B.pv, 4);
    if (UPPER) copy(dinv, pa, pb - pa, (int)sizeof(DT), B.in, 5);
}

// the levels of batch b by threads tid of T (a barrier of those T threads,
// id level_bar, after each level)
template <typename VT, typename FT, typename DT, bool UPPER>
__device__ __forceinline__ void lu_batch_levels(const TrsvArgs<FT> &P, const int *__restrict__ ls,
                                                const int *__restrict__ lub, int b, const DT *__restrict__ dinv,
                                                VT *ys, const unsigned char *buf, const LuBatchSmem<FT, DT> &B, int tid,
                                                int T, int level_bar)
{
    // the batch's header and level starts come from shared memory (the
    // copiers wrote them), so a level step touches shared memory only
    const int *hdr = (const int *)(buf + B.hdr);
    const int lb = hdr[0];
    if (lb >= 0) {
        const int l0 = lb, l1 = hdr[1], pa = hdr[2], ea = hdr[3];
        const int *s_lvl = (const int *)(buf + B.lvl) + hdr[4];
        const int *s_row = (const int *)(buf + B.row) + hdr[5];
        const int *s_eptr = (const int *)(buf + B.eptr) + hdr[6];
        const int *s_pci = (const int *)(buf + B.pci) + hdr[7];
        const FT *pv = (const FT *)(buf + B.pv) + hdr[8];
        const DT *s_in = (const DT *)(buf + B.in) + (UPPER ? hdr[9] : 0);
        for (int l = l0; l < l1; l++) {
            const int q0 = s_lvl[l - l0] - pa, q1 = s_lvl[l - l0 + 1] - pa;
            for (int i = q0 + tid; i < q1; i += T) {
                const int row = s_row[i];
                VT acc = UPPER ? (VT)(ys[row] * (VT)s_in[i]) : ys[row];
                const int k1 = s_eptr[i + 1] - ea;
                for (int k = s_eptr[i] - ea; k < k1; k++) acc = msub(acc, ys[s_pci[k]], (VT)FVal<FT>::cvt(pv[k]));
                ys[row] = acc;
            }
            named_sync(level_bar, T);
        }
    } else {  // one level too large to stage: its rows from global memory
        const int l = -1 - lb;
        for (int p = __ldg(ls + l) + tid; p < __ldg(ls + l + 1); p += T) {
            const int row = __ldg(P.perm + p);
            VT acc = UPPER ? (VT)(ys[row] * (VT)__ldg(dinv + p)) : ys[row];
            for (int k = __ldg(P.prp + p); k < __ldg(P.prp + p + 1); k++)
                acc = msub(acc, ys[__ldg(P.pci + k)], (VT)FVal<FT>::ld(P.pv, k));
            ys[row] = acc;
        }
        named_sync(level_bar, T);
    }
}

// Warp-specialised: the first cw warps walk the levels (a barrier of those
// warps only between levels), the other warps copy the batches, L's then
// U's, into nbuf buffers up to nbuf - 1 batches ahead; named barriers
// 1..nbuf ("batch in buffer k landed": the copiers arrive, the walkers wait)
// and nbuf+1..2*nbuf ("buffer k free": the walkers arrive, the copiers wait
// before reusing it) hand the buffers over; barrier 2*nbuf+1 is the walkers'.
template <typename VT, typename FT, typename DT>
__global__ void __launch_bounds__(LU_BLOCK_THREADS) k_lu_staged(TrsvArgs<FT> L, const int *__restrict__ lstart,
                                                                 const int *__restrict__ lubL, int nbL, TrsvArgs<FT> U,
                                                                 const int *__restrict__ ustart,
                                                                 const int *__restrict__ lubU, int nbU,
                                                                 const DT *__restrict__ dinv, const VT *__restrict__ x,
                                                                 VT *__restrict__ z, const int *done_flag, int cw,
                                                                 int brows, int bents, int nbuf)
{
    extern __shared__ __align__(16) unsigned char lus_smem[];
    if (done_flag && *done_flag) return;
    const LuBatchSmem<FT, DT> B = LuBatchSmem<FT, DT>::of(brows, bents);
    const size_t yb = ((size_t)L.n * sizeof(VT) + 15) & ~(size_t)15;
    VT *ys = (VT *)lus_smem;
    for (int i = threadIdx.x; i < L.n; i += blockDim.x) ys[i] = x[i];
    __syncthreads();
    const int all = blockDim.x, ct = cw * 32, nb = nbL + nbU;
    const int level_bar = 2 * nbuf + 1;
    if ((int)threadIdx.x >= ct) {  // copiers
        const int tid = threadIdx.x - ct, T = all - ct;
        for (int g = 0; g < nb; g++) {
            const int k = g % nbuf;
            unsigned char *buf = lus_smem + yb + (size_t)k * B.bytes;
            if (g >= nbuf) named_sync(1 + nbuf + k, all);  // the walkers are done with batch g - nbuf
            if (g < nbL) lu_stage_batch<FT, DT, false>(L, lstart, lubL, g, nullptr, buf, B, tid, T);
            else lu_stage_batch<FT, DT, true>(U, ustart, lubU, g - nbL, dinv, buf, B, tid, T);
            cp_async_commit();
            cp_async_wait<0>();
            named_arrive(1 + k, all);
        }
    } else {  // walkers
        for (int g = 0; g < nb; g++) {
            const int k = g % nbuf;
            const unsigned char *buf = lus_smem + yb + (size_t)k * B.bytes;
            named_sync(1 + k, all);  // batch g landed
            if (g < nbL)
                lu_batch_levels<VT, FT, DT, false>(L, lstart, lubL, g, nullptr, ys, buf, B, threadIdx.x, ct, level_bar);
            else
                lu_batch_levels<VT, FT, DT, true>(U, ustart, lubU, g - nbL, dinv, ys, buf, B, threadIdx.x, ct,
                                                  level_bar);
            if (g + nbuf < nb) named_arrive(1 + nbuf + k, all);  // buffer k free for batch g + nbuf
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < L.n; i += blockDim.x) z[i] = ys[i];
}

// whether the single-CTA solve serves this pair of plans for vectors of VT
template <typename VT>
inline bool lu_block_ok(const TriDev &L, const TriDev &U)
{
    const TrsvTuning &t = trsv_tuning();
    return !L.chunked && !U.chunked && L.n > 0 && L.n <= t.block_max_rows &&
           (size_t)L.n * sizeof(VT) <= LU_BLOCK_SMEM_MAX && L.lstart.p && U.lstart.p;
}

template <typename VT, typename FT, typename DT>
inline void launch_lu_block(const TriDev &L, const TriDev &U, const DT *dinv, const VT *x, VT *z, const int *done_flag,
                            cudaStream_t s)
{
    // the staged form when both triangles have level batches and the
    // solution vector plus two batches fit in shared memory
    const TrsvTuning &tu = trsv_tuning();
    const int brows = std::max(L.lub_rows, U.lub_rows), bents = std::max(L.lub_entries, U.lub_entries);
    const int nbuf = tu.lub_auto ? 2 : tu.lub_bufs;
    const size_t ssm = (((size_t)L.n * sizeof(VT) + 15) & ~(size_t)15) +
                       (size_t)nbuf * LuBatchSmem<FT, DT>::of(brows, bents).bytes;
    if (L.nlub > 0 && U.nlub > 0 && ssm <= LU_SMEM_LIMIT && trsv_tuning().lu_staged) {
        static size_t sattr = 0;
        if (ssm > sattr) {
            XS_CUDA(cudaFuncSetAttribute(k_lu_staged<VT, FT, DT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)ssm));
            sattr = ssm;
        }
        // 1024 threads: walker warps for the widest level's rows (at most 16),
        // the rest copy
        const int thr = LU_BLOCK_THREADS;
        const int wide = std::max(L.max_level_rows, U.max_level_rows);
        int cw = std::max(1, std::min(16, (wide + 31) / 32));
        if (trsv_tuning().lu_staged_threads > 0) cw = std::min(16, trsv_tuning().lu_staged_threads / 32);
        k_lu_staged<VT, FT, DT><<<1, thr, ssm, s>>>(L.args<FT>(), L.lstart.p, L.lub.p, L.nlub,
                                                                  U.args<FT>(), U.lstart.p, U.lub.p, U.nlub, dinv, x,
                                                                  z, done_flag, cw, brows, bents, nbuf);
        return;
    }
    static size_t attr = 0;  // largest dynamic shared memory enabled so far for this instantiation
    const size_t smem = (size_t)L.n * sizeof(VT);
    if (smem > attr) {
        XS_CUDA(cudaFuncSetAttribute(k_lu_block<VT, FT, DT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        attr = smem;
    }
    k_lu_block<VT, FT, DT><<<1, LU_BLOCK_THREADS, smem, s>>>(L.args<FT>(), L.lstart.p, L.nlevels, U.args<FT>(),
                                                              U.lstart.p, U.nlevels, dinv, x, z, done_flag);
}

template <typename VT, typename FT, typename DT, bool UPPER>
inline void launch_trsv(const TriDev &T, const DT *dinv, const VT *rhs, VT *self, VT *out_user, VT *reset_other,
                        const int *done_flag, int *err, cudaStream_t s)
{
    const int bo = trsv_tuning().backoff_ns;
    if (T.tiled) {
        static size_t attr = 0;  // largest dynamic shared memory enabled so far for this instantiation
        const size_t smem = TileSmem::of<VT, FT, DT>(T.t_max_rows, T.t_max_halo, T.t_max_entries).total;
        if (smem > attr) {
            XS_CUDA(cudaFuncSetAttribute(k_trsv_tiles<VT, FT, DT, UPPER>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem));
            attr = smem;
        }
        // resident boxes per SM: the tuning's count, fewer when shared memory limits it
        const int fit = std::max(1, (int)((220u * 1024u) / std::max<size_t>(smem + 1024, 1)));
        const int bps = std::max(1, std::min(tile_tuning().blocks_per_sm, fit));
        const int g = std::min(T.ntiles, geom().sms * bps);
        k_trsv_tiles<VT, FT, DT, UPPER><<<g, TILE_THREADS, smem, s>>>(T.targs<FT>(), dinv, rhs, self, out_user,
                                                                     reset_other, done_flag, err, T.ticket.p, bo);
    } else if (T.chunked) {
        static size_t attr = 0;  // largest dynamic shared memory enabled so far for this instantiation
        const size_t smem = (size_t)T.ch * sizeof(VT);
        if (smem > attr) {
            XS_CUDA(cudaFuncSetAttribute(k_trsv_chunked<VT, FT, DT, UPPER>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem));
            attr = smem;
        }
        const int g = std::min(T.nchunks, geom().sms);
        k_trsv_chunked<VT, FT, DT, UPPER><<<g, CH_THREADS, smem, s>>>(T.cargs<FT>(), dinv, rhs, self, out_user,
                                                                     reset_other, done_flag, err, T.ticket.p, bo);
    } else {
        k_trsv_syncfree<VT, FT, DT, UPPER><<<trsv_grid(T.n), TRSV_THREADS, 0, s>>>(
            T.args<FT>(), dinv, rhs, self, out_user, reset_other, done_flag, err, T.ticket.p, bo);
    }
}

}  // namespace xs
