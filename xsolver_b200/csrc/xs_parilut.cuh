// ParILUT on the GPU (replaces parilt::parilut_clean, hip/Precond/
// parilut.cpp:621-1206, with its binned warp SpGEMM candidate generation
// par_ilut_hip/My_computeSpmm.h:98-159, LU/L/U sweeps :392-560, threshold
// removal :283-380 and bucket k-th select par_ilut_hip/select_kth.h:501).
//
// Per sweep s (rate = (fill-1)/sweeps*(s+1)+1, :692):
//   1. candidates = pattern(A) u pattern(L*U): one warp per row marks A's
//      row and the U rows selected by L's row in a shared-memory bitmap over
//      the row's column window and reads the set bits back in order (rows
//      whose window exceeds the bitmap gather, bitonic-sort and de-duplicate
//      instead); a symbolic pass counts, a second pass writes.
//   2. values: entries already in L/U keep their value; a new entry gets
//      r_ij/u_jj (lower) or r_ij (upper), r = A - L*U accumulated as
//      c = -a_ij; c += l_ik u_kj (k ascending); r = -c.
//   3. split into L (CSR, unit diagonal last) and U (CSR, diagonal first);
//      both factors stay row-major throughout, so no transposes are formed.
//   4. one synchronous sweep over every L and U entry (fixed point of the
//      ILU equations on the current pattern), row-wise: a warp per row
//      subtracts l_ik * u_kj walking the U rows k of its L row.
//   5. if the candidate count exceeds round(rate*nnz(A)): per factor keep
//      (int)(rate*nnz0) entries — threshold = k-th smallest |v| by an 8-pass
//      radix select on the IEEE bit patterns — plus the optional drop
//      tolerance; diagonals are always kept.
//   6. synchronous L sweep, then U sweep with the new L.
// All sweeps are synchronous (new values from a snapshot), so the result is
// deterministic and equal to the CPU restatement in oracle/xs_oracle.cpp.
// Differences from the reference (which updates in place asynchronously):
// existing entries keep their values instead of being reset to a_ij each
// sweep, and the initial L is scaled by 1/a_jj — the published ParILUT
// algorithm; the reference's reset only converges with asynchronous sweeps.
#pragma once
#include <climits>
#include <numeric>
#include "xs_trsv.cuh"
#include "xs_spmv.cuh"

namespace xs {

struct DCsr {
    int n = 0;
    long nnz = 0;
    DBuf<int> rp, ci;
    DBuf<double> v;
};

struct ParilutResult {
    int n = 0;
    long nnzL = 0, nnzU = 0;
    DBuf<int> lrp, lci, urp, uci;  // strict triangles (seqilu0 layout)
    DBuf<double> lv, uv, dinv;
    DBuf<long> diag_ident;
    HostArray<int> hlrp, hlci, hurp, huci;  // the pattern on the host (box analysis)
};

constexpr int PLT_CAP = 2048;  // candidate columns gathered per row (with duplicates)
constexpr int PLT_WARPS = 4;

// ---------------------------------------------------------------- helpers
// device binary search: position of column j in row [a, b) of ci, or -1
__device__ __forceinline__ int find_pos(const int *ci, int a, int b, int j)
{
    int l = a, r = b;
    while (l < r) {
        const int m = l + ((r - l) >> 1);
        if (ci[m] < j) l = m + 1;
        else r = m;
    }
    return (l < b && ci[l] == j) ? l : -1;
}

// ---------------------------------------------------------------- candidates
// mode 0: count unique candidate columns per row into cnt[i]
// mode 1: write them (sorted) into dci[drp[i] ...]
// Row i's candidates lie in [lo, hi]: the smallest/largest column of A's row
// and the first/last column of the U rows k of L row i (U rows are sorted).  When the window fits PLT_BM_WORDS*32 columns the
// warp marks a bitmap with shared atomics and reads the set bits back word by
// word (ascending, a warp prefix sum gives each word's output offset); wider
// windows gather every column (duplicates included, at most PLT_CAP) and
// bitonic-sort them.
constexpr int PLT_BM_WORDS = PLT_CAP;  // bitmap words per warp (same buffer)

static __global__ void __launch_bounds__(32 * PLT_WARPS) k_candidates(int n, const int *__restrict__ arp,
                                                               const int *__restrict__ aci, const int *__restrict__ lrp,
                                                               const int *__restrict__ lci, const int *__restrict__ urp,
                                                               const int *__restrict__ uci, int mode, int *cnt,
                                                               const int *__restrict__ drp, int *dci, int *err)
{
    __shared__ int sbuf[PLT_WARPS][PLT_CAP];
    __shared__ int scount[PLT_WARPS];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int *buf = sbuf[w];
    unsigned *bm = reinterpret_cast<unsigned *>(buf);
    for (int i = blockIdx.x * PLT_WARPS + w; i < n; i += gridDim.x * PLT_WARPS) {
        const int a0 = arp[i], a1 = arp[i + 1], l0 = lrp[i], l1 = lrp[i + 1];
        int lo = INT_MAX, hi = INT_MIN;
        for (int q = a0 + lane; q < a1; q += 32) {
            lo = min(lo, aci[q]);
            hi = max(hi, aci[q]);
        }
        for (int q = l0 + lane; q < l1; q += 32) {
            const int k = lci[q];
            const int e0 = urp[k], e1 = urp[k + 1];
            if (e1 > e0) {
                lo = min(lo, uci[e0]);
                hi = max(hi, uci[e1 - 1]);
            }
        }
        for (int o = 16; o > 0; o >>= 1) {
            lo = min(lo, __shfl_xor_sync(0xffffffffu, lo, o));
            hi = max(hi, __shfl_xor_sync(0xffffffffu, hi, o));
        }
        const long words = hi >= lo ? (((long)hi - lo) >> 5) + 1 : 0;
        if (words <= PLT_BM_WORDS) {
            const int nw = (int)words;
            for (int q = lane; q < nw; q += 32) bm[q] = 0u;
            __syncwarp();
            const unsigned span = (unsigned)nw << 5;  // every column lies in [lo, hi]; the test only bounds the store
            for (int q = a0 + lane; q < a1; q += 32) {
                const unsigned d = (unsigned)(aci[q] - lo);
                if (d < span) atomicOr(bm + (d >> 5), 1u << (d & 31));
            }
            // U row ranges of 32 L entries at a time, one per lane, by shuffle
            for (int qb = l0; qb < l1; qb += 32) {
                int mb = 0, me = 0;
                if (qb + lane < l1) {
                    const int k = lci[qb + lane];
                    mb = urp[k];
                    me = urp[k + 1];
                }
                const int cnt = min(32, l1 - qb);
                for (int c = 0; c < cnt; c++) {
                    const int t0 = __shfl_sync(0xffffffffu, mb, c), t1 = __shfl_sync(0xffffffffu, me, c);
                    for (int t = t0 + lane; t < t1; t += 32) {
                        const unsigned d = (unsigned)(uci[t] - lo);
                        if (d < span) atomicOr(bm + (d >> 5), 1u << (d & 31));
                    }
                }
            }
            __syncwarp();
            int run = 0;
            for (int base = 0; base < nw; base += 32) {
                const int q = base + lane;
                unsigned wv = q < nw ? bm[q] : 0u;
                const int c = __popc(wv);
                int incl = c;
                for (int o = 1; o < 32; o <<= 1) {
                    const int y = __shfl_up_sync(0xffffffffu, incl, o);
                    if (lane >= o) incl += y;
                }
                if (mode == 1 && wv) {
                    int p = drp[i] + run + incl - c;
                    const int colbase = lo + (q << 5);
                    while (wv) {
                        dci[p++] = colbase + __ffs(wv) - 1;
                        wv &= wv - 1;
                    }
                }
                run += __shfl_sync(0xffffffffu, incl, 31);
            }
            if (mode == 0 && lane == 0) cnt[i] = run;
            __syncwarp();
            continue;
        }
        // total with duplicates (A's row counted once, by lane 0)
        int tot = lane == 0 ? a1 - a0 : 0;
        for (int q = l0 + lane; q < l1; q += 32) {
            const int k = lci[q];
            tot += urp[k + 1] - urp[k];
        }
        for (int o = 16; o > 0; o >>= 1) tot += __shfl_xor_sync(0xffffffffu, tot, o);
        if (tot > PLT_CAP) {
            if (lane == 0) {
                atomicOr(err, DEV_CAPACITY);
                if (mode == 0) cnt[i] = 0;
            }
            continue;
        }
        if (lane == 0) scount[w] = 0;
        __syncwarp();
        for (int q = a0 + lane; q < a1; q += 32) buf[atomicAdd(&scount[w], 1)] = aci[q];
        for (int q = l0; q < l1; q++) {
            const int k = lci[q];
            for (int t = urp[k] + lane; t < urp[k + 1]; t += 32) buf[atomicAdd(&scount[w], 1)] = uci[t];
        }
        __syncwarp();
        tot = scount[w];  // exactly the entries gathered
        int N = 1;
        while (N < tot) N <<= 1;
        for (int q = tot + lane; q < N; q += 32) buf[q] = INT_MAX;
        __syncwarp();
        for (int k = 2; k <= N; k <<= 1) {
            for (int j = k >> 1; j > 0; j >>= 1) {
                for (int q = lane; q < N; q += 32) {
                    const int p = q ^ j;
                    if (p > q) {
                        const int a = buf[q], b = buf[p];
                        const bool up = (q & k) == 0;
                        if ((a > b) == up) {
                            buf[q] = b;
                            buf[p] = a;
                        }
                    }
                }
                __syncwarp();
            }
        }
        // unique
        int run = 0;
        for (int base = 0; base < tot; base += 32) {
            const int q = base + lane;
            bool first = false;
            int val = 0;
            if (q < tot) {
                val = buf[q];
                first = (q == 0) || (buf[q - 1] != val);
            }
            const unsigned m = __ballot_sync(0xffffffffu, first);
            if (mode == 1 && first) dci[drp[i] + run + __popc(m & ((1u << lane) - 1))] = val;
            run += __popc(m);
        }
        if (mode == 0 && lane == 0) cnt[i] = run;
        __syncwarp();
    }
}

// candidate values (warp per row, lanes over the row's entries)
// value of candidate (i, j): an entry already in L or U keeps its value, a
// new one gets r_ij (/u_jj below the diagonal), r = A - L*U accumulated as
// c = -a_ij; c += l_ik u_kj for k of L row i (increasing) with (k, j) in U
// (the products of the merge of L row i with U column j, in its order)
__device__ __forceinline__ double cand_value(int i, int j, const int *arp, const int *aci, const double *av,
                                            const int *lrp, const int *lci, const double *lv, const int *urp,
                                            const int *uci, const double *uv, const double *udiag)
{
    int pos = -1;
    if (j < i) pos = find_pos(lci, lrp[i], lrp[i + 1], j);
    if (pos >= 0) return lv[pos];
    const int pu = (j >= i) ? find_pos(uci, urp[i], urp[i + 1], j) : -1;
    if (pu >= 0) return uv[pu];
    const int pa = find_pos(aci, arp[i], arp[i + 1], j);
    double c = -(pa >= 0 ? av[pa] : 0.0);
    for (int q = lrp[i]; q < lrp[i + 1]; q++) {
        const int k = lci[q];
        const int pk = find_pos(uci, urp[k], urp[k + 1], j);
        if (pk >= 0) c += lv[q] * uv[pk];
    }
    const double r = -c;
    return (j < i) ? r / udiag[j] : r;
}

// Candidate values, one warp per row i.  Existing entries copy their value;
// for the new ones the row's accumulators c_j = -a_ij are staged in shared
// memory and every k of L row i (increasing, the stored unit diagonal
// included) adds l_ik u_kj for each u_kj of U row k whose column is a new
// candidate of row i — the products and order of the per-entry merge, with
// contiguous reads of U rows.  Rows with more than PLT_CAND_CAP candidates
// use the per-entry merge.
constexpr int PLT_CAND_CAP = 512;
constexpr int PLT_CV_WARPS = 4;

static __global__ void __launch_bounds__(32 * PLT_CV_WARPS) k_candidate_values(
    int n, const int *__restrict__ arp, const int *__restrict__ aci, const double *__restrict__ av,
    const int *__restrict__ lrp, const int *__restrict__ lci, const double *__restrict__ lv,
    const int *__restrict__ urp, const int *__restrict__ uci, const double *__restrict__ uv,
    const double *__restrict__ udiag, const int *__restrict__ drp, const int *__restrict__ dci,
    double *__restrict__ dv)
{
    __shared__ int s_col[PLT_CV_WARPS][PLT_CAND_CAP];
    __shared__ double s_c[PLT_CV_WARPS][PLT_CAND_CAP];
    __shared__ unsigned char s_new[PLT_CV_WARPS][PLT_CAND_CAP];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int *col = s_col[w];
    double *cc = s_c[w];
    unsigned char *isnew = s_new[w];
    for (int i = blockIdx.x * PLT_CV_WARPS + w; i < n; i += gridDim.x * PLT_CV_WARPS) {
        const int d0 = drp[i], m = drp[i + 1] - d0;
        if (m > PLT_CAND_CAP) {
            for (int q = lane; q < m; q += 32)
                dv[d0 + q] = cand_value(i, dci[d0 + q], arp, aci, av, lrp, lci, lv, urp, uci, uv, udiag);
            continue;
        }
        bool any_new = false;
        for (int q = lane; q < m; q += 32) {
            const int j = dci[d0 + q];
            col[q] = j;
            int pos = -1;
            if (j < i) pos = find_pos(lci, lrp[i], lrp[i + 1], j);
            if (pos >= 0) {
                dv[d0 + q] = lv[pos];
                isnew[q] = 0;
                continue;
            }
            const int pu = (j >= i) ? find_pos(uci, urp[i], urp[i + 1], j) : -1;
            if (pu >= 0) {
                dv[d0 + q] = uv[pu];
                isnew[q] = 0;
                continue;
            }
            const int pa = find_pos(aci, arp[i], arp[i + 1], j);
            cc[q] = -(pa >= 0 ? av[pa] : 0.0);
            isnew[q] = 1;
            any_new = true;
        }
        if (!__any_sync(0xffffffffu, any_new)) continue;
        __syncwarp();
        const int l0 = lrp[i], l1 = lrp[i + 1];
        // L entries (value, U row range) 32 at a time, one per lane, by shuffle
        for (int kb = l0; kb < l1; kb += 32) {
            int mb = 0, me = 0;
            double ml = 0.0;
            if (kb + lane < l1) {
                const int k = lci[kb + lane];
                ml = lv[kb + lane];
                mb = urp[k];
                me = urp[k + 1];
            }
            const int cnt = min(32, l1 - kb);
            for (int cq = 0; cq < cnt; cq++) {
                const double lk = __shfl_sync(0xffffffffu, ml, cq);
                const int e0 = __shfl_sync(0xffffffffu, mb, cq), e1 = __shfl_sync(0xffffffffu, me, cq);
                for (int e = e0 + lane; e < e1; e += 32) {
                    const int j = uci[e];
                    int lo = 0, hi = m;
                    while (lo < hi) {
                        const int mid = (lo + hi) >> 1;
                        if (col[mid] < j) lo = mid + 1;
                        else hi = mid;
                    }
                    if (lo < m && col[lo] == j && isnew[lo]) cc[lo] += lk * uv[e];
                }
                __syncwarp();
            }
        }
        for (int q = lane; q < m; q += 32) {
            if (!isnew[q]) continue;
            const int j = col[q];
            const double r = -cc[q];
            dv[d0 + q] = (j < i) ? r / udiag[j] : r;
        }
        __syncwarp();
    }
}

static __global__ void k_udiag(int n, const int *__restrict__ urp, const double *__restrict__ uv, double *__restrict__ d)
{
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) d[j] = uv[urp[j]];
}

// split counts: lower entries + 1 (unit diagonal), upper entries (warp per row)
static __global__ void k_split_count(int n, const int *__restrict__ drp, const int *__restrict__ dci, int *lc, int *uc)
{
    const int lane = threadIdx.x & 31;
    const int wpb = blockDim.x >> 5;
    for (int i = blockIdx.x * wpb + (threadIdx.x >> 5); i < n; i += gridDim.x * wpb) {
        const int a = drp[i], b = drp[i + 1];
        int l = 0;
        for (int k = a + lane; k < b; k += 32) l += dci[k] < i;
        for (int o = 16; o > 0; o >>= 1) l += __shfl_xor_sync(0xffffffffu, l, o);
        if (lane == 0) {
            lc[i] = l + 1;
            uc[i] = (b - a) - l;
        }
    }
}
// rows are sorted, so the lower part is the prefix [a, a + nl) and the upper
// part the rest; L gets its unit diagonal last
static __global__ void k_split_fill(int n, const int *__restrict__ drp, const int *__restrict__ dci, const double *__restrict__ dv,
                             const int *__restrict__ lrp, int *lci, double *lv, const int *__restrict__ urp, int *uci,
                             double *uv)
{
    const int lane = threadIdx.x & 31;
    const int wpb = blockDim.x >> 5;
    for (int i = blockIdx.x * wpb + (threadIdx.x >> 5); i < n; i += gridDim.x * wpb) {
        const int a = drp[i], b = drp[i + 1];
        const int pl = lrp[i], nl = lrp[i + 1] - pl - 1, pu = urp[i];
        for (int k = a + lane; k < b; k += 32) {
            const int q = k - a;
            if (q < nl) { lci[pl + q] = dci[k]; lv[pl + q] = dv[k]; }
            else { uci[pu + q - nl] = dci[k]; uv[pu + q - nl] = dv[k]; }
        }
        if (lane == 0) {
            lci[pl + nl] = i;
            lv[pl + nl] = 1.0;
        }
    }
}

// ParILUT sweep value of entry (i, j) by a walk of L row i: a_ij minus
// l_ik * u_kj for every k of L row i (increasing) with k < min(i, j) and
// (k, j) in U, u_kj found by binary search in U row k (CSR, diagonal first).
// The same products in the same order as the merge of L row i with U column
// j in the reference's sweep (hip/Precond/parilut.cpp:392-441).
__device__ __forceinline__ double plt_sweep_value(const int *arp, const int *aci, const double *av, const int *lrp,
                                                  const int *lci, const double *lv, const int *urp, const int *uci,
                                                  const double *uv, int i, int j)
{
    const int pa = find_pos(aci, arp[i], arp[i + 1], j);
    double t = pa >= 0 ? av[pa] : 0.0;
    const int last = (i <= j) ? i : j;
    for (int q = lrp[i]; q < lrp[i + 1]; q++) {
        const int k = lci[q];
        if (k >= last) break;
        const int pu = find_pos(uci, urp[k], urp[k + 1], j);
        if (pu >= 0) t = t - lv[q] * uv[pu];
    }
    return t;
}

// Row-wise synchronous sweep, one warp per row i.  The row's pattern (L row
// i without its stored unit diagonal, then U row i) and its values
// t_ij = a_ij are staged in shared memory; then for every k of L row i in
// increasing order the lanes walk U row k (CSR) and, for each column j != k
// found in row i's pattern, subtract l_ik * u_kj.  That is the same set of
// products, subtracted in the same (increasing k) order, as the per-entry
// walk of plt_sweep_value, so the values are identical; but U rows are read
// contiguously and no lane walks a dependent index chain.  Results: L part
// t / u_jj into lnew, U part t into unew, both at the entry's CSR position.
// parts: 1 L only, 2 U only, 3 both.  Rows whose pattern exceeds
// PLT_ROW_CAP fall back to the per-entry walk.
constexpr int PLT_ROW_CAP = 256;
constexpr int PLT_SW_WARPS = 4;
// column -> pattern position of the row being swept: open addressing in
// shared memory, at most half full (PLT_HASH >= 2 * PLT_ROW_CAP), linear
// probing; a lookup costs one or two loads where a binary search over the
// sorted pattern costs eight.  One 32-bit word per slot: the column's low 24
// bits above the position (< PLT_ROW_CAP - 1 = 255, 8 bits), so a warp's table
// is 2 KB and more rows are in flight per SM.  Columns below 2^24 - 1 are
// told apart by their 24 bits alone; for larger systems a match of the low
// bits is confirmed against the staged column (plt_hash_find).
constexpr int PLT_HASH = 512;
constexpr unsigned PLT_HASH_EMPTY = ~0u;
__device__ __forceinline__ unsigned plt_hash_key(int j, int q) { return ((unsigned)j << 8) | (unsigned)q; }

__device__ __forceinline__ unsigned plt_hash_slot(int j)
{
    return ((unsigned)j * 2654435761u) >> (32 - 9);  // log2(PLT_HASH) = 9
}
static_assert(PLT_HASH == 512 && PLT_HASH >= 2 * PLT_ROW_CAP && PLT_ROW_CAP <= 256, "hash table size");
// position of column j in the staged pattern (col), or -1
__device__ __forceinline__ int plt_hash_find(const unsigned *ht, const int *col, bool wide, int j)
{
    const unsigned lo = (unsigned)j & 0xffffffu;
    for (unsigned sl = plt_hash_slot(j);; sl = (sl + 1) & (PLT_HASH - 1)) {
        const unsigned kv = ht[sl];
        if (kv == PLT_HASH_EMPTY) return -1;
        if ((kv >> 8) == lo) {
            const int q = (int)(kv & 0xffu);
            if (!wide || col[q] == j) return q;
        }
    }
}

static __global__ void __launch_bounds__(32 * PLT_SW_WARPS) k_plt_sweep_rows(
    int n, int parts, const int *__restrict__ arp, const int *__restrict__ aci, const double *__restrict__ av,
    const int *__restrict__ lrp, const int *__restrict__ lci, const double *__restrict__ lv_k,
    const double *__restrict__ lv_old, const int *__restrict__ urp, const int *__restrict__ uci,
    const double *__restrict__ uv, double *__restrict__ lnew, double *__restrict__ unew)
{
    __shared__ int s_col[PLT_SW_WARPS][PLT_ROW_CAP];
    __shared__ double s_t[PLT_SW_WARPS][PLT_ROW_CAP];
    __shared__ unsigned s_h[PLT_SW_WARPS][PLT_HASH];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int *col = s_col[w];
    double *t = s_t[w];
    unsigned *ht = s_h[w];
    const bool wide = n > 0xffffff;  // columns up to n - 1 may share their low 24 bits
    for (int i = blockIdx.x * PLT_SW_WARPS + w; i < n; i += gridDim.x * PLT_SW_WARPS) {
        const int l0 = lrp[i], l1 = lrp[i + 1];
        // L row i: strict entries first (ascending), the unit diagonal (col i) last
        const int nl = (l1 > l0 && lci[l1 - 1] >= i) ? l1 - l0 - 1 : l1 - l0;
        const int u0 = urp[i], nu = urp[i + 1] - u0;
        const int m = nl + nu;
        if (m >= PLT_ROW_CAP) {
            // per-entry walk for an unusually long row (the table takes rows
            // of up to PLT_ROW_CAP - 1 entries: positions below 255, so no
            // key equals the empty word)
            if (parts & 1) {
                for (int q = lane; q < l1 - l0; q += 32) {
                    const int k = l0 + q, j = lci[k];
                    if (j >= i) { lnew[k] = lv_old[k]; continue; }
                    const double tv = plt_sweep_value(arp, aci, av, lrp, lci, lv_k, urp, uci, uv, i, j);
                    lnew[k] = tv / uv[urp[j]];
                }
            }
            if (parts & 2) {
                for (int q = lane; q < nu; q += 32)
                    unew[u0 + q] = plt_sweep_value(arp, aci, av, lrp, lci, lv_k, urp, uci, uv, i, uci[u0 + q]);
            }
            continue;
        }
        for (int s2 = lane; s2 < PLT_HASH; s2 += 32) ht[s2] = PLT_HASH_EMPTY;
        __syncwarp();
        for (int q = lane; q < m; q += 32) {
            const int j = q < nl ? lci[l0 + q] : uci[u0 + q - nl];
            col[q] = j;
            const int pa = find_pos(aci, arp[i], arp[i + 1], j);
            t[q] = pa >= 0 ? av[pa] : 0.0;
            const unsigned kv = plt_hash_key(j, q);
            for (unsigned sl = plt_hash_slot(j);; sl = (sl + 1) & (PLT_HASH - 1))
                if (atomicCAS(ht + sl, PLT_HASH_EMPTY, kv) == PLT_HASH_EMPTY) break;
        }
        __syncwarp();
        // only the products that reach a requested part: L part needs k < j < i
        // (every k of L row i may contribute); U part needs k < i
        // the L entries' columns, values and U row ranges are loaded 32 at a
        // time, one per lane, and handed out by shuffle: per L entry only the
        // U row's own loads remain on the dependent path
        for (int kb = 0; kb < nl; kb += 32) {
            const int myq = kb + lane;
            int mk = 0, mb = 0, me = 0;
            double ml = 0.0;
            if (myq < nl) {
                mk = lci[l0 + myq];
                ml = lv_k[l0 + myq];
                mb = urp[mk];
                me = urp[mk + 1];
            }
            const int cnt = min(32, nl - kb);
            for (int cq = 0; cq < cnt; cq++) {
                const int k = __shfl_sync(0xffffffffu, mk, cq);
                const double lk = __shfl_sync(0xffffffffu, ml, cq);
                const int e0 = __shfl_sync(0xffffffffu, mb, cq), e1 = __shfl_sync(0xffffffffu, me, cq);
                for (int e = e0 + lane; e < e1; e += 32) {
                    const int j = uci[e];
                    if (j == k) continue;
                    if (!(parts & 2) && j >= i) continue;
                    if (!(parts & 1) && j < i) continue;
                    // position of j in the row's pattern (hash lookup)
                    const int pos = plt_hash_find(ht, col, wide, j);
                    if (pos >= 0) t[pos] = t[pos] - lk * uv[e];
                }
                __syncwarp();
            }
        }
        for (int q = lane; q < m; q += 32) {
            const int j = col[q];
            if (q < nl) {
                if (parts & 1) lnew[l0 + q] = t[q] / uv[urp[j]];  // u_jj: first entry of U row j
            } else if (parts & 2) {
                unew[u0 + q - nl] = t[q];
            }
        }
        if ((parts & 1) && nl < l1 - l0 && lane == 0) lnew[l1 - 1] = lv_old[l1 - 1];  // unit diagonal unchanged
        __syncwarp();
    }
}

// radix-select histogram: count |v| bit patterns whose bits above `shift+8`
// equal the prefix selected so far (state[0]), binned by the 8 bits at `shift`
static __global__ void k_radix_hist(long m, const double *__restrict__ v, const unsigned long long *state, int shift,
                             unsigned long long *hist)
{
    __shared__ unsigned int sh[256];
    for (int q = threadIdx.x; q < 256; q += blockDim.x) sh[q] = 0;
    __syncthreads();
    const unsigned long long prefix = state[0];
    const int hi = shift + 8;
    for (long k = blockIdx.x * (long)blockDim.x + threadIdx.x; k < m; k += (long)gridDim.x * blockDim.x) {
        const unsigned long long b = (unsigned long long)__double_as_longlong(fabs(v[k]));
        if (hi >= 64 || (b >> hi) == prefix) atomicAdd(&sh[(b >> shift) & 255u], 1u);
    }
    __syncthreads();
    for (int q = threadIdx.x; q < 256; q += blockDim.x)
        if (sh[q]) atomicAdd(hist + q, (unsigned long long)sh[q]);
}

// one thread: the bin holding the state[1]-th smallest pattern (1-based) of
// this pass's histogram; state[0] = (state[0] << 8) | bin, state[1] -= the
// counts of the bins below; the histogram is cleared for the next pass
static __global__ void k_radix_pick(unsigned long long *state, unsigned long long *hist)
{
    unsigned long long k = state[1];
    int bin = 0;
    for (; bin < 256; bin++) {
        if (hist[bin] >= k) break;
        k -= hist[bin];
    }
    if (bin == 256) bin = 255;
    state[0] = (state[0] << 8) | (unsigned long long)bin;
    state[1] = k;
    for (int q = 0; q < 256; q++) hist[q] = 0;
}

// Threshold keep rule, one row of L (upper = 0: unit diagonal last, drop
// |l_ij| < droptol) or of U (upper = 1: diagonal first, drop |u_ij| <
// droptol*|u_jj|, u_jj the first entry of U row j); diagonals are kept.
__device__ __forceinline__ bool plt_keep(int k, int a, int b, int upper, const int *rp, const int *ci, const double *v,
                                         double thr, double droptol)
{
    if (k == (upper ? a : b - 1)) return true;
    const double x = fabs(v[k]);
    if (x < thr) return false;
    if (droptol > 0) {
        const double lim = upper ? droptol * fabs(v[rp[ci[k]]]) : droptol;
        if (x < lim) return false;
    }
    return true;
}
// keep counts per row (warp per row)
static __global__ void k_keep_count(int n, const int *__restrict__ rp, const int *__restrict__ ci,
                             const double *__restrict__ v, double thr, double droptol, int upper, int *cnt)
{
    const int lane = threadIdx.x & 31;
    const int wpb = blockDim.x >> 5;
    for (int i = blockIdx.x * wpb + (threadIdx.x >> 5); i < n; i += gridDim.x * wpb) {
        const int a = rp[i], b = rp[i + 1];
        int c = 0;
        for (int k = a + lane; k < b; k += 32) c += plt_keep(k, a, b, upper, rp, ci, v, thr, droptol);
        for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
        if (lane == 0) cnt[i] = c;
    }
}
// kept entries in order (warp per row, ballot compaction)
static __global__ void k_keep_fill(int n, const int *__restrict__ rp, const int *__restrict__ ci, const double *__restrict__ v,
                            double thr, double droptol, int upper, const int *__restrict__ nrp, int *nci, double *nv)
{
    const int lane = threadIdx.x & 31;
    const int wpb = blockDim.x >> 5;
    for (int i = blockIdx.x * wpb + (threadIdx.x >> 5); i < n; i += gridDim.x * wpb) {
        const int a = rp[i], b = rp[i + 1];
        int p = nrp[i];
        for (int base = a; base < b; base += 32) {
            const int k = base + lane;
            const bool keep = k < b && plt_keep(k, a, b, upper, rp, ci, v, thr, droptol);
            const unsigned m = __ballot_sync(0xffffffffu, keep);
            if (keep) {
                const int q = p + __popc(m & ((1u << lane) - 1));
                nci[q] = ci[k];
                nv[q] = v[k];
            }
            p += __popc(m);
        }
    }
}

// final conversion: L strict (drop the unit diagonal), dinv, U' = dinv*U strict
static __global__ void k_plt_final_count(int n, const int *__restrict__ lrp, const int *__restrict__ urp, int *lc, int *uc)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        lc[i] = lrp[i + 1] - lrp[i] - 1;
        uc[i] = urp[i + 1] - urp[i] - 1;
    }
}
static __global__ void k_plt_final_fill(int n, const int *__restrict__ lrp, const int *__restrict__ lci, const double *__restrict__ lv,
                                 const int *__restrict__ urp, const int *__restrict__ uci, const double *__restrict__ uv,
                                 const int *__restrict__ olrp, int *olci, double *olv, double *dinv,
                                 const int *__restrict__ ourp, int *ouci, double *ouv)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        int p = olrp[i];
        for (int k = lrp[i]; k < lrp[i + 1]; k++)
            if (lci[k] < i) { olci[p] = lci[k]; olv[p] = lv[k]; p++; }
        double d = 0.0;
        for (int k = urp[i]; k < urp[i + 1]; k++)
            if (uci[k] == i) d = uv[k];
        const double di = 1.0 / d;
        dinv[i] = di;
        p = ourp[i];
        for (int k = urp[i]; k < urp[i + 1]; k++)
            if (uci[k] > i) { ouci[p] = uci[k]; ouv[p] = uv[k] * di; p++; }
    }
}

// position of each row's diagonal entry (binary search of the sorted row);
// a row without one sets DEV_NO_DIAG
static __global__ void k_plt_diag_pos(int n, const int *__restrict__ arp, const int *__restrict__ aci, int *uptr, int *err)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int p = find_pos(aci, arp[i], arp[i + 1], i);
        uptr[i] = p;
        if (p < 0) atomicOr(err, DEV_NO_DIAG);
    }
}

// initial factors: L = strict lower(A)/a_jj + unit diag (last), U = upper(A)
static __global__ void k_plt_init_count(int n, const int *__restrict__ arp, const int *__restrict__ aci, int *lc, int *uc)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        int l = 0;
        for (int k = arp[i]; k < arp[i + 1]; k++) l += aci[k] < i;
        lc[i] = l + 1;
        uc[i] = arp[i + 1] - arp[i] - l;
    }
}
static __global__ void k_plt_init_fill(int n, const int *__restrict__ arp, const int *__restrict__ aci,
                                const double *__restrict__ av, const int *__restrict__ uptr, const int *__restrict__ lrp,
                                int *lci, double *lv, const int *__restrict__ urp, int *uci, double *uv)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        int pl = lrp[i], pu = urp[i];
        for (int k = arp[i]; k < arp[i + 1]; k++) {
            const int c = aci[k];
            if (c < i) { lci[pl] = c; lv[pl] = av[k] / av[uptr[c]]; pl++; }
            else { uci[pu] = c; uv[pu] = av[k]; pu++; }
        }
        lci[pl] = i;
        lv[pl] = 1.0;
    }
}

// ---------------------------------------------------------------- host driver
// Exclusive scan of the per-row counts into a row pointer, on the device:
// tile sums (SCAN_TILE counts per block), one block scans the tile sums,
// then every tile rescans its counts from its offset.  Totals are formed in
// 64 bits; a row pointer that would pass INT_MAX - 64 sets DEV_CAPACITY.
constexpr int SCAN_THREADS = 1024, SCAN_IPT = 8, SCAN_TILE = SCAN_THREADS * SCAN_IPT;

__device__ __forceinline__ long block_excl_scan(long v, long *sw, long &total)
{
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    long incl = v;
    for (int o = 1; o < 32; o <<= 1) {
        const long y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += y;
    }
    if (lane == 31) sw[w] = incl;
    __syncthreads();
    if (w == 0) {
        long x = lane < nw ? sw[lane] : 0;
        for (int o = 1; o < 32; o <<= 1) {
            const long y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        if (lane < nw) sw[lane] = x;  // inclusive warp totals
    }
    __syncthreads();
    total = sw[nw - 1];
    const long r = (w > 0 ? sw[w - 1] : 0) + incl - v;
    __syncthreads();  // sw is reused by the next call
    return r;
}

static __global__ void __launch_bounds__(SCAN_THREADS) k_scan_tile_sums(int n, const int *__restrict__ cnt, long *bsum)
{
    __shared__ long sw[32];
    const long base = (long)blockIdx.x * SCAN_TILE;
    long v = 0;
    for (int q = threadIdx.x; q < SCAN_TILE; q += SCAN_THREADS)
        if (base + q < n) v += cnt[base + q];
    long total;
    block_excl_scan(v, sw, total);
    if (threadIdx.x == 0) bsum[blockIdx.x] = total;
}

// one block: exclusive scan of nb tile sums in place, grand total into bsum[nb]
static __global__ void __launch_bounds__(SCAN_THREADS) k_scan_tile_offsets(int nb, long *bsum)
{
    __shared__ long sw[32];
    long carry = 0;
    for (int base = 0; base < nb; base += SCAN_THREADS) {
        const int q = base + threadIdx.x;
        const long v = q < nb ? bsum[q] : 0;
        long total;
        const long e = block_excl_scan(v, sw, total);
        if (q < nb) bsum[q] = carry + e;
        carry += total;
    }
    if (threadIdx.x == 0) bsum[nb] = carry;
}

static __global__ void __launch_bounds__(SCAN_THREADS) k_scan_tile_write(int n, const int *__restrict__ cnt,
                                                                  const long *__restrict__ boff, int *rp, int *err)
{
    __shared__ long sw[32];
    const long base = (long)blockIdx.x * SCAN_TILE + (long)threadIdx.x * SCAN_IPT;
    int c[SCAN_IPT];
    long v = 0;
#pragma unroll
    for (int u = 0; u < SCAN_IPT; u++) {
        c[u] = base + u < n ? cnt[base + u] : 0;
        v += c[u];
    }
    long total;
    long acc = boff[blockIdx.x] + block_excl_scan(v, sw, total);
    bool over = false;
#pragma unroll
    for (int u = 0; u < SCAN_IPT; u++) {
        if (base + u < n) {
            over |= acc > 0x7fffffffL - 64;
            rp[base + u] = (int)acc;
        }
        acc += c[u];
    }
    if (base < n && base + SCAN_IPT >= n) {  // the thread holding the last row writes rp[n]
        over |= acc > 0x7fffffffL - 64;
        rp[n] = (int)acc;
    }
    if (over) atomicOr(err, DEV_CAPACITY);
}

// Grid of a warp-per-row kernel: every block resident at once (the blocks
// take rows grid-strided, so each gets the same share; a grid larger than
// what fits would run its surplus as a partial second wave), at most one
// warp per row.
template <typename K>
inline int plt_resident_grid(K kern, int warps, int n)
{
    int per_sm = 0;
    XS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 32 * warps, 0));
    const long rows_cap = ((long)n + warps - 1) / warps;
    return (int)std::max(1L, std::min(rows_cap, (long)std::max(per_sm, 1) * geom().sms));
}

struct PltCtx {
    cudaStream_t s;
    int *err;
    int n;
    DBuf<long> bsum;
    int grid() const { return geom().sms * 8; }
};

// counts (device, n) -> rowptr (device, n+1) on the device; returns nnz
inline long scan_counts(PltCtx &c, const DBuf<int> &cnt, DBuf<int> &rp)
{
    const int n = c.n;
    const int nb = std::max(1, (n + SCAN_TILE - 1) / SCAN_TILE);
    if (c.bsum.n < (size_t)nb + 1) c.bsum.alloc(nb + 1);
    if (rp.n != (size_t)n + 1) rp.alloc(n + 1);
    k_scan_tile_sums<<<nb, SCAN_THREADS, 0, c.s>>>(n, cnt, c.bsum);
    k_scan_tile_offsets<<<1, SCAN_THREADS, 0, c.s>>>(nb, c.bsum);
    k_scan_tile_write<<<nb, SCAN_THREADS, 0, c.s>>>(n, cnt, c.bsum, rp, c.err);
    check_launch();
    long total = 0;
    int e = 0;
    XS_CUDA(cudaMemcpyAsync(&total, c.bsum.p + nb, sizeof(long), cudaMemcpyDeviceToHost, c.s));
    XS_CUDA(cudaMemcpyAsync(&e, c.err, sizeof(int), cudaMemcpyDeviceToHost, c.s));
    XS_CUDA(cudaStreamSynchronize(c.s));
    if (e) throw Status(dev_err_to_status(e));
    if (total > 0x7fffffffL - 64) throw Status(XS_ERR_CAPACITY);
    return total;
}

// k-th smallest |v| (1-based) by radix select over the IEEE bit patterns
inline double plt_kth_abs(PltCtx &c, const DBuf<double> &v, long m, long k)
{
    if (k <= 0 || m <= 0) return 0.0;
    // the 8 passes run on the device (the bin of each pass picked by one
    // thread); the host reads the selected pattern once
    DBuf<unsigned long long> hist, state;
    hist.alloc(256);
    state.alloc(2);
    const unsigned long long init[2] = {0ull, (unsigned long long)k};
    state.upload(init, 2, c.s);
    for (int shift = 56; shift >= 0; shift -= 8) {
        k_radix_hist<<<c.grid(), 256, 0, c.s>>>(m, v, state, shift, hist);
        k_radix_pick<<<1, 1, 0, c.s>>>(state, hist);
        check_launch();
    }
    unsigned long long prefix = 0;
    XS_CUDA(cudaMemcpyAsync(&prefix, state.p, sizeof(prefix), cudaMemcpyDeviceToHost, c.s));
    XS_CUDA(cudaStreamSynchronize(c.s));
    double out;
    std::memcpy(&out, &prefix, sizeof(double));
    return out;
}

inline void parilut_build(cudaStream_t s, int *err, int n, const Operator &A, double fill, int sweeps, double droptol,
                          ParilutResult &R)
{
    Trace tr_all("parilut_build", s);
    // every temporary of the sweeps comes from the stream-ordered pool
    PoolScope pool(s);
    Trace tr_init("  initial factors", s);
    PltCtx c{s, err, n, {}};
    const int G = c.grid();
    const long nnzA = A.nnz;
    XS_CUDA(cudaMemsetAsync(err, 0, sizeof(int), s));
    // diagonal positions (rows are sorted)
    DBuf<int> d_uptr;
    d_uptr.alloc(n);
    k_plt_diag_pos<<<G, 256, 0, s>>>(n, A.rp, A.ci, d_uptr, err);
    check_launch();
    {
        int e = 0;
        XS_CUDA(cudaMemcpyAsync(&e, err, sizeof(int), cudaMemcpyDeviceToHost, s));
        XS_CUDA(cudaStreamSynchronize(s));
        if (e) throw Status(dev_err_to_status(e));
    }
    // initial factors
    DCsr L, U;
    DBuf<int> lc, uc;
    lc.alloc(n);
    uc.alloc(n);
    k_plt_init_count<<<G, 256, 0, s>>>(n, A.rp, A.ci, lc, uc);
    check_launch();
    L.n = U.n = n;
    L.nnz = scan_counts(c, lc, L.rp);
    U.nnz = scan_counts(c, uc, U.rp);
    L.ci.alloc(L.nnz); L.v.alloc(L.nnz);
    U.ci.alloc(std::max<long>(U.nnz, 1)); U.v.alloc(std::max<long>(U.nnz, 1));
    k_plt_init_fill<<<G, 256, 0, s>>>(n, A.rp, A.ci, A.v, d_uptr, L.rp, L.ci, L.v, U.rp, U.ci, U.v);
    check_launch();
    const long l0nnz = L.nnz, u0nnz = U.nnz;
    DBuf<double> udiag;
    udiag.alloc(n);
    DBuf<int> cnt;
    cnt.alloc(n);
    tr_init.stop();
    for (int sw = 0; sw < sweeps; sw++) {
        Trace tr_sw("parilut sweep", s);
        const double rate = (fill - 1) / sweeps * (sw + 1) + 1;
        k_udiag<<<G, 256, 0, s>>>(n, U.rp, U.v, udiag);
        check_launch();
        // candidates
        Trace tr_cand("  candidates", s);
        DCsr D;
        D.n = n;
        const int cg = plt_resident_grid(k_candidates, PLT_WARPS, n);
        k_candidates<<<cg, 32 * PLT_WARPS, 0, s>>>(n, A.rp, A.ci, L.rp, L.ci, U.rp, U.ci, 0, cnt, nullptr, nullptr, err);
        check_launch();
        D.nnz = scan_counts(c, cnt, D.rp);
        D.ci.alloc(std::max<long>(D.nnz, 1));
        D.v.alloc(std::max<long>(D.nnz, 1));
        k_candidates<<<cg, 32 * PLT_WARPS, 0, s>>>(n, A.rp, A.ci, L.rp, L.ci, U.rp, U.ci, 1, nullptr, D.rp, D.ci, err);
        check_launch();
        tr_cand.stop();
        Trace tr_val("  candidate values", s);
        k_candidate_values<<<plt_resident_grid(k_candidate_values, PLT_CV_WARPS, n),
                             32 * PLT_CV_WARPS, 0, s>>>(n, A.rp, A.ci, A.v, L.rp, L.ci, L.v, U.rp, U.ci, U.v, udiag,
                                                        D.rp, D.ci, D.v);
        check_launch();
        {
            int e = 0;
            XS_CUDA(cudaMemcpyAsync(&e, err, sizeof(int), cudaMemcpyDeviceToHost, s));
            XS_CUDA(cudaStreamSynchronize(s));
            if (e) throw Status(dev_err_to_status(e));
        }
        tr_val.stop();
        Trace tr_split("  split", s);
        // split
        DCsr L2, U2;
        L2.n = U2.n = n;
        k_split_count<<<G, 256, 0, s>>>(n, D.rp, D.ci, lc, uc);
        check_launch();
        L2.nnz = scan_counts(c, lc, L2.rp);
        U2.nnz = scan_counts(c, uc, U2.rp);
        L2.ci.alloc(L2.nnz); L2.v.alloc(L2.nnz);
        U2.ci.alloc(std::max<long>(U2.nnz, 1)); U2.v.alloc(std::max<long>(U2.nnz, 1));
        k_split_fill<<<G, 256, 0, s>>>(n, D.rp, D.ci, D.v, L2.rp, L2.ci, L2.v, U2.rp, U2.ci, U2.v);
        check_launch();
        const long nnzD = D.nnz;
        D = DCsr();
        tr_split.stop();
        Trace tr_s1("  LU sweep", s);
        // LU sweep (synchronous): both parts from the old values
        const int rg = plt_resident_grid(k_plt_sweep_rows, PLT_SW_WARPS, n);
        {
            DBuf<double> lnew, unew;
            lnew.alloc(L2.nnz);
            unew.alloc(std::max<long>(U2.nnz, 1));
            k_plt_sweep_rows<<<rg, 32 * PLT_SW_WARPS, 0, s>>>(n, 3, A.rp, A.ci, A.v, L2.rp, L2.ci, L2.v, L2.v, U2.rp,
                                                               U2.ci, U2.v, lnew, unew);
            check_launch();
            L2.v = std::move(lnew);
            U2.v = std::move(unew);
        }
        tr_s1.stop();
        Trace tr_th("  threshold", s);
        // threshold removal
        const long keep_nnz = std::lround(rate * (double)nnzA);
        const long remove_nnz = nnzD - keep_nnz;
        DCsr L3, U3;
        if (remove_nnz > 0 || droptol > 0) {
            double lthr = 0.0, uthr = 0.0;
            if (remove_nnz > 0) {
                const long lkeep = (long)(rate * l0nnz);
                const long lremove = std::max(L2.nnz - lkeep, 0L);
                const long ukeep = (long)(rate * u0nnz);
                const long uremove = std::max(U2.nnz - ukeep, 0L);
                lthr = plt_kth_abs(c, L2.v, L2.nnz, lremove);
                uthr = plt_kth_abs(c, U2.v, U2.nnz, uremove);
            }
            L3.n = U3.n = n;
            k_keep_count<<<G, 256, 0, s>>>(n, L2.rp, L2.ci, L2.v, lthr, droptol, 0, lc);
            k_keep_count<<<G, 256, 0, s>>>(n, U2.rp, U2.ci, U2.v, uthr, droptol, 1, uc);
            check_launch();
            L3.nnz = scan_counts(c, lc, L3.rp);
            U3.nnz = scan_counts(c, uc, U3.rp);
            L3.ci.alloc(L3.nnz); L3.v.alloc(L3.nnz);
            U3.ci.alloc(std::max<long>(U3.nnz, 1)); U3.v.alloc(std::max<long>(U3.nnz, 1));
            k_keep_fill<<<G, 256, 0, s>>>(n, L2.rp, L2.ci, L2.v, lthr, droptol, 0, L3.rp, L3.ci, L3.v);
            k_keep_fill<<<G, 256, 0, s>>>(n, U2.rp, U2.ci, U2.v, uthr, droptol, 1, U3.rp, U3.ci, U3.v);
            check_launch();
        } else {
            L3 = std::move(L2);
            U3 = std::move(U2);
        }
        tr_th.stop();
        Trace tr_s2("  L/U sweeps", s);
        // L sweep, then U sweep with the new L
        {
            DBuf<double> lnew, unew;
            lnew.alloc(L3.nnz);
            k_plt_sweep_rows<<<rg, 32 * PLT_SW_WARPS, 0, s>>>(n, 1, A.rp, A.ci, A.v, L3.rp, L3.ci, L3.v, L3.v, U3.rp,
                                                               U3.ci, U3.v, lnew, nullptr);
            check_launch();
            L3.v = std::move(lnew);
            unew.alloc(std::max<long>(U3.nnz, 1));
            k_plt_sweep_rows<<<rg, 32 * PLT_SW_WARPS, 0, s>>>(n, 2, A.rp, A.ci, A.v, L3.rp, L3.ci, L3.v, L3.v, U3.rp,
                                                               U3.ci, U3.v, nullptr, unew);
            check_launch();
            U3.v = std::move(unew);
        }
        L = std::move(L3);
        U = std::move(U3);
    }
    // seqilu0 layout (kept after the build: ordinary allocations)
    pool.end();
    Trace tr_fin("  final layout + download", s);
    R.n = n;
    k_plt_final_count<<<G, 256, 0, s>>>(n, L.rp, U.rp, lc, uc);
    check_launch();
    R.nnzL = scan_counts(c, lc, R.lrp);
    R.nnzU = scan_counts(c, uc, R.urp);
    R.lci.alloc(std::max<long>(R.nnzL, 1)); R.lv.alloc(std::max<long>(R.nnzL, 1));
    R.uci.alloc(std::max<long>(R.nnzU, 1)); R.uv.alloc(std::max<long>(R.nnzU, 1));
    R.dinv.alloc(n);
    k_plt_final_fill<<<G, 256, 0, s>>>(n, L.rp, L.ci, L.v, U.rp, U.ci, U.v, R.lrp, R.lci, R.lv, R.dinv, R.urp, R.uci,
                                       R.uv);
    check_launch();
    Trace tr_dl("    pattern download", s);
    // uninitialised host arrays whose pages are first touched by parallel
    // threads (a zero-filling resize faults them in on one thread)
    auto fetch = [&](HostArray<int> &h, const DBuf<int> &d, long cnt) {
        h.resize(cnt);
        host_parallel_for((cnt + 262143) / 262144, 1, [&](long b) {
            const long k1 = std::min(cnt, (b + 1) * 262144L);
            for (long k = b * 262144L; k < k1; k += 1024) h[k] = 0;
        });
        if (cnt) d.download(h.data(), cnt, s);
    };
    fetch(R.hlrp, R.lrp, n + 1);
    fetch(R.hurp, R.urp, n + 1);
    fetch(R.hlci, R.lci, R.nnzL);
    fetch(R.huci, R.uci, R.nnzU);
    std::vector<long> ident(n);
    std::iota(ident.begin(), ident.end(), 0L);
    R.diag_ident.alloc(n);
    R.diag_ident.upload(ident.data(), n, s);
    XS_CUDA(cudaStreamSynchronize(s));
}

// prepare the sync-free solve plans for ParILUT factors (own pattern)
inline void ilut_to_tri(cudaStream_t s, int n, ParilutResult &R, TriDev &L, TriDev &U, bool need32)
{
    Trace tr_all("ilut_to_tri", s);
    auto up = [&](TriDev &T, const HostArray<int> &nrp, const HostArray<int> &nci, const int *drp, const int *dci,
                  bool upper, const double *vals) {
        T = TriDev();
        {
            Trace tr("  build_tri_dev", s);
            build_tri_dev(T, n, nrp, nci, upper, [](int k) { return (long)k; }, s, /*identity_src=*/true, drp, dci,
                          /*need_levels=*/false);
        }
        const long m = std::max<long>(T.nnz, 1);
        const int g = geom().sms * 4;
        T.pv64.alloc(m, 8); T.nv64.alloc(m);
        if (T.nnz) {
            k_gather_convert<double><<<g, 256, 0, s>>>(T.nnz, T.src.p, vals, T.pv64.p);
            k_gather_convert<double><<<g, 256, 0, s>>>(T.nnz, T.src_nat.p, vals, T.nv64.p);
        }
        if (need32) {
            T.pv32.alloc(m, 8); T.nv32.alloc(m); T.pvbf.alloc(m, 8); T.nvbf.alloc(m); T.pvh.alloc(m, 8); T.nvh.alloc(m);
            if (T.nnz) {
                k_gather_convert<float><<<g, 256, 0, s>>>(T.nnz, T.src.p, vals, T.pv32.p);
                k_gather_convert<float><<<g, 256, 0, s>>>(T.nnz, T.src_nat.p, vals, T.nv32.p);
                k_gather_convert<__nv_bfloat16><<<g, 256, 0, s>>>(T.nnz, T.src.p, vals, T.pvbf.p);
                k_gather_convert<__nv_bfloat16><<<g, 256, 0, s>>>(T.nnz, T.src_nat.p, vals, T.nvbf.p);
                k_gather_convert<__half><<<g, 256, 0, s>>>(T.nnz, T.src.p, vals, T.pvh.p);
                k_gather_convert<__half><<<g, 256, 0, s>>>(T.nnz, T.src_nat.p, vals, T.nvh.p);
            }
        }
        load_tri_ell(T, vals, need32, s);
        check_launch();
        XS_CUDA(cudaStreamSynchronize(s));
    };
    host_both([&] { up(L, R.hlrp, R.hlci, R.lrp.p, R.lci.p, false, R.lv.p); },
              [&] { up(U, R.hurp, R.huci, R.urp.p, R.uci.p, true, R.uv.p); });
    const int g = geom().sms * 4;
    U.dinv64.alloc(n, 4); U.dinv64_nat.alloc(n);
    k_gather_dinv<double><<<g, 256, 0, s>>>(n, U.perm.p, R.diag_ident.p, R.dinv.p, U.dinv64.p);
    k_gather_dinv<double><<<g, 256, 0, s>>>(n, nullptr, R.diag_ident.p, R.dinv.p, U.dinv64_nat.p);
    if (need32) {
        U.dinv32.alloc(n, 4); U.dinv32_nat.alloc(n);
        k_gather_dinv<float><<<g, 256, 0, s>>>(n, U.perm.p, R.diag_ident.p, R.dinv.p, U.dinv32.p);
        k_gather_dinv<float><<<g, 256, 0, s>>>(n, nullptr, R.diag_ident.p, R.dinv.p, U.dinv32_nat.p);
    }
    check_launch();
    XS_CUDA(cudaStreamSynchronize(s));
}

}  // namespace xs
