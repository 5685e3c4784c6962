// ILU(0) factorisations on A's sparsity pattern.
//
// Exact ILU(0): the reference factorises on the CPU (hip/Precond/
// ilut_diag_in_csr.cpp:347-405, ilu0_simple: IKJ order, pivots clamped to
// 1e-20).  Here the same up-looking row update runs on the GPU: row i is
// processed by one thread once every row k it references (its strictly lower
// columns) is final, so rows of one dependency level run in parallel.  The
// row update is performed in exactly the CPU order (pivot division, then the
// merge with row k's upper part), so the factors are bitwise identical to the
// reference's.  Completion of a row is published with a release store of the
// launch's epoch in a flag array; waiters poll with acquire loads (bounded).
//
// ParILU: the reference's fixed-point sweep (hip/Precond/gpuparilu.cpp:46-102,
// ilu0_ij_aw, one thread per nonzero, pivot clamp 1e-10) applied as
// synchronous sweeps (read the previous iterate, write the next), which makes
// the result deterministic; the reference updates in place asynchronously.
//
// Split: the combined values are rewritten into the seqilu0 layout
// (hip/HostMatrix/HostMatrixCSR.cpp:164-197): L entries unchanged, diagonal
// entry := dinv_i = 1/u_ii, U entries := u_ij * dinv_i.
#pragma once
#include "xs_internal.cuh"

namespace xs {


// position of column c in the sorted index range [a, b) of ci, or -1
__device__ __forceinline__ int find_col(const int *__restrict__ ci, int a, int b, int c)
{
    int l = a, r = b;
    while (l < r) {
        const int m = (l + r) >> 1;
        if (__ldg(ci + m) < c) l = m + 1;
        else r = m;
    }
    return (l < b && __ldg(ci + l) == c) ? l : -1;
}

// exact ILU(0), thread per row in level order (perm/level from the L analysis);
// used for patterns with rows of more than 32 entries.  Persistent CTAs take
// 128-row tickets in order, so only the rows a few tickets ahead of the
// slowest level are in flight: a launch with one CTA per 128 rows kept every
// resident row polling its dependencies, and those polls crowded the L2 that
// the rows on the critical path read their pivots from.  Waits back off
// exponentially up to backoff_ns.  Every ticket depends only on smaller
// tickets (level order), each held by a running CTA, so the loop progresses.
static __global__ void __launch_bounds__(128) k_ilu0_rows(int n, const int *__restrict__ rp, const int *__restrict__ ci,
                                                  const int *__restrict__ uptr, const int *__restrict__ perm, double *luv,
                                                  int *flag, int epoch, int *err, unsigned *ticket, int backoff_ns)
{
    __shared__ int s_blk;
    const int ntk = (n + 127) / 128;
    while (true) {
        if (threadIdx.x == 0) {
            const unsigned t = atomicAdd(ticket, 1u);
            // every CTA ends with one failing claim; the last of them re-arms
            if (t == (unsigned)(ntk + gridDim.x - 1)) *ticket = 0u;
            s_blk = (int)t;
        }
        __syncthreads();
        const int blk = s_blk;
        __syncthreads();
        if (blk >= ntk) return;
        const int p = blk * 128 + (int)threadIdx.x;
        if (p >= n) continue;
        if (*(volatile int *)err) continue;
        const int i = perm[p];
        const int rs = rp[i], re = rp[i + 1], up = uptr[i];
        bool ok = true;
        for (int j = rs; j < up && ok; j++) {
            const int k = ci[j];
            long spins = 0;
            unsigned long long t0 = 0;
            unsigned ns = 32;
            while (ld_acquire(flag + k) != epoch) {
                __nanosleep(ns);  // yield point: the producer may be a lane of this warp
                if (ns < (unsigned)backoff_ns) ns <<= 1;
                if ((++spins & 63) == 0) {
                    const unsigned long long t = gtimer();
                    if (t0 == 0) t0 = t;
                    else if (t - t0 > WAIT_LIMIT_NS) {
                        atomicOr(err, DEV_FACTOR_TIMEOUT);
                        ok = false;
                        break;
                    }
                    if (*(volatile int *)err) {
                        ok = false;
                        break;
                    }
                }
            }
            if (!ok) break;
            const int ukp = uptr[k];
            const int kend = rp[k + 1];
            double piv = __ldcg(luv + ukp);
            if (fabs(piv) < 1e-20) piv = 1e-20;  // no-op: row k clamped its own pivot
            const double lij = luv[j] / piv;
            luv[j] = lij;
            int subptr = ukp;
            for (int jj = j + 1; jj < re; jj++) {
                const int kk = ci[jj];
                while (subptr < kend && __ldg(ci + subptr) < kk) subptr++;
                if (subptr < kend) {
                    if (__ldg(ci + subptr) == kk) {
                        const double t = lij * __ldcg(luv + subptr);
                        luv[jj] = luv[jj] - t;
                    }
                } else
                    break;
            }
        }
        if (!ok) continue;
        double d = luv[up];
        if (fabs(d) < 1e-20) {
            d = 1e-20;
            luv[up] = d;
        }
        __threadfence();
        st_release(flag + i, epoch);
    }
}

// Exact ILU(0) with a group of G lanes per row (G >= the longest row, G a
// power of two <= 32), 128/G rows per ticket, tickets in level order as in
// k_ilu0_rows.  Lane q holds entry rs+q of row i in a register.  Rows with at
// most PLT_L_MAX strictly lower entries (nl) go in three phases:
//   1. pattern only, before any wait: lane q finds its column in the upper
//      part of every row k_j (k_j = column of L entry j < q);
//   2. lanes 0..nl-1 wait for the flags of their own columns k_q at once,
//      then every lane loads the values it needs (the pivots u_kk by lanes
//      0..nl-1, u_{k_j,c_q} at the positions of phase 1) in one round;
//   3. for j = 0..nl-1 in order: l = a_j / u_{k_j k_j} (a_j, u from lane j
//      by shuffle), lane j keeps l, every lane q > j with a match does
//      a_q = a_q - l * u_{k_j,c_q}; then the diagonal clamp, the row is
//      written back and its flag released.
// These are the operations of the thread-per-row IKJ update entry by entry
// in the same j order, so the factors are bitwise the same; the critical
// path of a row is one wait for its latest dependency, one L2 round trip
// and a few shuffles.  Rows with more lower entries take the elimination
// steps one at a time (locate, wait, load, update per L entry).
constexpr int ILU_L_MAX = 16;

template <int G>
__global__ void __launch_bounds__(128) k_ilu0_groups(int n, const int *__restrict__ rp, const int *__restrict__ ci,
                                                    const int *__restrict__ uptr, const int *__restrict__ perm,
                                                    double *luv, int *flag, int epoch, int *err, unsigned *ticket,
                                                    int backoff_ns)
{
    constexpr int RPB = 128 / G;  // rows per ticket
    constexpr int LM = G - 1 < ILU_L_MAX ? G - 1 : ILU_L_MAX;  // register-resident L entries
    __shared__ int s_blk, s_err;
    const int g = threadIdx.x / G, q = threadIdx.x % G;
    const unsigned gmask = G == 32 ? 0xffffffffu : (((1u << G) - 1u) << ((threadIdx.x & 31) / G * G));
    const int ntk = (n + RPB - 1) / RPB;
    // bounded wait of one lane for flag k; false after the limit or another error
    auto wait_flag = [&](int k) -> bool {
        long spins = 0;
        unsigned long long t0 = 0;
        unsigned ns = 32;
        while (ld_acquire(flag + k) != epoch) {
            __nanosleep(ns);  // yield point: the producer may be a lane of this warp
            if (ns < (unsigned)backoff_ns) ns <<= 1;
            if ((++spins & 63) == 0) {
                const unsigned long long t = gtimer();
                if (t0 == 0) t0 = t;
                else if (t - t0 > WAIT_LIMIT_NS) {
                    atomicOr(err, DEV_FACTOR_TIMEOUT);
                    return false;
                }
                if (*(volatile int *)err) return false;
            }
        }
        return true;
    };
    while (true) {
        if (threadIdx.x == 0) {
            const unsigned t = atomicAdd(ticket, 1u);
            // every CTA ends with one failing claim; the last of them re-arms
            if (t == (unsigned)(ntk + gridDim.x - 1)) *ticket = 0u;
            s_blk = (int)t;
            s_err = *(volatile int *)err;
        }
        __syncthreads();
        const int blk = s_blk, blk_err = s_err;
        __syncthreads();
        if (blk >= ntk) return;
        const int p = blk * RPB + g;
        if (p >= n || blk_err) continue;  // uniform over the group
        const int i = perm[p];
        const int rs = rp[i], re = rp[i + 1], up = uptr[i];
        const int nl = up - rs;
        bool ok = true;
        if (nl <= LM) {
            const bool mine = rs + q < re;
            const int c = mine ? ci[rs + q] : 0;
            double a = mine ? luv[rs + q] : 0.0;
            // phase 1: pattern lookups
            int pos[LM > 0 ? LM : 1];
#pragma unroll
            for (int j = 0; j < LM; j++) {
                pos[j] = -1;
                if (j < nl && j < q && mine) {
                    const int k = ci[rs + j];
                    pos[j] = find_col(ci, uptr[k] + 1, rp[k + 1], c);
                }
            }
            // phase 2: wait for every dependency at once, then load
            if (q < nl) ok = wait_flag(c);
            ok = __all_sync(gmask, ok);
            if (!ok) continue;
            __syncwarp(gmask);  // orders the group's loads after the acquires
            const double pv = q < nl ? __ldcg(luv + uptr[c]) : 1.0;
            double u[LM > 0 ? LM : 1];
#pragma unroll
            for (int j = 0; j < LM; j++) u[j] = pos[j] >= 0 ? __ldcg(luv + pos[j]) : 0.0;
            // phase 3: the eliminations in order, in registers
#pragma unroll
            for (int j = 0; j < LM; j++) {
                if (j < nl) {
                    double piv = __shfl_sync(gmask, pv, j, G);
                    if (fabs(piv) < 1e-20) piv = 1e-20;  // no-op: row k clamped its own pivot
                    const double lij = __shfl_sync(gmask, a, j, G) / piv;
                    if (q == j) a = lij;
                    if (pos[j] >= 0) {
                        const double t = lij * u[j];
                        a = a - t;
                    }
                }
            }
            if (q == nl && fabs(a) < 1e-20) a = 1e-20;  // diagonal clamp (entry up = rs + nl)
            if (mine) luv[rs + q] = a;
        } else {
            for (int j = rs; j < up; j++) {
                const int k = ci[j];
                const int ukp = uptr[k], kend = rp[k + 1];
                // this lane's first entry after j and its match in row k (pattern only)
                const int e0 = j + 1 + q;
                int pos0 = -1;
                if (e0 < re) pos0 = find_col(ci, ukp + 1, kend, ci[e0]);
                if (q == 0) ok = wait_flag(k);
                ok = __shfl_sync(gmask, ok, 0, G);
                if (!ok) break;
                __syncwarp(gmask);  // orders the group's loads of row k after lane 0's acquire
                double piv = __ldcg(luv + ukp);
                if (fabs(piv) < 1e-20) piv = 1e-20;  // no-op: row k clamped its own pivot
                const double lij = luv[j] / piv;
                __syncwarp(gmask);  // every lane has read a_ij before its owner overwrites it
                if (((j - rs) % G) == q) luv[j] = lij;
                for (int e = e0, pos = pos0; e < re; e += G) {
                    if (e != e0) pos = find_col(ci, ukp + 1, kend, ci[e]);
                    if (pos >= 0) {
                        const double t = lij * __ldcg(luv + pos);
                        luv[e] = luv[e] - t;
                    }
                }
                __syncwarp(gmask);  // the next L entry's value is final
            }
            if (!ok) continue;
            if (((up - rs) % G) == q) {
                const double d = luv[up];
                if (fabs(d) < 1e-20) luv[up] = 1e-20;
            }
        }
        __threadfence();
        __syncwarp(gmask);
        if (q == 0) st_release(flag + i, epoch);
    }
}

// ---------------------------------------------------------------- box-scheduled ILU(0)
// Exact ILU(0) on the box schedule of the L solve (the dependency graph of
// ILU(0) is L's): persistent CTAs take boxes in wavefront order by ticket.
// A CTA stages its box's entries — values and column indices, in the box's
// entry order (rows by position, each row's entries in column order) — with
// each row's entry offset and diagonal offset (= its count of strictly lower
// entries) and, per strictly lower entry, the box-local row of its column
// (-1 for a row of an earlier box); waits once for the published flags of
// the box's halo rows; then updates the rows level by level with a barrier
// between levels.  A dependency row in the box is read from shared memory; a
// halo row (final in global memory) has its pivot and upper part loaded in
// one round of independent loads.  Each row update is the reference's IKJ
// step: the pivot division, then for every later entry of the row the
// subtraction of l_ik * u_kj where row k's upper part has that column — the
// same operations in the same order as the thread-per-row kernel, so the
// factors are bitwise the same.  The rows are written back and their flags
// released.  Waits are bounded.
//   ent[e]   : A's entry index of box entry e (boxes consecutive; ebase[t])
//   roff[p]  : entry offset of the row at position p within its box
//   rdiag[p] : offset of that row's diagonal within the row
//   loff[p]  : offset of the row's strictly lower entries among the box's
//              (boxes consecutive; lbase[t])
//   dep[l]   : box-local row (position - first position of the box) of the
//              column of strictly lower entry l, or -1 (a halo row)
constexpr int ILU_TILE_THREADS = 256;
constexpr size_t ILU_TILE_SMEM_MAX = 224 * 1024;
constexpr int ILU_HALO_U = 8;   // upper-part entries of a halo row held in registers
constexpr int ILU_STAGE_U = 8;  // entries per thread per staging round

struct IluTileArgs {
    int ntiles;
    const int *rp, *ci, *uptr;
    double *luv;
    const int *tile_pos, *tile_lvl, *lvl_ptr, *perm, *halo_ptr, *halo_row;
    const int *ebase, *ent, *roff, *rdiag, *lbase, *loff, *dep;
    int *flag, epoch, *err;
    unsigned *ticket;
};

// shared-memory layout of a box with E entries, EL strictly lower ones and R rows
struct IluTileSmem {
    size_t val, col, row, diag, lof, dep, total;
    static __host__ __device__ IluTileSmem of(int E, int EL, int R)
    {
        auto al = [](size_t b) { return (b + 15) & ~(size_t)15; };
        IluTileSmem m;
        m.val = 0;
        m.col = m.val + al((size_t)E * sizeof(double));
        m.row = m.col + al((size_t)E * sizeof(int));
        m.diag = m.row + al((size_t)(R + 1) * sizeof(int));
        m.lof = m.diag + al((size_t)R * sizeof(int));
        m.dep = m.lof + al((size_t)R * sizeof(int));
        m.total = m.dep + al((size_t)EL * sizeof(int));
        return m;
    }
};

static __global__ void __launch_bounds__(ILU_TILE_THREADS) k_ilu0_tiles(IluTileArgs A, int max_entries, int max_lower,
                                                                          int max_rows)
{
    extern __shared__ __align__(16) unsigned char ilu_smem[];
    const IluTileSmem L = IluTileSmem::of(max_entries, max_lower, max_rows);
    double *sv = (double *)(ilu_smem + L.val);
    int *sc = (int *)(ilu_smem + L.col);
    int *srow = (int *)(ilu_smem + L.row);
    int *sdg = (int *)(ilu_smem + L.diag);
    int *slof = (int *)(ilu_smem + L.lof);
    int *sdep = (int *)(ilu_smem + L.dep);
    __shared__ int s_t, s_err;
    while (true) {
        if (threadIdx.x == 0) {
            const unsigned t = atomicAdd(A.ticket, 1u);
            // every CTA ends with one failing claim; the last of them re-arms
            if (t == (unsigned)(A.ntiles + gridDim.x - 1)) *A.ticket = 0u;
            s_t = (int)t;
            s_err = *(volatile int *)A.err;
        }
        __syncthreads();
        const int t = s_t, e0 = s_err;
        __syncthreads();
        if (t >= A.ntiles) return;
        if (e0) continue;
        const int p0 = A.tile_pos[t], p1 = A.tile_pos[t + 1], rows = p1 - p0;
        const int eb = A.ebase[t], E = A.ebase[t + 1] - eb;
        const int lb = A.lbase[t], EL = A.lbase[t + 1] - lb;
        // stage (A's values: nothing else writes the box's rows), ILU_STAGE_U
        // entries per thread per round so their gathers are in flight together
        for (int e0 = threadIdx.x; e0 < E; e0 += blockDim.x * ILU_STAGE_U) {
            int jv[ILU_STAGE_U];
#pragma unroll
            for (int u = 0; u < ILU_STAGE_U; u++) {
                const int e = e0 + u * (int)blockDim.x;
                jv[u] = e < E ? __ldg(A.ent + eb + e) : -1;
            }
            double vv[ILU_STAGE_U];
            int cv[ILU_STAGE_U];
#pragma unroll
            for (int u = 0; u < ILU_STAGE_U; u++) {
                if (jv[u] >= 0) {
                    vv[u] = __ldcg(A.luv + jv[u]);
                    cv[u] = __ldg(A.ci + jv[u]);
                }
            }
#pragma unroll
            for (int u = 0; u < ILU_STAGE_U; u++) {
                if (jv[u] >= 0) {
                    const int e = e0 + u * (int)blockDim.x;
                    sv[e] = vv[u];
                    sc[e] = cv[u];
                }
            }
        }
        for (int r = threadIdx.x; r < rows; r += blockDim.x) {
            srow[r] = A.roff[p0 + r];
            sdg[r] = A.rdiag[p0 + r];
            slof[r] = A.loff[p0 + r];
        }
        for (int l = threadIdx.x; l < EL; l += blockDim.x) sdep[l] = A.dep[lb + l];
        if (threadIdx.x == 0) srow[rows] = E;
        // the halo rows' flags (bounded waits)
        bool ok = true;
        for (int h = A.halo_ptr[t] + (int)threadIdx.x; h < A.halo_ptr[t + 1] && ok; h += blockDim.x) {
            const int k = A.halo_row[h];
            long spins = 0;
            unsigned long long t0 = 0;
            unsigned ns = 32;
            while (ld_acquire(A.flag + k) != A.epoch) {
                __nanosleep(ns);
                if (ns < 512u) ns <<= 1;
                if ((++spins & 63) == 0) {
                    const unsigned long long tn = gtimer();
                    if (t0 == 0) t0 = tn;
                    else if (tn - t0 > WAIT_LIMIT_NS) {
                        atomicOr(A.err, DEV_FACTOR_TIMEOUT);
                        ok = false;
                        break;
                    }
                    if (*(volatile int *)A.err) {
                        ok = false;
                        break;
                    }
                }
            }
        }
        if (!__syncthreads_and(ok)) continue;
        for (int l = A.tile_lvl[t]; l < A.tile_lvl[t + 1]; l++) {
            for (int p = A.lvl_ptr[l] + (int)threadIdx.x; p < A.lvl_ptr[l + 1]; p += blockDim.x) {
                const int r = p - p0;
                const int b = srow[r], e = srow[r + 1], nd = sdg[r], lo = slof[r];
                for (int q = 0; q < nd; q++) {
                    const int jl = b + q;  // this L entry
                    const int dk = sdep[lo + q];
                    if (dk >= 0) {  // row k in the box
                        const int kb = srow[dk], ke = srow[dk + 1], kd = kb + sdg[dk];
                        double piv = sv[kd];
                        if (fabs(piv) < 1e-20) piv = 1e-20;  // no-op: row k clamped its own pivot
                        const double lij = sv[jl] / piv;
                        sv[jl] = lij;
                        int sub = kd;
                        for (int jj = jl + 1; jj < e; jj++) {
                            const int kk = sc[jj];
                            while (sub < ke && sc[sub] < kk) sub++;
                            if (sub < ke) {
                                if (sc[sub] == kk) {
                                    const double tt = lij * sv[sub];
                                    sv[jj] = sv[jj] - tt;
                                }
                            } else
                                break;
                        }
                    } else {  // a halo row: final values in global memory
                        const int k = sc[jl];
                        const int ukp = __ldg(A.uptr + k), kend = __ldg(A.rp + k + 1);
                        double piv = __ldcg(A.luv + ukp);
                        const int ulen = kend - ukp - 1;  // upper entries after the diagonal
                        int uc[ILU_HALO_U];
                        double uv[ILU_HALO_U];
#pragma unroll
                        for (int w = 0; w < ILU_HALO_U; w++) {
                            uc[w] = w < ulen ? __ldg(A.ci + ukp + 1 + w) : 0x7fffffff;
                            uv[w] = w < ulen ? __ldcg(A.luv + ukp + 1 + w) : 0.0;
                        }
                        if (fabs(piv) < 1e-20) piv = 1e-20;
                        const double lij = sv[jl] / piv;
                        sv[jl] = lij;
                        if (ulen <= ILU_HALO_U) {
                            // row k's upper columns are distinct and sorted, as
                            // are row i's later columns: subtracting at every
                            // matching column is the two-pointer merge's update
                            for (int jj = jl + 1; jj < e; jj++) {
                                const int kk = sc[jj];
#pragma unroll
                                for (int w = 0; w < ILU_HALO_U; w++) {
                                    if (uc[w] == kk) {
                                        const double tt = lij * uv[w];
                                        sv[jj] = sv[jj] - tt;
                                    }
                                }
                            }
                        } else {
                            int sub = ukp;
                            for (int jj = jl + 1; jj < e; jj++) {
                                const int kk = sc[jj];
                                while (sub < kend && __ldg(A.ci + sub) < kk) sub++;
                                if (sub < kend) {
                                    if (__ldg(A.ci + sub) == kk) {
                                        const double tt = lij * __ldcg(A.luv + sub);
                                        sv[jj] = sv[jj] - tt;
                                    }
                                } else
                                    break;
                            }
                        }
                    }
                }
                if (fabs(sv[b + nd]) < 1e-20) sv[b + nd] = 1e-20;
            }
            __syncthreads();
        }
        for (int e0 = threadIdx.x; e0 < E; e0 += blockDim.x * ILU_STAGE_U) {
            int jv[ILU_STAGE_U];
#pragma unroll
            for (int u = 0; u < ILU_STAGE_U; u++) {
                const int e = e0 + u * (int)blockDim.x;
                jv[u] = e < E ? __ldg(A.ent + eb + e) : -1;
            }
#pragma unroll
            for (int u = 0; u < ILU_STAGE_U; u++)
                if (jv[u] >= 0) A.luv[jv[u]] = sv[e0 + u * (int)blockDim.x];
        }
        __threadfence();
        __syncthreads();
        for (int r = threadIdx.x; r < rows; r += blockDim.x) st_release(A.flag + A.perm[p0 + r], A.epoch);
    }
}

// ---------------------------------------------------------------- IC(0)
// hip/Precond/ic0.cpp:4-70 (initLByA + ic0_fact, Precond_ic0 defaults
// smallnum = droptol = 1e-4) on A's lower part, in place in A's layout: at
// the end entry (i, j<i) holds l_ij and the diagonal 1 / l_ii.
// tnorm_i = droptol * ||row i of A|| (the pivot replacement scale).
static __global__ void k_ic0_tnorm(int n, const int *__restrict__ rp, const double *__restrict__ v, double droptol,
                            double *__restrict__ tnorm)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double t = 0.0;
        for (int k = rp[i]; k < rp[i + 1]; k++) t += v[k] * v[k];
        t = sqrt(t);
        tnorm[i] = t * droptol;
    }
}

// One thread per row, rows in L's level order, persistent CTAs taking
// 128-row tickets as k_ilu0_rows.  Row i waits for each row c of its lower
// part (acquire of c's epoch flag), then l_ij = (a_ij - sum_k l_ik l_ck) *
// (1 / l_cc) with the reference's walk of row c (a column index that only
// moves forward), then l_ii = sqrt(a_ii - sum_j l_ij^2) (a pivot under 1e-20
// replaced by smallnum / droptol * tnorm_i + tnorm_i) stored inverted; the
// operations and their order are the reference's, so the factor is bitwise
// the same.
static __global__ void __launch_bounds__(128) k_ic0_rows(int n, const int *__restrict__ rp, const int *__restrict__ ci,
                                                 const int *__restrict__ uptr, const int *__restrict__ perm,
                                                 const double *__restrict__ tnorm, double smallnum, double droptol,
                                                 double *luv, int *flag, int epoch, int *err, unsigned *ticket,
                                                 int backoff_ns)
{
    __shared__ int s_blk;
    const int ntk = (n + 127) / 128;
    while (true) {
        if (threadIdx.x == 0) {
            const unsigned t = atomicAdd(ticket, 1u);
            // every CTA ends with one failing claim; the last of them re-arms
            if (t == (unsigned)(ntk + gridDim.x - 1)) *ticket = 0u;
            s_blk = (int)t;
        }
        __syncthreads();
        const int blk = s_blk;
        __syncthreads();
        if (blk >= ntk) return;
        const int p = blk * 128 + (int)threadIdx.x;
        if (p >= n) continue;
        if (*(volatile int *)err) continue;
        const int i = perm[p];
        const int rs = rp[i], dl = uptr[i];
        bool ok = true;
        for (int j = rs; j < dl && ok; j++) {
            const int c = ci[j];
            long spins = 0;
            unsigned long long t0 = 0;
            unsigned ns = 32;
            while (ld_acquire(flag + c) != epoch) {
                __nanosleep(ns);  // yield point: the producer may be a lane of this warp
                if (ns < (unsigned)backoff_ns) ns <<= 1;
                if ((++spins & 63) == 0) {
                    const unsigned long long t = gtimer();
                    if (t0 == 0) t0 = t;
                    else if (t - t0 > WAIT_LIMIT_NS) {
                        atomicOr(err, DEV_FACTOR_TIMEOUT);
                        ok = false;
                        break;
                    }
                    if (*(volatile int *)err) {
                        ok = false;
                        break;
                    }
                }
            }
            if (!ok) break;
            int idxu = rp[c];
            const int du = uptr[c];
            double a = luv[j];
            for (int k = rs; k < j; k++) {
                const int ck = ci[k];
                for (int q = idxu; q < du; q++) {
                    const int cq = __ldg(ci + q);
                    if (cq == ck) {
                        const double t = luv[k] * __ldcg(luv + q);
                        a = a - t;
                    } else if (cq > ck) {
                        idxu = q;
                        break;
                    }
                }
            }
            a = a * __ldcg(luv + du);
            luv[j] = a;
        }
        if (!ok) continue;
        double d = luv[dl];
        for (int j = rs; j < dl; j++) {
            const double t = luv[j] * luv[j];
            d = d - t;
        }
        d = sqrt(d);
        if (fabs(d) < 1e-20) d = smallnum / droptol * tnorm[i] + tnorm[i];
        luv[dl] = 1 / d;
        __threadfence();
        st_release(flag + i, epoch);
    }
}

// HostMatrixCSR::seqic0 (hip/HostMatrix/HostMatrixCSR.cpp:269-326): the
// IC(0) factor as the seqilu0 values of the LU solve, in A's layout:
// lower (i, j): l_ij * d_j; diagonal: d_i * d_i; upper (i, j): the lower
// entry (j, i) (position tpos[k]) times d_i, with d the stored 1 / l_ii.
static __global__ void k_ic0_split(long nnz, const int *__restrict__ rowof, const int *__restrict__ ci,
                            const int *__restrict__ uptr, const int *__restrict__ tpos, const double *__restrict__ luv,
                            double *__restrict__ fv)
{
    for (long k = blockIdx.x * (long)blockDim.x + threadIdx.x; k < nnz; k += (long)gridDim.x * blockDim.x) {
        const int i = rowof[k], j = ci[k];
        if (j < i) fv[k] = luv[k] * luv[uptr[j]];
        else if (j == i) fv[k] = luv[k] * luv[k];
        else fv[k] = luv[tpos[k]] * luv[uptr[i]];
    }
}

// one synchronous ParILU sweep over A's nonzeros
//   rowof[k]  row of entry k;  uptr[i] diagonal position of row i
//   ucp/ucpos: upper part by columns: for column j, positions ucpos[ucp[j]..ucp[j+1])
//              of the entries (r, j) with r <= j, rows ascending (diagonal last)
static __global__ void k_parilu_sweep(long nnz, const int *__restrict__ rp, const int *__restrict__ ci,
                               const int *__restrict__ rowof, const int *__restrict__ uptr, const int *__restrict__ ucp,
                               const int *__restrict__ ucpos, const double *__restrict__ a, const double *__restrict__ cur,
                               double *__restrict__ nxt)
{
    for (long k = blockIdx.x * (long)blockDim.x + threadIdx.x; k < nnz; k += (long)gridDim.x * blockDim.x) {
        const int i = rowof[k], j = ci[k];
        double s = a[k], sp = 0.0;
        int il = rp[i];
        const int ilend = uptr[i] + 1;  // position uptr[i] stands for L's unit diagonal
        int iu = ucp[j];
        const int iuend = ucp[j + 1];
        while (il < ilend && iu < iuend) {
            sp = 0.0;
            const int jl = ci[il];
            const int upos = ucpos[iu];
            const int ju = rowof[upos];
            const double lval = (il == uptr[i]) ? 1.0 : cur[il];
            const double uval = cur[upos];
            sp = (jl == ju) ? lval * uval : sp;
            s = (jl == ju) ? s - sp : s;
            il = (jl <= ju) ? il + 1 : il;
            iu = (jl >= ju) ? iu + 1 : iu;
        }
        s += sp;  // undo the last subtraction (the k = min(i,j) term)
        double out;
        if (i > j) {
            double t = cur[uptr[j]];
            if (fabs(t) < 1e-10) t = (t >= 0 ? 1e-10 : -1e-10);
            t = s / t;
            out = isfinite(t) ? t : cur[k];
        } else {
            if (i == j && fabs(s) < 1e-10) s = (s >= 0 ? 1e-10 : -1e-10);
            out = isfinite(s) ? s : cur[k];
        }
        nxt[k] = out;
    }
}

// combined LU values -> seqilu0 layout (in place into fv)
static __global__ void k_split_lu(int n, const int *__restrict__ rp, const int *__restrict__ ci, const int *__restrict__ uptr,
                           const double *__restrict__ luv, double *__restrict__ fv)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int up = uptr[i];
        const double dinv = 1 / luv[up];
        for (int k = rp[i]; k < up; k++) fv[k] = luv[k];
        fv[up] = dinv;
        for (int k = up + 1; k < rp[i + 1]; k++) fv[k] = luv[k] * dinv;
    }
}

// Jacobi: dinv_i = 1/(a_ii + 1e-20) (intel/HostMatrix.h:127-137)
template <typename DT>
__global__ void k_jacobi_init(int n, const int *__restrict__ uptr, const double *__restrict__ a, DT *dinv)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const double t = a[uptr[i]] + 1e-20;
        dinv[i] = (DT)(1.0 / t);
    }
}

}  // namespace xs
