// Tile-scheduled exact triangular solves for matrices on structured grids.
//
// Replaces, for stencil-like patterns, the level-ordered sync-free solve
// (k_trsv_syncfree) that stands in for the reference's
// Lcsr_trsv_sync_free / Ucsc_trsv_sync_free (hip/Precond/gpuparilu.cpp:
// 257-364).  On a natural-order 3D grid the row dependency chain is
// hundreds of levels deep (382 at 128^3 for the 7-point stencil), and a
// row-per-thread solve pays one cross-SM hand-off (a store reaching L2, a
// poll seeing it) per level.  Here one CTA owns a compact box of the grid (a
// "tile") and resolves every dependency inside the box in shared memory,
// with a block barrier between the box's internal levels; only the values
// the box reads from earlier boxes (its "halo") cross SMs, once per box.
//
// Grid detection (host, from the triangle's pattern alone): find nx, ny, nz
// with n = nx*ny*nz such that, with row q at (q % nx, q/nx % ny, q/(nx*ny)),
// every dependency lies within 8 grid steps in each direction (for the
// upper triangle q is the reversed row index n-1-row, so dependencies again
// point to smaller q).  The dependency vectors d = coord(dep) - coord(row)
// are then sheared, x' = x + a*y + b*z, y' = y + c*z, z' = z, with small
// (a, b, c) that make every component of every d' <= 0 (7-point: no shear;
// 27-point: (1, 2, 1); ParILUT fill of the 27-point operator reaches further
// and needs a larger shear).  Boxes of the sheared grid then depend
// only on boxes with smaller or equal coordinates, so ordering boxes by
// wavefront (sum of box coordinates) is a topological order.  A pattern that
// fits no grid keeps the level-ordered solve.
//
// Kernel: persistent CTAs take boxes in that order from a ticket counter (a
// CTA only waits on boxes taken earlier, by running CTAs: forward progress
// without co-residency).  A CTA first loads the data of its first rows,
// then polls its halo values (the NaN sentinel of the solve buffer marks a
// value not yet published, as in the level-ordered kernel; every wait is
// bounded) into shared memory, then walks the box's internal levels: each
// row's dependencies are shared-memory slots, its entries are summed in the
// same order with the same operations as the CPU reference's LUsolve
// (hip/HostMatrix/HostMatrixCSR.cpp:385-409), so FP64 results are bitwise
// identical to the level-ordered solve and to the oracle.
#pragma once
#include <algorithm>
#include <climits>
#include <atomic>
#include <cstring>
#include <thread>
#include <vector>
#include "xs_internal.cuh"

namespace xs {

// fn(i) for i in [0, count) on up to 16 host threads, chunks of `chunk`
// handed out in order from a shared counter (fn must only write data that
// belongs to its own i)
template <typename F>
inline void host_parallel_for(long count, long chunk, F fn)
{
    const int hc = (int)std::max(1u, std::thread::hardware_concurrency());
    const int T = (int)std::max(1L, std::min<long>(std::min(hc, 16), count / std::max(1L, chunk)));
    if (T == 1) {
        for (long i = 0; i < count; i++) fn(i);
        return;
    }
    std::atomic<long> next(0);
    auto work = [&]() {
        while (true) {
            const long i0 = next.fetch_add(chunk);
            if (i0 >= count) return;
            const long i1 = std::min(count, i0 + chunk);
            for (long i = i0; i < i1; i++) fn(i);
        }
    };
    std::vector<std::thread> th;
    for (int t = 1; t < T; t++) th.emplace_back(work);
    work();
    for (auto &x : th) x.join();
}

// Tile sizes (in sheared grid steps) and when tiles are used: triangles
// with at least min_rows rows whose pattern fits a grid.  Process-wide;
// fixed when a preconditioner's triangles are analysed.
struct TileTuning {
    int enable = 1;
    int tx = 16, ty = 16, tz = 8;
    int min_rows = 65536;
    int blocks_per_sm = 4;
    int user_box = 0;  // tx/ty/tz set by the caller (xs_set_trsv_tiles, XS_TRSV_TILES): no dense-row default
};
// Triangles with at least this many entries per row on average start from
// TILE_DENSE_BOX boxes instead of tx/ty/tz: small boxes, long along x, four
// resident per SM.  Measured on the 160^3 27-point ParILUT factors (about
// 27 entries per row): GMRES(30) solve 222 ms with 8x4x2 boxes against
// 294 ms with the 8x8x8 boxes the size-only shrink reached; 8x2x2 239,
// 8x4x4 243, 16x8x4 248, 16x4x2 275, 32x4x4 349, 4x8x8 407 ms.  Sparse
// rows (7-point ILU(0), 3 per row) keep 16x16x8: 0.45 ms per triangle
// against 0.51-0.57 ms with 8x8x8 or 16x8x8.
constexpr double TILE_DENSE_ROW = 20.0;
constexpr int TILE_DENSE_BOX[3] = {8, 4, 2};
TileTuning &tile_tuning();

constexpr int TILE_THREADS = 256;
constexpr int TILE_PF = 8;  // entries of a row held in registers ahead of its level
constexpr int TILE_REACH_MAX = 8;  // largest grid step of a dependency in any direction
constexpr size_t TILE_SMEM_MAX = 200 * 1024;

// an allocator whose resize leaves the elements uninitialised (arrays that
// are written in full afterwards, by several threads: no serial zero fill)
template <typename T>
struct UninitAlloc : std::allocator<T> {
    template <typename U>
    struct rebind {
        using other = UninitAlloc<U>;
    };
    UninitAlloc() = default;
    template <typename U>
    UninitAlloc(const UninitAlloc<U> &) noexcept
    {
    }
    template <typename U>
    void construct(U *p) noexcept
    {
        ::new ((void *)p) U;
    }
    template <typename U, typename... A>
    void construct(U *p, A &&...a)
    {
        ::new ((void *)p) U(std::forward<A>(a)...);
    }
};
template <typename T>
using HostArray = std::vector<T, UninitAlloc<T>>;

struct TileHostPlan {
    int n = 0, ntiles = 0, max_rows = 0, max_halo = 0, max_entries = 0;
    int nx = 0, ny = 0, nz = 0, sa = 0, sb = 0, sc = 0;
    std::vector<int> perm, prp, tile_pos, tile_lvl, lvl_ptr, halo_ptr, halo_row;
    HostArray<int> pci;   // every entry written by the layout (entries = true)
    HostArray<long> src;
    // entries = false: what a device pass needs to write pci/src itself
    HostArray<int> tile_of;  // by logical index (row, or n-1-row for U): the row's box
    std::vector<int> pos_of;  // by row: its position
};

// ---------------------------------------------------------------- grid fit
struct GridCoord {
    long nx, nxy;
    void of(long q, int &x, int &y, int &z) const
    {
        z = (int)(q / nxy);
        const long r = q - (long)z * nxy;
        y = (int)(r / nx);
        x = (int)(r - (long)y * nx);
    }
};

// balanced digits of an offset o = dx + dy*nx + dz*nxy with |d| small
inline bool offset_fits(long o, long nx, long nxy, int reach)
{
    const long dz = (o + (o >= 0 ? nxy / 2 : -nxy / 2)) / nxy;
    const long r = o - dz * nxy;
    const long dy = (r + (r >= 0 ? nx / 2 : -nx / 2)) / nx;
    const long dx = r - dy * nx;
    return std::labs(dz) <= reach && std::labs(dy) <= reach && std::labs(dx) <= reach;
}

// Largest coordinate step of any dependency under (nx, nxy), or reach+1 as
// soon as one exceeds reach; the distinct dependency vectors go to vecs.
// logical(r) maps a row to its logical index (dependencies at smaller ones).
template <typename LogF>
inline int grid_reach(int n, const int *rp, const int *ci, LogF logical, const GridCoord &g, int reach,
                      std::vector<int> &vecs, int row_step = 1)
{
    const int W = 2 * reach + 1;
    const long RB = 65536L * row_step;  // rows per work item
    const long items = (n + RB - 1) / RB;
    std::vector<int> worst_of(items, 0);
    std::vector<std::vector<char>> seen_of(items);
    std::atomic<int> over(0);
    host_parallel_for(items, 1, [&](long it) {
        std::vector<char> seen((size_t)W * W * W, 0);
        int worst = 0;
        const int r0 = (int)(it * RB), r1 = (int)std::min<long>(n, r0 + RB);
        for (int r = r0; r < r1 && !over.load(std::memory_order_relaxed); r += row_step) {
            int xi, yi, zi;
            g.of(logical(r), xi, yi, zi);
            for (int k = rp[r]; k < rp[r + 1]; k++) {
                int xj, yj, zj;
                g.of(logical(ci[k]), xj, yj, zj);
                const int dx = xj - xi, dy = yj - yi, dz = zj - zi;
                const int m = std::max(std::abs(dx), std::max(std::abs(dy), std::abs(dz)));
                if (m > reach) {
                    over.store(1);
                    return;
                }
                worst = std::max(worst, m);
                seen[((size_t)(dz + reach) * W + (dy + reach)) * W + (dx + reach)] = 1;
            }
        }
        worst_of[it] = worst;
        seen_of[it].swap(seen);
    });
    if (over.load()) return reach + 1;
    int worst = 0;
    std::vector<char> seen((size_t)W * W * W, 0);
    for (long it = 0; it < items; it++) {
        worst = std::max(worst, worst_of[it]);
        for (size_t q = 0; q < seen.size(); q++) seen[q] |= seen_of[it][q];
    }
    vecs.clear();
    for (int z = 0; z < W; z++)
        for (int y = 0; y < W; y++)
            for (int x = 0; x < W; x++)
                if (seen[((size_t)z * W + y) * W + x]) {
                    vecs.push_back(x - reach);
                    vecs.push_back(y - reach);
                    vecs.push_back(z - reach);
                }
    return worst;
}

// The grid a strict triangle's pattern lives on and the shear that makes
// every dependency vector non-positive (the first half of the analysis; it
// does not depend on the box dimensions).
struct TileGrid {
    GridCoord g{0, 0};
    int nx = 0, ny = 0, nz = 0, sa = 0, sb = 0, sc = 0;
};

inline bool tile_detect(int n, const int *rp, const int *ci, bool upper, TileGrid &G)
{
    const long nnz = rp[n];
    if (n < 8 || nnz == 0) return false;
    auto logical = [&](int r) -> long { return upper ? (long)n - 1 - r : (long)r; };
    // distinct offsets |row - dep| of a sample of rows (give up beyond 512
    // of them); a grid chosen from them is checked on every entry below
    const int step = std::max(1, n / 16384);
    std::vector<long> offs;
    {
        const int TAB = 2048;
        std::vector<long> tab(TAB, -1);
        int cnt = 0;
        for (int r = 0; r < n && cnt <= 512; r += step)
            for (int k = rp[r]; k < rp[r + 1]; k++) {
                const long o = std::labs((long)ci[k] - r);
                unsigned hsh = (unsigned)((o * 2654435761ul) % TAB);
                while (tab[hsh] != -1 && tab[hsh] != o) hsh = (hsh + 1) % TAB;
                if (tab[hsh] == -1) {
                    tab[hsh] = o;
                    offs.push_back(o);
                    if (++cnt > 512) break;
                }
            }
        if (cnt > 512) return false;
    }
    std::sort(offs.begin(), offs.end());
    // try growing reaches: a dependency may lie up to R grid steps away in
    // each direction (ParILUT fill reaches several steps along x)
    int best_reach = TILE_REACH_MAX + 1;
    GridCoord g{0, 0};
    std::vector<int> vecs, v;
    for (int R = 2; R <= TILE_REACH_MAX && best_reach > TILE_REACH_MAX; R *= 2) {
        // the smallest offset beyond a pure x step lies within R of nx
        long o_y = -1;
        for (long o : offs)
            if (o > R) { o_y = o; break; }
        if (o_y < 0) return false;  // a band of width <= R: nothing to gain
        struct Cand { long nx, nxy; };
        std::vector<Cand> cands;
        for (long nx = std::max<long>(2 * R + 1, o_y - R); nx <= o_y + R; nx++) {
            if (n % nx) continue;
            long o_z = -1;
            for (long o : offs)
                if (o > R * nx + R) { o_z = o; break; }
            std::vector<long> nxys;
            if (o_z < 0) nxys.push_back(n);  // no step beyond y: a 2D grid
            else
                for (long dy = -R; dy <= R; dy++)
                    for (long dx = -R; dx <= R; dx++) nxys.push_back(o_z - dy * nx - dx);
            for (long nxy : nxys) {
                if (nxy <= nx || nxy % nx || n % nxy) continue;
                if (nxy < n && nxy / nx <= 2 * R) continue;  // y extent too small to tell y from z steps
                bool ok = true;
                for (long o : offs)
                    if (!offset_fits(o, nx, nxy, R)) { ok = false; break; }
                if (ok) cands.push_back({nx, nxy});
            }
        }
        // rank the candidates on the sampled rows, then check the best ones
        // on every entry
        std::vector<std::pair<int, int>> rank;  // (sampled reach, candidate)
        for (int q = 0; q < (int)cands.size(); q++) {
            const GridCoord gc{cands[q].nx, cands[q].nxy};
            const int r = grid_reach(n, rp, ci, logical, gc, R, v, step);
            if (r <= R) rank.push_back({r, q});
        }
        std::sort(rank.begin(), rank.end());
        for (const auto &rq : rank) {
            const GridCoord gc{cands[rq.second].nx, cands[rq.second].nxy};
            const int r = grid_reach(n, rp, ci, logical, gc, R, v);
            if (r <= R && r < best_reach) {
                best_reach = r;
                g = gc;
                vecs = v;
                break;
            }
        }
    }
    if (best_reach > TILE_REACH_MAX) return false;
    // a shear making every dependency vector non-positive, component by
    // component: c from the vectors that step down in z, then a from those
    // that stay in their z plane and step down in y, then b (for a fixed a)
    // from the z steps; each the smallest that works.  Every dependency is
    // lexicographically smaller in (z, y, x), so such a shear always exists.
    auto ceil_div = [](int a, int b) { return a >= 0 ? (a + b - 1) / b : -((-a) / b); };  // b > 0
    int sa = 0, sb = 0, sc = 0;
    for (size_t q = 0; q < vecs.size(); q += 3) {
        const int dx = vecs[q], dy = vecs[q + 1], dz = vecs[q + 2];
        if (dz > 0 || (dz == 0 && dy > 0) || (dz == 0 && dy == 0 && dx >= 0)) return false;
        if (dz < 0) sc = std::max(sc, ceil_div(dy, -dz));
        else if (dy < 0) sa = std::max(sa, ceil_div(dx, -dy));
    }
    for (size_t q = 0; q < vecs.size(); q += 3) {
        const int dx = vecs[q], dy = vecs[q + 1], dz = vecs[q + 2];
        if (dz < 0) sb = std::max(sb, ceil_div(dx + sa * dy, -dz));
    }
    G.g = g;
    G.nx = (int)g.nx;
    G.ny = (int)(g.nxy / g.nx);
    G.nz = (int)(n / g.nxy);
    G.sa = sa; G.sb = sb; G.sc = sc;
    return true;
}

// Box layout of a strict triangle on a detected grid (the second half).
template <typename SrcF>
inline bool tile_layout(int n, const int *rp, const int *ci, bool upper, SrcF src_of, const TileGrid &G,
                        const TileTuning &tt, TileHostPlan &h, bool entries = true)
{
    const long nnz = rp[n];
    auto logical = [&](int r) -> long { return upper ? (long)n - 1 - r : (long)r; };
    const GridCoord g = G.g;
    const int sa = G.sa, sb = G.sb, sc = G.sc;
    h.n = n;
    h.nx = G.nx;
    h.ny = G.ny;
    h.nz = G.nz;
    h.sa = sa; h.sb = sb; h.sc = sc;
    // tile coordinates of every logical index
    const int tx = std::max(1, tt.tx), ty = std::max(1, tt.ty), tz = std::max(1, tt.tz);
    const long X = (long)(h.nx - 1) + (long)sa * (h.ny - 1) + (long)sb * (h.nz - 1) + 1;
    const long Y = (long)(h.ny - 1) + (long)sc * (h.nz - 1) + 1;
    const long Z = h.nz;
    const long ntx = (X + tx - 1) / tx, nty = (Y + ty - 1) / ty, ntz = (Z + tz - 1) / tz;
    if (ntx * nty * ntz > (1L << 26)) return false;
    HostArray<int> tile_of(n);  // by logical index: box id in the sheared box grid
    std::vector<int> cnt((size_t)(ntx * nty * ntz), 0);
    host_parallel_for((n + 65535) / 65536, 1, [&](long b) {
        const long q1 = std::min<long>(n, (b + 1) * 65536);
        for (long q = b * 65536; q < q1; q++) {
            int x, y, z;
            g.of(q, x, y, z);
            const long xs = x + (long)sa * y + (long)sb * z, ys = y + (long)sc * z;
            tile_of[q] = (int)(((long)(z / tz) * nty + ys / ty) * ntx + xs / tx);
        }
    });
    for (long q = 0; q < n; q++) cnt[tile_of[q]]++;
    // order the non-empty boxes by wavefront, then z, y, x
    std::vector<std::pair<long, int>> order;
    for (long id = 0; id < (long)cnt.size(); id++) {
        if (!cnt[id]) continue;
        const long bx = id % ntx, by = (id / ntx) % nty, bz = id / (ntx * nty);
        order.push_back({((bx + by + bz) << 40) | id, (int)id});
    }
    std::sort(order.begin(), order.end());
    h.ntiles = (int)order.size();
    std::vector<int> rank_of(cnt.size(), -1);
    for (int t = 0; t < h.ntiles; t++) rank_of[order[t].second] = t;
    // rows of each box in increasing logical index (a topological order)
    std::vector<int> start(h.ntiles + 1, 0);
    for (int t = 0; t < h.ntiles; t++) start[t + 1] = start[t] + cnt[order[t].second];
    std::vector<int> byq(n);
    {
        std::vector<int> fill(start.begin(), start.end() - 1);
        for (long q = 0; q < n; q++) {
            const int t = rank_of[tile_of[q]];
            tile_of[q] = t;  // from here on: the box's rank
            byq[fill[t]++] = (int)q;
        }
    }
    // local levels, then positions: box-major, level-major, logical index
    // (boxes are independent here: in parallel, each writing its own ranges)
    std::vector<int> lev(n, 0);  // by logical index
    auto row_of = [&](long q) -> int { return upper ? (int)(n - 1 - q) : (int)q; };
    h.perm.assign(n, 0);
    h.tile_pos.assign(start.begin(), start.end());
    h.tile_lvl.assign(h.ntiles + 1, 0);
    std::vector<int> nlev(h.ntiles, 0);
    host_parallel_for(h.ntiles, 16, [&](long t) {
        int maxl = 0;
        for (int k = start[t]; k < start[t + 1]; k++) {
            const long q = byq[k];
            const int r = row_of(q);
            int l = 0;
            for (int e = rp[r]; e < rp[r + 1]; e++) {
                const long qd = logical(ci[e]);
                if (tile_of[qd] == t) l = std::max(l, lev[qd] + 1);
            }
            lev[q] = l;
            maxl = std::max(maxl, l);
        }
        nlev[t] = maxl + 1;
    });
    for (int t = 0; t < h.ntiles; t++) {
        h.tile_lvl[t + 1] = h.tile_lvl[t] + nlev[t];
        h.max_rows = std::max(h.max_rows, start[t + 1] - start[t]);
    }
    h.lvl_ptr.assign(h.tile_lvl[h.ntiles] + 1, 0);
    std::vector<int> pos_of(n);  // by row
    host_parallel_for(h.ntiles, 16, [&](long t) {
        const int nl = nlev[t], pos = start[t];
        std::vector<int> lcnt(nl + 1, 0);
        for (int k = start[t]; k < start[t + 1]; k++) lcnt[lev[byq[k]] + 1]++;
        for (int l = 0; l < nl; l++) lcnt[l + 1] += lcnt[l];
        for (int l = 0; l < nl; l++) h.lvl_ptr[h.tile_lvl[t] + l] = pos + lcnt[l];
        for (int k = start[t]; k < start[t + 1]; k++) {
            const long q = byq[k];
            const int p = pos + lcnt[lev[q]]++;
            h.perm[p] = row_of(q);
            pos_of[row_of(q)] = p;
        }
    });
    h.lvl_ptr[h.tile_lvl[h.ntiles]] = n;
    // entries in accumulation order; dependencies as shared-memory slots:
    // [0, rows) the box's own rows by position, then the box's halo
    h.prp.assign(n + 1, 0);
    for (int p = 0; p < n; p++) {
        const int r = h.perm[p];
        h.prp[p + 1] = h.prp[p] + (rp[r + 1] - rp[r]);
    }
    if (entries) {
        h.pci.resize(nnz);  // written in full below (each box its rows' entries)
        h.src.resize(nnz);
    }
    h.halo_ptr.assign(h.ntiles + 1, 0);
    std::vector<std::vector<int>> ext_of(h.ntiles);
    host_parallel_for(h.ntiles, 16, [&](long t) {
        const int p0 = h.tile_pos[t], p1 = h.tile_pos[t + 1], rows = p1 - p0;
        std::vector<int> &ext = ext_of[t];
        int lo = INT_MAX, hi = -1;
        for (int p = p0; p < p1; p++) {
            const int r = h.perm[p];
            for (int e = rp[r]; e < rp[r + 1]; e++)
                if (tile_of[logical(ci[e])] != t) {
                    ext.push_back(ci[e]);
                    lo = std::min(lo, ci[e]);
                    hi = std::max(hi, ci[e]);
                }
        }
        // sorted, without duplicates: through a bitmap over [lo, hi] when
        // that window is narrow against the list, else by sorting
        const long words = hi >= lo ? ((long)hi - lo) / 64 + 1 : 0;
        if (words > 0 && words <= 8 * (long)ext.size() + 64) {
            thread_local std::vector<unsigned long long> bm;
            bm.assign(words, 0ull);
            for (int d : ext) bm[(d - lo) >> 6] |= 1ull << ((d - lo) & 63);
            ext.clear();
            for (long w = 0; w < words; w++)
                for (unsigned long long x = bm[w]; x; x &= x - 1)
                    ext.push_back(lo + (int)(w * 64) + __builtin_ctzll(x));
        } else {
            std::sort(ext.begin(), ext.end());
            ext.erase(std::unique(ext.begin(), ext.end()), ext.end());
        }
        if (!entries) return;
        for (int p = p0; p < p1; p++) {
            const int r = h.perm[p];
            int o = h.prp[p];
            auto put = [&](int e) {
                const int d = ci[e];
                if (tile_of[logical(d)] == t) h.pci[o] = pos_of[d] - p0;
                else h.pci[o] = rows + (int)(std::lower_bound(ext.begin(), ext.end(), d) - ext.begin());
                h.src[o] = src_of(e);
                o++;
            };
            if (!upper)
                for (int e = rp[r]; e < rp[r + 1]; e++) put(e);
            else
                for (int e = rp[r + 1] - 1; e >= rp[r]; e--) put(e);
        }
    });
    for (int t = 0; t < h.ntiles; t++) {
        h.halo_ptr[t + 1] = h.halo_ptr[t] + (int)ext_of[t].size();
        h.max_halo = std::max(h.max_halo, (int)ext_of[t].size());
        h.max_entries = std::max(h.max_entries, h.prp[h.tile_pos[t + 1]] - h.prp[h.tile_pos[t]]);
    }
    h.halo_row.resize(std::max(h.halo_ptr[h.ntiles], 0));
    host_parallel_for(h.ntiles, 64, [&](long t) {
        if (!ext_of[t].empty())
            std::memcpy(h.halo_row.data() + h.halo_ptr[t], ext_of[t].data(), sizeof(int) * ext_of[t].size());
    });
    if (!entries) {
        h.tile_of = std::move(tile_of);
        h.pos_of = std::move(pos_of);
    }
    return true;
}

// The entries of a box layout in accumulation order, one thread per
// position: the same slots tile_layout writes on the host (a dependency in
// the row's own box: its position minus the box's first; otherwise the box's
// row count plus its index in the box's sorted halo list) and each entry's
// value source (src_nat of the natural entry).  Inputs from tile_layout with
// entries = false; rp/ci/src_nat the natural CSR on the device.
template <bool UPPER>
__global__ void k_tile_entries(int n, const int *__restrict__ perm, const int *__restrict__ prp,
                               const int *__restrict__ rp, const int *__restrict__ ci,
                               const long *__restrict__ src_nat, const int *__restrict__ tile_of,
                               const int *__restrict__ pos_of, const int *__restrict__ tile_pos,
                               const int *__restrict__ halo_ptr, const int *__restrict__ halo_row, int *__restrict__ pci,
                               long *__restrict__ src)
{
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
        const int r = perm[p];
        const int t = tile_of[UPPER ? n - 1 - r : r];
        const int p0 = tile_pos[t], rows = tile_pos[t + 1] - p0;
        const int h0 = halo_ptr[t], nh = halo_ptr[t + 1] - h0;
        const int e0 = rp[r], e1 = rp[r + 1];
        long o = prp[p];
        for (int j = 0; j < e1 - e0; j++, o++) {
            const int e = UPPER ? e1 - 1 - j : e0 + j;
            const int d = ci[e];
            int slot;
            if (tile_of[UPPER ? n - 1 - d : d] == t) {
                slot = pos_of[d] - p0;
            } else {  // first halo index whose row is >= d (the row is in the list)
                int lo = 0, hi = nh;
                while (lo < hi) {
                    const int mid = (lo + hi) >> 1;
                    if (halo_row[h0 + mid] < d) lo = mid + 1;
                    else hi = mid;
                }
                slot = rows + lo;
            }
            pci[o] = slot;
            src[o] = src_nat[e];
        }
    }
}

// Tile layout of a strict triangle (both halves, the given box dimensions); false when the pattern fits no grid
// (the caller then keeps the level-ordered layout).  rp/ci: natural CSR of
// the strict triangle, 0-based; upper: dependencies on larger rows, entries
// summed in decreasing column order; src_of(k) maps entry k to the index of
// its value.
template <typename SrcF>
inline bool tri_analyse_tiles(int n, const int *rp, const int *ci, bool upper, SrcF src_of, const TileTuning &tt,
                              TileHostPlan &h)
{
    TileGrid G;
    return tile_detect(n, rp, ci, upper, G) && tile_layout(n, rp, ci, upper, src_of, G, tt, h);
}

// ---------------------------------------------------------------- kernel
template <typename FT>
struct TileArgs {
    int n, ntiles;
    const int *tile_pos;  // ntiles + 1: first position of each box
    const int *tile_lvl;  // ntiles + 1: first internal level of each box (index into lvl_ptr)
    const int *lvl_ptr;   // first position of each internal level (+ n at the end)
    const int *halo_ptr;  // ntiles + 1
    const int *halo_row;  // rows of earlier boxes that a box reads
    const int *perm;      // position -> row
    const int *prp;       // position row pointer
    const int *pci;       // shared-memory slot of each dependency
    const FT *pv;         // entry values (the array is padded by at least 4 bytes)
    int max_rows, max_halo, max_entries;
};

// shared-memory layout of one box (byte offsets; every part 16-byte aligned)
struct TileSmem {
    size_t y, rhs, dinv, pv, row, eptr, pci, total;
    template <typename VT, typename FT, typename DT>
    static __host__ __device__ TileSmem of(int rows, int halo, int entries)
    {
        auto al = [](size_t b) { return (b + 15) & ~(size_t)15; };
        TileSmem m;
        m.y = 0;
        m.rhs = m.y + al((size_t)(rows + halo) * sizeof(VT));
        m.dinv = m.rhs + al((size_t)rows * sizeof(VT));
        m.pv = m.dinv + al((size_t)rows * sizeof(DT));
        m.row = m.pv + al((size_t)entries * sizeof(FT) + 8);  // + the 4-byte rounding of the value range
        m.eptr = m.row + al((size_t)rows * sizeof(int));
        m.pci = m.eptr + al((size_t)(rows + 1) * sizeof(int));
        m.total = m.pci + al((size_t)entries * sizeof(int));
        return m;
    }
};

// 16 bytes global -> shared, bypassing L1 (both addresses 16-byte aligned)
__device__ __forceinline__ void cp_async16(void *dst, const void *src)
{
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async4(void *dst, const void *src)
{
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async8(void *dst, const void *src)
{
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(d), "l"(src) : "memory");
}
template <int B>
__device__ __forceinline__ void cp_async_n(void *dst, const void *src)
{
    if constexpr (B == 8) cp_async8(dst, src);
    else cp_async4(dst, src);
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

// poll one published value (bounded); false on timeout or a recorded error
template <typename VT>
__device__ __forceinline__ bool tile_poll(const VT *p, int *err, int backoff_ns, VT &y)
{
    y = ld_poll(p);
    if (!Sentinel<VT>::is(y)) return true;
    const unsigned long long t0 = gtimer();
    unsigned ns = 8;
    long spins = 0;
    while (Sentinel<VT>::is(y)) {
        __nanosleep(ns);
        if (ns < (unsigned)backoff_ns) ns <<= 1;
        y = ld_poll(p);
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

// A box's data is staged in shared memory before its first level: its rows
// and entry ranges, entry slots and values, and (U) dinv by asynchronous
// copies; then the rows' right-hand sides, gathered through the staged row
// numbers; the halo values are polled while those copies are in flight.
// The internal levels then read shared memory only.
template <typename VT, typename FT, typename DT, bool UPPER>
__global__ void __launch_bounds__(TILE_THREADS) k_trsv_tiles(TileArgs<FT> P, const DT *__restrict__ dinv,
                                                             const VT *rhs, VT *self, VT *out_user, VT *reset_other,
                                                             const int *done_flag, int *err, unsigned *ticket,
                                                             int backoff_ns)
{
    if (done_flag && *done_flag) return;
    extern __shared__ __align__(16) unsigned char tile_smem[];
    const TileSmem L = TileSmem::of<VT, FT, DT>(P.max_rows, P.max_halo, P.max_entries);
    VT *ysh = (VT *)(tile_smem + L.y);
    VT *s_rhs = (VT *)(tile_smem + L.rhs);
    DT *s_dinv = (DT *)(tile_smem + L.dinv);
    unsigned char *s_pv = tile_smem + L.pv;
    int *s_row = (int *)(tile_smem + L.row);
    int *s_eptr = (int *)(tile_smem + L.eptr);
    int *s_pci = (int *)(tile_smem + L.pci);
    __shared__ int s_tile;
    const unsigned last = (unsigned)P.ntiles + gridDim.x - 1;
    const int tid = threadIdx.x;
    bool ok = true;
    while (true) {
        __syncthreads();
        if (tid == 0) {
            const unsigned t = atomicAdd(ticket, 1u);
            if (t == last) *ticket = 0u;  // every CTA has drawn its final ticket
            s_tile = (int)t;
        }
        __syncthreads();
        const int t = s_tile;
        if (t >= P.ntiles) break;
        const int p0 = __ldg(P.tile_pos + t), p1 = __ldg(P.tile_pos + t + 1);
        const int l0 = __ldg(P.tile_lvl + t), l1 = __ldg(P.tile_lvl + t + 1);
        const int h0 = __ldg(P.halo_ptr + t), h1 = __ldg(P.halo_ptr + t + 1);
        const int rows = p1 - p0;
        const int e0 = __ldg(P.prp + p0), e1 = __ldg(P.prp + p1);
        // group 0: row numbers; group 1: entry ranges, slots, values, dinv
        for (int i = tid; i < rows; i += TILE_THREADS) cp_async4(s_row + i, P.perm + p0 + i);
        cp_async_commit();
        for (int i = tid; i <= rows; i += TILE_THREADS) cp_async4(s_eptr + i, P.prp + p0 + i);
        for (int i = tid; i < e1 - e0; i += TILE_THREADS) cp_async4(s_pci + i, P.pci + e0 + i);
        const long vb0 = ((long)e0 * (long)sizeof(FT)) & ~3L, vb1 = ((long)e1 * (long)sizeof(FT) + 3) & ~3L;
        const unsigned char *vsrc = (const unsigned char *)P.pv;
        for (long w = tid; w < (vb1 - vb0) / 4; w += TILE_THREADS) cp_async4(s_pv + 4 * w, vsrc + vb0 + 4 * w);
        if (UPPER)
            for (int i = tid; i < rows; i += TILE_THREADS) cp_async_n<sizeof(DT)>(s_dinv + i, dinv + p0 + i);
        cp_async_commit();
        cp_async_wait<1>();
        __syncthreads();
        // group 2: right-hand sides through the staged row numbers
        for (int i = tid; i < rows; i += TILE_THREADS) cp_async_n<sizeof(VT)>(s_rhs + i, rhs + s_row[i]);
        cp_async_commit();
        for (int k = h0 + tid; k < h1; k += TILE_THREADS) {
            VT y = (VT)0;
            if (ok) ok = tile_poll<VT>(self + __ldg(P.halo_row + k), err, backoff_ns, y);
            ysh[rows + (k - h0)] = y;
        }
        cp_async_wait<0>();
        __syncthreads();
        const FT *pv = (const FT *)(s_pv + ((long)e0 * (long)sizeof(FT) - vb0));
        for (int l = l0; l < l1; l++) {
            const int pa = __ldg(P.lvl_ptr + l) - p0, pb = __ldg(P.lvl_ptr + l + 1) - p0;
            for (int i = pa + tid; i < pb; i += TILE_THREADS) {
                const int row = s_row[i];
                VT acc = UPPER ? (VT)(s_rhs[i] * (VT)s_dinv[i]) : s_rhs[i];
                if (reset_other) reset_other[row] = Sentinel<VT>::value();
                const int k1 = s_eptr[i + 1] - e0;
                for (int k = s_eptr[i] - e0; k < k1; k++) acc = msub(acc, ysh[s_pci[k]], (VT)FVal<FT>::cvt(pv[k]));
                ysh[i] = acc;
                st_publish(self + row, acc);
                if (out_user) out_user[row] = acc;
            }
            __syncthreads();
        }
    }
}

}  // namespace xs
