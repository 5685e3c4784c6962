// Host threshold factorizations (Saad ILUT, ICT): see xs_hostilu.h.
//
// Both are computed with a dense working row that persists across rows (as
// the reference's do), so every value, every drop decision and every tie
// between equal magnitudes comes out as the reference's sequential code
// produces it; this unit is compiled without floating-point contraction.
#include "xs_hostilu.h"

#include <algorithm>
#include <cmath>
#include <functional>
#include <numeric>

namespace xs {
namespace {

// scale of the substitute for a zero pivot, relative to the row's drop
// threshold (hip/Precond/ilut_diag_in_csr.h:7; seqict passes the same
// constant as ICT's smallNum, hip/HostMatrix/HostMatrixCSR.cpp:331)
constexpr double PIVOT_SUBST = 1e-4;

// ---------------------------------------------------------------- ILUT
// std heap order of a row's kept entries (columns into the working row w):
// the entry of smallest magnitude is on top
struct SmallestOnTop {
    const double *w;
    bool operator()(int a, int b) const { return std::fabs(w[a]) > std::fabs(w[b]); }
};

// The top of a kept-entry heap was replaced: sink it.  It moves below a child
// of magnitude <= its own (the smaller child; the left one when the two are
// equal), so an equal magnitude sinks.  This is the rule of the reference's
// replace-top (ilut_diag_in_csr.cpp:2-19) and decides which entries a tie keeps.
void sink_top(int *h, int len, const double *w)
{
    const int top = h[0];
    const double mag = std::fabs(w[top]);
    int hole = 0;
    for (int c = 1; c < len; c = 2 * c + 1) {
        if (c + 1 < len && std::fabs(w[h[c]]) > std::fabs(w[h[c + 1]])) c++;
        if (std::fabs(w[h[c]]) > mag) break;
        h[hole] = h[c];
        hole = c;
    }
    h[hole] = top;
}

// Offer column c of the working row to a kept set of at most cap entries: a
// full set takes it only in place of a top of strictly smaller magnitude,
// which is zeroed in w; a refused entry is zeroed in w.
void offer(int *kept, int &len, int cap, int c, double *w)
{
    if (len < cap) {
        kept[len++] = c;
        std::push_heap(kept, kept + len, SmallestOnTop{w});
    } else if (std::fabs(w[c]) > std::fabs(w[kept[0]])) {
        w[kept[0]] = 0;
        kept[0] = c;
        sink_top(kept, len, w);
    } else {
        w[c] = 0;
    }
}

// Append a row's kept entries in ascending column order and clear them in w.
void flush_kept(int *kept, int len, double *w, std::vector<int> &fc, std::vector<double> &fv)
{
    std::sort(kept, kept + len);
    for (int t = 0; t < len; t++) {
        fc.push_back(kept[t]);
        fv.push_back(w[kept[t]]);
        w[kept[t]] = 0;
    }
}

// ---------------------------------------------------------------- ICT
// Sift entry i of a heap of the first m candidates (smallest magnitude on
// top) down: it moves below a child only when the child is strictly smaller,
// taking the right child only when it is strictly smaller than the left
// (hip/Precond/ict_l.cpp:3-22).
void sift_smallest(double *val, int *col, int i, int m)
{
    const double hv = val[i];
    const int hc = col[i];
    for (int k = 2 * i + 1; k < m; k = 2 * k + 1) {
        if (k + 1 < m && std::fabs(val[k]) > std::fabs(val[k + 1])) k++;
        if (!(std::fabs(val[k]) < std::fabs(hv))) break;
        val[i] = val[k];
        col[i] = col[k];
        i = k;
    }
    val[i] = hv;
    col[i] = hc;
}

// Leave the m candidates of largest magnitude (as the reference's partial
// heap selection of ict_l.cpp:23-39 picks them) in slots [0, m), ordered by
// column.
void keep_largest(double *val, int *col, int m, int cnt)
{
    for (int i = m / 2; i >= 0; i--) sift_smallest(val, col, i, m);
    for (int i = m; i < cnt; i++) {
        if (std::fabs(val[i]) > std::fabs(val[0])) {
            val[0] = val[i];
            col[0] = col[i];
            sift_smallest(val, col, 0, m);
        }
    }
    std::vector<int> ord(m);
    std::iota(ord.begin(), ord.end(), 0);
    std::sort(ord.begin(), ord.end(), [&](int a, int b) { return col[a] < col[b]; });  // columns are distinct
    std::vector<double> tv(m);
    std::vector<int> tc(m);
    for (int t = 0; t < m; t++) {
        tv[t] = val[ord[t]];
        tc[t] = col[ord[t]];
    }
    std::copy(tv.begin(), tv.end(), val);
    std::copy(tc.begin(), tc.end(), col);
}

}  // namespace

void host_ilut(int n, const int *rp, const int *ci, const double *v, int lfil, double droptol, HostTriFactors &F)
{
    std::vector<double> w(n, 0.0), piv(n, 0.0);  // working row; 1/u_kk
    // rows of the combined factor as produced: L entries (the multipliers),
    // u_ii, then U entries, each part in ascending column order
    std::vector<int> fc, fend(n + 1, 0), fdiag(n, 0);
    std::vector<double> fv;
    fc.reserve((size_t)n * (2 * lfil + 1));
    fv.reserve((size_t)n * (2 * lfil + 1));
    std::vector<int> lq, uq;  // pending L columns (a min-heap); U columns in order of first appearance
    std::vector<int> kept(std::max(lfil, 1));
    const std::greater<int> lowest_first;
    for (int i = 0; i < n; i++) {
        lq.clear();
        uq.clear();
        double ss = 0;
        for (int q = rp[i]; q < rp[i + 1]; q++) {
            const int c = ci[q];
            w[c] = v[q];
            ss += v[q] * v[q];
            if (c < i) lq.push_back(c);  // ascending: already a heap
            if (c > i) uq.push_back(c);
        }
        const double thr = std::sqrt(ss) * droptol;
        int nk = 0;
        while (!lq.empty()) {
            const int k = lq.front();
            std::pop_heap(lq.begin(), lq.end(), lowest_first);
            lq.pop_back();
            const double f = w[k] * piv[k];
            if (std::fabs(f) < thr) {
                w[k] = 0;
                continue;
            }
            for (int q = fdiag[k] + 1; q < fend[k + 1]; q++) {
                const int j = fc[q];
                const double old = w[j];
                if (old == 0) {  // an entry of row i appears (or reappears)
                    if (j < i) {
                        lq.push_back(j);
                        std::push_heap(lq.begin(), lq.end(), lowest_first);
                    }
                    if (j > i) uq.push_back(j);
                }
                w[j] = old - f * fv[q];
            }
            w[k] = f;
            offer(kept.data(), nk, lfil, k, w.data());
        }
        flush_kept(kept.data(), nk, w.data(), fc, fv);
        fdiag[i] = (int)fc.size();
        if (w[i] != 0) {
            piv[i] = 1 / w[i];
            fv.push_back(w[i]);
            w[i] = 0;
        } else {
            const double d = PIVOT_SUBST / droptol * thr + thr;
            piv[i] = 1 / d;
            fv.push_back(d);
        }
        fc.push_back(i);
        nk = 0;
        for (const int c : uq) {
            if (std::fabs(w[c]) > thr) offer(kept.data(), nk, lfil, c, w.data());
            else w[c] = 0;
        }
        flush_kept(kept.data(), nk, w.data(), fc, fv);
        fend[i + 1] = (int)fc.size();
    }
    // split: L as produced, U' = U scaled by 1/u_ii, dinv = 1/u_ii
    F.lrp.assign(n + 1, 0);
    F.urp.assign(n + 1, 0);
    F.lci.clear(); F.lv.clear(); F.uci.clear(); F.uv.clear();
    for (int i = 0; i < n; i++) {
        for (int q = fend[i]; q < fdiag[i]; q++) {
            F.lci.push_back(fc[q]);
            F.lv.push_back(fv[q]);
        }
        for (int q = fdiag[i] + 1; q < fend[i + 1]; q++) {
            F.uci.push_back(fc[q]);
            F.uv.push_back(fv[q] * piv[i]);
        }
        F.lrp[i + 1] = (int)F.lci.size();
        F.urp[i + 1] = (int)F.uci.size();
    }
    F.dinv = std::move(piv);
}

int host_ict(int n, const int *rp, const int *ci, const double *v, int maxfil, double droptol, HostTriFactors &F)
{
    F = HostTriFactors();
    F.lrp.assign(n + 1, 0);
    F.urp.assign(n + 1, 0);
    if (n == 0) return -1;
    if (maxfil > n - 1) maxfil = n - 1;
    if (maxfil < 0) maxfil = 0;
    std::vector<double> thr(n);
    for (int i = 0; i < n; i++) {
        double s = 0;
        bool diag = false;
        for (int q = rp[i]; q < rp[i + 1]; q++) {
            s += v[q] * v[q];
            diag |= ci[q] == i;
        }
        if (!diag) return i;
        thr[i] = std::sqrt(s) * droptol;
    }
    // rows of the Cholesky factor: its kept entries (ascending columns), then
    // 1/sqrt(pivot) as the last entry
    std::vector<int> lp(n + 1, 0), lc;
    std::vector<double> lx;
    lc.reserve((size_t)n * (maxfil + 1));
    lx.reserve((size_t)n * (maxfil + 1));
    double d0 = v[rp[0]];
    if (std::fabs(d0) < 1e-20) d0 = PIVOT_SUBST * (1 / droptol) * thr[0] + thr[0];
    lc.push_back(0);
    lx.push_back(1 / std::sqrt(std::fabs(d0)));
    lp[1] = 1;
    std::vector<double> w(n, 0.0), cv;
    std::vector<int> cc;
    for (int i = 1; i < n; i++) {
        const int c0 = ci[rp[i]];
        // clear the band from the first column of factor row c0 (row i's
        // own slot alone when it has no lower entry)
        for (int j = c0 < i ? lc[lp[c0]] : i; j <= i; j++) w[j] = 0;
        for (int q = rp[i]; q < rp[i + 1]; q++) w[ci[q]] = v[q];
        cv.clear();
        cc.clear();
        for (int j = c0; j < i; j++) {
            const int dg = lp[j + 1] - 1;
            double acc = 0;
            for (int p = lp[j]; p < dg; p++) acc += w[lc[p]] * lx[p];
            w[j] -= acc;
            w[j] *= lx[dg];
            if (std::fabs(w[j]) > thr[i]) {
                cv.push_back(w[j]);
                cc.push_back(j);
                w[i] -= w[j] * w[j];
            }
        }
        if (std::fabs(w[i]) < 1e-20) w[i] = PIVOT_SUBST * (1 / droptol) * thr[i] + thr[i];
        w[i] = 1 / std::sqrt(std::fabs(w[i]));
        int cnt = (int)cc.size();
        if (cnt > maxfil) {
            keep_largest(cv.data(), cc.data(), maxfil, cnt);
            cnt = maxfil;
        }
        for (int t = 0; t < cnt; t++) {
            lc.push_back(cc[t]);
            lx.push_back(cv[t]);
        }
        lc.push_back(i);
        lx.push_back(w[i]);
        lp[i + 1] = (int)lc.size();
    }
    // conversion: L' = L D (D = the stored 1/sqrt(pivot)), U' = L'^T,
    // dinv = D^2; U' rows list their columns in ascending order
    std::vector<double> d(n);
    for (int i = 0; i < n; i++) d[i] = lx[lp[i + 1] - 1];
    std::vector<int> ucount(n + 1, 0);
    for (int i = 0; i < n; i++)
        for (int p = lp[i]; p < lp[i + 1] - 1; p++) ucount[lc[p] + 1]++;
    for (int i = 0; i < n; i++) F.urp[i + 1] = F.urp[i] + ucount[i + 1];
    F.uci.resize(F.urp[n]);
    F.uv.resize(F.urp[n]);
    std::vector<int> fill(F.urp.begin(), F.urp.end() - 1);
    for (int i = 0; i < n; i++) {
        for (int p = lp[i]; p < lp[i + 1] - 1; p++) {
            const int j = lc[p];
            const double x = lx[p] * d[j];
            F.lci.push_back(j);
            F.lv.push_back(x);
            F.uci[fill[j]] = i;
            F.uv[fill[j]++] = x;
        }
        F.lrp[i + 1] = (int)F.lci.size();
    }
    F.dinv.resize(n);
    for (int i = 0; i < n; i++) F.dinv[i] = d[i] * d[i];
    return -1;
}

}  // namespace xs
