// Matrix Market coordinate files into CSR (host code).  Replaces the
// reference's reader (hip/Tool/ReadMatrix/csr_mmio_highlevel.h:8-233,
// mmio_info / mmio_data over the NIST mmio.h) used by its drivers
// (hip/main_solve_base.cpp:36-45).
//
// Same result as the reference for the files it reads: 1-based indices made
// 0-based; a general file stores -value (the reference negates, :63-68), a
// symmetric or hermitian file stores value at (i, j) and, off the diagonal,
// at (j, i) (:69-79); diag[i] = the value of entry (i, i) as read; rows are
// filled in file order by a counting sort (:200-214), so columns within a
// row keep the file's order (the solver accepts unsorted rows).
// reference_quirks = 0 keeps general files' values as written.
//
// Unlike the reference, which ignores a bad banner and would misread them,
// complex, pattern and skew-symmetric files are refused (XS_ERR_UNSUPPORTED),
// and a missing banner, a short entry list or an index out of range is an
// error (XS_ERR_INVALID) instead of undefined behaviour.
#pragma once
#include <cctype>
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>
#include "xs_internal.cuh"

namespace xs {

struct MmFile {
    int m = 0, n = 0;
    long reported = 0;   // entries listed in the file
    bool symmetric = false;
    std::vector<int> ei, ej;  // 0-based
    std::vector<double> ev;
};

inline std::string mm_lower(std::string s)
{
    for (auto &c : s) c = (char)std::tolower((unsigned char)c);
    return s;
}

inline void mm_parse(const char *path, MmFile &F)
{
    if (!path) throw Status(XS_ERR_INVALID);
    FILE *f = std::fopen(path, "rb");
    if (!f) throw Status(XS_ERR_INVALID);
    std::string buf;
    {
        char tmp[1 << 16];
        size_t got;
        while ((got = std::fread(tmp, 1, sizeof(tmp), f)) > 0) buf.append(tmp, got);
        std::fclose(f);
    }
    const char *p = buf.c_str(), *end = p + buf.size();
    // banner: %%MatrixMarket matrix coordinate <field> <symmetry>
    const char *eol = p;
    while (eol < end && *eol != '\n') eol++;
    {
        std::vector<std::string> tok;
        std::string cur;
        for (const char *q = p; q < eol; q++) {
            if (std::isspace((unsigned char)*q)) {
                if (!cur.empty()) tok.push_back(mm_lower(cur)), cur.clear();
            } else {
                cur += *q;
            }
        }
        if (!cur.empty()) tok.push_back(mm_lower(cur));
        if (tok.size() < 5 || tok[0] != "%%matrixmarket" || tok[1] != "matrix" || tok[2] != "coordinate")
            throw Status(XS_ERR_INVALID);
        if (tok[3] != "real" && tok[3] != "double" && tok[3] != "integer") throw Status(XS_ERR_UNSUPPORTED);
        if (tok[4] == "symmetric" || tok[4] == "hermitian") F.symmetric = true;
        else if (tok[4] == "general") F.symmetric = false;
        else throw Status(XS_ERR_UNSUPPORTED);
    }
    p = eol;
    // comments and blank lines, then the size line
    while (p < end) {
        while (p < end && (*p == '\n' || *p == '\r' || *p == ' ' || *p == '\t')) p++;
        if (p < end && *p == '%') {
            while (p < end && *p != '\n') p++;
            continue;
        }
        break;
    }
    char *q;
    const long m = std::strtol(p, &q, 10);
    if (q == p) throw Status(XS_ERR_INVALID);
    p = q;
    const long n = std::strtol(p, &q, 10);
    if (q == p) throw Status(XS_ERR_INVALID);
    p = q;
    const long nnz = std::strtol(p, &q, 10);
    if (q == p || m < 0 || n < 0 || nnz < 0 || m > 0x7ffffffeL || n > 0x7ffffffeL) throw Status(XS_ERR_INVALID);
    p = q;
    // a symmetric file mirrors (i, j) into row j: only square matrices
    if (F.symmetric && m != n) throw Status(XS_ERR_INVALID);
    // an entry takes at least "i j v" plus a separator: a count the rest of
    // the file cannot hold is a short list, refused before any allocation
    if (nnz > (long)(end - p) / 6 + 1) throw Status(XS_ERR_INVALID);
    F.m = (int)m;
    F.n = (int)n;
    F.reported = nnz;
    F.ei.resize(nnz);
    F.ej.resize(nnz);
    F.ev.resize(nnz);
    for (long k = 0; k < nnz; k++) {
        const long i = std::strtol(p, &q, 10);
        if (q == p) throw Status(XS_ERR_INVALID);
        p = q;
        const long j = std::strtol(p, &q, 10);
        if (q == p) throw Status(XS_ERR_INVALID);
        p = q;
        const double v = std::strtod(p, &q);
        if (q == p) throw Status(XS_ERR_INVALID);
        p = q;
        if (i < 1 || i > m || j < 1 || j > n) throw Status(XS_ERR_INVALID);
        F.ei[k] = (int)(i - 1);
        F.ej[k] = (int)(j - 1);
        F.ev[k] = v;
    }
}

// CSR entry count after the symmetric expansion
inline long mm_csr_nnz(const MmFile &F)
{
    long c = 0;
    for (long k = 0; k < F.reported; k++) c += (F.symmetric && F.ei[k] != F.ej[k]) ? 2 : 1;
    return c;
}

// rowptr[m+1], colidx/val[mm_csr_nnz], diag[m] (optional)
inline void mm_to_csr(const MmFile &F, bool quirks, int *rowptr, int *colidx, double *val, double *diag)
{
    const int m = F.m;
    std::vector<long> cnt(m + 1, 0);
    for (long k = 0; k < F.reported; k++) {
        cnt[F.ei[k]]++;
        if (F.symmetric && F.ei[k] != F.ej[k]) cnt[F.ej[k]]++;
    }
    long acc = 0;
    for (int i = 0; i < m; i++) {
        rowptr[i] = (int)acc;
        acc += cnt[i];
        if (acc > 0x7fffffffL) throw Status(XS_ERR_CAPACITY);
    }
    rowptr[m] = (int)acc;
    if (diag)
        for (int i = 0; i < m; i++) diag[i] = 0.0;
    std::vector<long> fill(m);
    for (int i = 0; i < m; i++) fill[i] = rowptr[i];
    for (long k = 0; k < F.reported; k++) {
        const int i = F.ei[k], j = F.ej[k];
        const double v = F.ev[k];
        if (!F.symmetric) {
            const long at = fill[i]++;
            colidx[at] = j;
            val[at] = quirks ? -v : v;
        } else {
            long at = fill[i]++;
            colidx[at] = j;
            val[at] = v;
            if (i != j) {
                at = fill[j]++;
                colidx[at] = i;
                val[at] = v;
            }
        }
        if (diag && i == j) diag[i] = v;
    }
}

}  // namespace xs
