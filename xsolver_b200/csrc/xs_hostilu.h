// Threshold factorizations that run on the host: Saad's dual-threshold ILUT
// and the left-looking incomplete Cholesky with threshold (ICT).  Both are
// one dependency chain over the rows (a row's last elimination step needs the
// row just before it on a natural-order stencil), so they are computed by the
// CPU and only their triangular solves run on the GPU.  The factors come out
// in the layout of the other ILU factors: L strict lower with unit diagonal,
// dinv, and U' strict upper scaled row-wise by dinv, applied as
// z = U'^-1 (dinv * L^-1 x).
#pragma once
#include <vector>

namespace xs {

struct HostTriFactors {
    std::vector<int> lrp, lci, urp, uci;
    std::vector<double> lv, uv, dinv;
};

// Saad ILUT(droptol, lfil) of a sorted 0-based CSR matrix (hip/Precond/
// ilut_diag_in_csr.cpp:20-251, ilutp_final) followed by the split of
// hip/HostMatrix/HostMatrixCSR.cpp:230-268 (seqilut).  lfil >= 1.
void host_ilut(int n, const int *rp, const int *ci, const double *v, int lfil, double droptol, HostTriFactors &F);

// ICT(droptol, maxfil) (hip/Precond/ict_l.cpp:130-205, ict_fact_l, with the
// row norms of :112-129) followed by the conversion of hip/HostMatrix/
// HostMatrixCSR.cpp:327-384 (seqict).  The matrix is the full symmetric CSR;
// maxfil is clamped to n-1 as hip/Precond/precon_ict.cpp:3-4 does.
// Returns the first row without a diagonal entry, or -1.
int host_ict(int n, const int *rp, const int *ci, const double *v, int maxfil, double droptol, HostTriFactors &F);

}  // namespace xs
