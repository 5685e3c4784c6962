// Adjoint of the linear solve (no reference counterpart).
//
// For x = A^{-1} b and a loss L(x):  A^T lambda = dL/dx,  dL/db = lambda,
// dL/dA_ij = -lambda_i x_j on A's sparsity pattern.
// The backward solve runs the same Krylov method on A^T (an explicit CSR of
// A^T built once, so the transposed SpMV is the same gather kernel) with the
// transposed preconditioner: for M^{-1} = U'^{-1} Dinv L^{-1} (the seqilu0
// layout), M^{-T} = L^{-T} Dinv U'^{-T}, i.e. a unit lower solve with U'^T,
// the same Dinv, and a unit upper solve with L^T — both run by the sync-free
// kernels on transposed plans whose values are gathered from the forward
// factor array.  dL/db and dL/dA are formed by one fused kernel.
#pragma once
#include "xs_solvers.cuh"
#include "xs_gmres.cuh"

namespace xs {

// the solver drivers of one vector type
template <typename VT>
struct RunSet {
    PcgRun<VT, VT> pcg;
    CgLeftRun<VT, VT> cgl;
    IcgRun<VT, VT> icg;
    IcgmRun<VT, VT> icgm;
    IbicgRun<VT, VT> ibicg;
    BicgRun<VT, VT> bicg;
    GmresRun<VT, VT> gmres;
    GcrRun<VT, VT> gcr;
};

// dLdb = lambda ; dLdA[k] = -lambda_i * x_j for entry k = (i, j)
static __global__ void k_adjoint_grad(int n, const int *__restrict__ rp, const int *__restrict__ ci,
                               const double *__restrict__ lambda, const double *__restrict__ x, double *__restrict__ dLdb,
                               double *__restrict__ dLdA)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const double li = lambda[i];
        if (dLdb) dLdb[i] = li;
        if (dLdA) {
            const double mli = -li;
            for (int k = rp[i]; k < rp[i + 1]; k++) dLdA[k] = mli * __ldg(x + ci[k]);
        }
    }
}

struct AdjointState {
    DBuf<double> x_last;   // forward solution
    bool have_At = false;
    Operator At;
    PrecondDev Mt;
    bool have_Mt = false;
    int Mt_type = -1;
    DBuf<double> lam, rhs, grad_tmp;
    DBuf<double> gb, gA;  // gradient staging, kept across calls
    RunSet<double> runs;
    // forget the transposed operator/preconditioner (matrix or values changed)
    void reset()
    {
        have_At = false;
        have_Mt = false;
        Mt_type = -1;
    }
};

inline void adjoint_record_solution(AdjointState &a, cudaStream_t s, int n, const double *d_x)
{
    if (a.x_last.n != (size_t)n) a.x_last.alloc(n);
    XS_CUDA(cudaMemcpyAsync(a.x_last.p, d_x, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
}
inline void adjoint_set_solution(AdjointState &a, cudaStream_t s, int n, const double *h_x)
{
    if (a.x_last.n != (size_t)n) a.x_last.alloc(n);
    XS_CUDA(cudaMemcpyAsync(a.x_last.p, h_x, sizeof(double) * n, cudaMemcpyHostToDevice, s));
}

// host transpose of a CSR (rows of the result ascending in column order)
inline void host_transpose(int n, const int *rp, const int *ci, const double *v, std::vector<int> &trp,
                           std::vector<int> &tci, std::vector<double> *tv, std::vector<long> *tsrc)
{
    long nnz = rp[n];
    trp.assign(n + 1, 0);
    for (long k = 0; k < nnz; k++) trp[ci[k] + 1]++;
    for (int i = 0; i < n; i++) trp[i + 1] += trp[i];
    tci.resize(nnz);
    if (tv) tv->resize(nnz);
    if (tsrc) tsrc->resize(nnz);
    std::vector<int> pos(trp.begin(), trp.end() - 1);
    for (int i = 0; i < n; i++)
        for (int k = rp[i]; k < rp[i + 1]; k++) {
            int p = pos[ci[k]]++;
            tci[p] = i;
            if (tv) (*tv)[p] = v[k];
            if (tsrc) (*tsrc)[p] = k;
        }
}

}  // namespace xs
