// ParILUT placeholder: replaced by the full implementation below.
#pragma once
#include "xs_trsv.cuh"
#include "xs_spmv.cuh"

namespace xs {

struct ParilutResult {
    int n = 0;
    long nnzL = 0, nnzU = 0;
    DBuf<int> lrp, lci, urp, uci;
    DBuf<double> lv, uv, dinv;
    std::vector<int> hlrp, hlci, hurp, huci;
};

inline void parilut_build(cudaStream_t, int *, int, const Operator &, const std::vector<int> &, const std::vector<int> &,
                          double, int, double, ParilutResult &)
{
    throw Status(XS_ERR_UNSUPPORTED);
}
inline void ilut_to_tri(cudaStream_t, int, ParilutResult &, TriDev &, TriDev &, bool) { throw Status(XS_ERR_UNSUPPORTED); }

}  // namespace xs
