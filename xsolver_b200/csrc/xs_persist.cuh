// BiCGSTAB iterations as one persistent kernel (xs_persist.cu): the
// declarations BicgRun calls.
#pragma once
#include "xs_internal.cuh"

namespace xs {

struct SolveCtx;
struct Operator;
struct PrecondDev;

template <typename VT>
struct PersistVectors {
    VT *x, *r, *rhat, *p, *p2, *u, *s, *v, *z1, *z2;
};

struct PersistTuning {
    int enabled = 0;  // off by default: a fault in its first GPU run is not yet explained
};
PersistTuning &persist_tuning();

// Run BicgRun's iteration (after its initial sequence) as one cooperative
// launch until KState says done or max_iters more iterations ran; bar is a
// 2-word device array (grid barrier count and generation, zero on first
// use).  False (nothing launched) when the configuration is not served:
// the caller then replays its graph.
bool persist_bicgstab(SolveCtx &c, const PersistVectors<float> &V, int max_iters, unsigned *bar);
bool persist_bicgstab(SolveCtx &c, const PersistVectors<double> &V, int max_iters, unsigned *bar);

}  // namespace xs
