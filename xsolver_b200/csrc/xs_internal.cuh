// Internal definitions shared by the xsolver_b200 CUDA sources.
//
// Conventions
//  * Matrices are CSR, 0-based, int32 indices, sorted columns, stored on the
//    device; rows are the reference's "cells" (nInterior).
//  * Every reduction uses a fixed grid and a fixed element->block mapping, and
//    the last block to finish (ticket counter) sums the per-block partials in
//    block order, so results are run-to-run deterministic.
//  * Scalars of a Krylov iteration (alpha, beta, omega, residual norms,
//    convergence flag) live in device memory (KState) and never travel to the
//    host inside the iteration loop.
//  * Every spin-wait in a kernel is bounded; on expiry the kernel records an
//    error in the device status word and returns.
#pragma once

#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <stdint.h>
#include <cstdio>
#include <cstdlib>
#include <algorithm>
#include <chrono>
#include <mutex>
#include <thread>
#include <utility>
#include <vector>

#include "../../include/xsolver_c.h"

namespace xs {

// Setup phase tracing: with XS_TRACE=1 in the environment, each traced
// phase waits for its stream and prints its wall time to stderr.
inline bool trace_on()
{
    static int on = -1;
    if (on < 0) {
        const char *e = getenv("XS_TRACE");
        on = (e && atoi(e) != 0) ? 1 : 0;
    }
    return on == 1;
}
struct Trace {
    const char *what;
    cudaStream_t s;
    std::chrono::steady_clock::time_point t0;
    Trace(const char *w, cudaStream_t st) : what(w), s(st)
    {
        if (trace_on()) {
            cudaStreamSynchronize(s);
            t0 = std::chrono::steady_clock::now();
        }
    }
    void stop()
    {
        if (trace_on() && what) {
            cudaStreamSynchronize(s);
            const double ms =
                std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
            fprintf(stderr, "[xs trace] %-28s %10.2f ms\n", what, ms);
        }
        what = nullptr;
    }
    ~Trace() { stop(); }
};

// Host pattern scans over [0, n) split into contiguous ranges, one per host
// thread (at most 16, and none for ranges under 64K rows); fn(lo, hi, t)
// must not throw.  Returns the number of ranges.
template <typename F>
inline int host_parallel_rows(long n, F fn)
{
    const long hc = std::max(1u, std::thread::hardware_concurrency());
    const int T = (int)std::max(1L, std::min(std::min(hc, 16L), n / 65536));
    if (T == 1) {
        fn(0L, n, 0);
        return 1;
    }
    std::vector<std::thread> th;
    th.reserve(T);
    for (int t = 0; t < T; t++) th.emplace_back([&, t] { fn(n * t / T, n * (t + 1) / T, t); });
    for (auto &x : th) x.join();
    return T;
}

// ---------------------------------------------------------------- errors
struct CudaError {
    cudaError_t err;
};

#define XS_CUDA(call)                                                                            \
    do {                                                                                         \
        cudaError_t _e = (call);                                                                 \
        if (_e != cudaSuccess) {                                                                 \
            if (getenv("XS_DEBUG")) fprintf(stderr, "xsolver_b200: %s failed: %s (%s:%d)\n", #call, \
                                            cudaGetErrorString(_e), __FILE__, __LINE__);         \
            throw ::xs::Status(_e == cudaErrorMemoryAllocation ? XS_ERR_NOMEM : XS_ERR_CUDA);    \
        }                                                                                        \
    } while (0)

struct Status {
    int code;
    explicit Status(int c) : code(c) {}
};

// ---------------------------------------------------------------- programmatic dependent launch
// Kernels of the Krylov iteration bodies are launched with programmatic
// stream serialization: a kernel may start while its predecessor on the
// stream drains, run its independent prologue (shared-memory staging, loads
// of constant matrix data), and must execute pdl_wait() before it reads
// anything the predecessor produced or writes anything the predecessor
// reads.  pdl_trigger() lets the successor launch once every block of this
// kernel has started.  Outside a programmatic launch both are no-ops.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" :::); }

struct PdlTuning {
    int enabled = 1;
};
PdlTuning &pdl_tuning();
// vector updates fused into the preconditioner passes that read their
// result (process-wide; results are identical either way)
bool &vec_fusion_flag();
inline bool vec_fusion() { return vec_fusion_flag(); }

template <typename... KArgs, typename... Args>
inline void launch_pdl(void (*kern)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s, Args &&...args)
{
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = pdl_tuning().enabled ? 1 : 0;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    cudaError_t e = cudaLaunchKernelEx(&cfg, kern, std::forward<Args>(args)...);
    if (e != cudaSuccess) throw Status(XS_ERR_CUDA);
}

inline void check_launch()
{
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        if (getenv("XS_DEBUG")) fprintf(stderr, "xsolver_b200: launch failed: %s\n", cudaGetErrorString(e));
        throw Status(XS_ERR_CUDA);
    }
}

// ---------------------------------------------------------------- scratch pool
// A stream-ordered memory pool per device for the temporaries of a factor
// builder that allocates and frees multi-GB buffers every sweep.  Freed
// memory stays in the pool (release threshold: never) until pool_trim().
inline cudaMemPool_t scratch_pool()
{
    static std::mutex mu;
    static cudaMemPool_t pools[64] = {};
    int dev = 0;
    XS_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) throw Status(XS_ERR_CUDA);
    std::lock_guard<std::mutex> g(mu);
    if (!pools[dev]) {
        cudaMemPoolProps props = {};
        props.allocType = cudaMemAllocationTypePinned;
        props.handleTypes = cudaMemHandleTypeNone;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = dev;
        XS_CUDA(cudaMemPoolCreate(&pools[dev], &props));
        unsigned long long never = ~0ull;
        XS_CUDA(cudaMemPoolSetAttribute(pools[dev], cudaMemPoolAttrReleaseThreshold, &never));
    }
    return pools[dev];
}

// While a PoolScope is open on this host thread, DBuf::alloc takes memory
// from scratch_pool() in the order of the scope's stream and such a buffer is
// returned with cudaFreeAsync on that stream: every use of it must be on
// that stream.
struct PoolScope {
    static cudaStream_t &stream()
    {
        static thread_local cudaStream_t s = nullptr;
        return s;
    }
    static bool &open()
    {
        static thread_local bool o = false;
        return o;
    }
    cudaStream_t prev_s;
    bool prev_o, ended = false;
    explicit PoolScope(cudaStream_t s) : prev_s(stream()), prev_o(open())
    {
        stream() = s;
        open() = true;
    }
    void end()
    {
        if (ended) return;
        stream() = prev_s;
        open() = prev_o;
        ended = true;
    }
    ~PoolScope() { end(); }
};

// hand the pool's unused memory back to the device once the frees queued on
// stream s have run
inline void pool_trim(cudaStream_t s)
{
    XS_CUDA(cudaStreamSynchronize(s));
    XS_CUDA(cudaMemPoolTrimTo(scratch_pool(), 0));
}

// ---------------------------------------------------------------- device buffers
template <typename T>
struct DBuf {
    T *p = nullptr;
    size_t n = 0;
    cudaStream_t ps = nullptr;  // pooled buffers: the stream that frees them
    bool pooled = false;
    DBuf() = default;
    DBuf(const DBuf &) = delete;
    DBuf &operator=(const DBuf &) = delete;
    DBuf(DBuf &&o) noexcept : p(o.p), n(o.n), ps(o.ps), pooled(o.pooled)
    {
        o.p = nullptr;
        o.n = 0;
        o.pooled = false;
    }
    DBuf &operator=(DBuf &&o) noexcept
    {
        if (this != &o) {
            free();
            p = o.p; n = o.n; ps = o.ps; pooled = o.pooled;
            o.p = nullptr; o.n = 0; o.pooled = false;
        }
        return *this;
    }
    ~DBuf() { free(); }
    // pad: extra elements allocated (and zeroed) past n, e.g. for aligned bulk copies
    void alloc(size_t count, size_t pad = 0)
    {
        free();
        size_t bytes = (count + pad) * sizeof(T);
        if (bytes == 0) bytes = 16;
        if (PoolScope::open()) {
            ps = PoolScope::stream();
            XS_CUDA(cudaMallocFromPoolAsync((void **)&p, bytes, scratch_pool(), ps));
            pooled = true;
            XS_CUDA(cudaMemsetAsync(p, 0, bytes, ps));
        } else {
            XS_CUDA(cudaMalloc((void **)&p, bytes));
            // zero and wait: the handle's stream does not synchronise with the
            // legacy default stream, so an asynchronous memset there could land
            // after the handle's own first writes to this buffer
            XS_CUDA(cudaMemsetAsync(p, 0, bytes, 0));
            XS_CUDA(cudaStreamSynchronize(0));
        }
        n = count;
    }
    void free()
    {
        if (p) {
            if (pooled) cudaFreeAsync(p, ps);
            else cudaFree(p);
        }
        p = nullptr;
        n = 0;
        pooled = false;
    }
    void upload(const T *h, size_t count, cudaStream_t s)
    {
        XS_CUDA(cudaMemcpyAsync(p, h, count * sizeof(T), cudaMemcpyHostToDevice, s));
    }
    void download(T *h, size_t count, cudaStream_t s) const
    {
        XS_CUDA(cudaMemcpyAsync(h, p, count * sizeof(T), cudaMemcpyDeviceToHost, s));
    }
    operator T *() const { return p; }
};

// ---------------------------------------------------------------- device status
// status word bits written by kernels (device side), read by the host after a
// synchronisation point
enum DevErr : int {
    DEV_OK = 0,
    DEV_TRSV_TIMEOUT = 1,
    DEV_BREAKDOWN = 2,
    DEV_NAN = 4,
    DEV_TMA_TIMEOUT = 8,
    DEV_CAPACITY = 16,
    DEV_FACTOR_TIMEOUT = 32,
    DEV_NO_DIAG = 64
};

inline int dev_err_to_status(int e)
{
    if (e & (DEV_TRSV_TIMEOUT | DEV_FACTOR_TIMEOUT | DEV_TMA_TIMEOUT)) return XS_ERR_TRSV_TIMEOUT;
    if (e & DEV_CAPACITY) return XS_ERR_CAPACITY;
    if (e & DEV_NO_DIAG) return XS_ERR_NO_DIAG;
    if (e & DEV_NAN) return XS_ERR_NAN;
    if (e & DEV_BREAKDOWN) return XS_ERR_BREAKDOWN;
    return XS_OK;
}

// ---------------------------------------------------------------- Krylov state
// Scalar slots used by the solver bodies (indices into KState::sc)
constexpr int KS_SLOTS = 48;

struct KState {
    double sc[KS_SLOTS];  // method-defined scalars
    double res0;          // initial residual norm (the method's own norm)
    double rnorm;         // latest residual norm
    double tol;           // relative tolerance
    double abstol;        // absolute tolerance (hip: resl <= absolute_tol)
    int iter;             // iterations completed
    int maxiter;
    int done;             // 0 running, 1 converged, 2 maxiter, 3 breakdown/error
    int err;              // DevErr bits
    int conv_inner;       // GMRES/GCR: inner index at convergence
    int kcols;            // GMRES: columns used by the final update
    int finalized;        // GMRES: final update applied
    int cycle_i;          // GMRES/GCR: inner index inside the current cycle
    double *hist;         // device history: hist[0] = res0, hist[k+1] = after iteration k
    double *hist_rel;     // device history, method's relative residual per iteration (intel convention)
    int pbuf;             // BiCGSTAB with the p update fused: which of its two p buffers holds p (0/1)
};

// ---------------------------------------------------------------- launch geometry
struct Geom {
    int sms = 148;
    int red_grid = 1184;  // fixed grid of the vector-op reductions: 8 CTAs of 256 per SM (full occupancy)
    int red_block = 256;
};
Geom &geom();

// ---------------------------------------------------------------- sentinel values
// The sync-free triangular solves signal "row ready" through the value
// itself: a solve buffer holds a NaN bit pattern that IEEE arithmetic never
// produces (GPU arithmetic yields the canonical NaN 0x7fff...), and a row is
// ready once its value differs from that pattern.
__host__ __device__ constexpr uint64_t sentinel_bits64() { return 0x7ff4dead5e17e1a1ull; }
__host__ __device__ constexpr uint32_t sentinel_bits32() { return 0x7fa5e17eu; }

template <typename V>
struct Sentinel;
template <>
struct Sentinel<double> {
    __device__ static double value() { return __longlong_as_double((long long)sentinel_bits64()); }
    __device__ static bool is(double v) { return (uint64_t)__double_as_longlong(v) == sentinel_bits64(); }
};
template <>
struct Sentinel<float> {
    __device__ static float value() { return __int_as_float((int)sentinel_bits32()); }
    __device__ static bool is(float v) { return (uint32_t)__float_as_int(v) == sentinel_bits32(); }
};

// Load of a vector element that kernels read while another kernel wrote it
// earlier (gathers of x in SpMV, of iterates in sweep passes): through the
// read-only path by default.  The persistent iteration (a kernel whose
// phases write what its later phases read) is compiled with
// XS_COHERENT_VECTOR_LOADS, which reads those elements from L2 instead.
#ifdef XS_COHERENT_VECTOR_LOADS
#define XS_VLD(p) __ldcg(p)
#else
#define XS_VLD(p) __ldg(p)
#endif

// nanosecond wall clock for bounding every spin-wait
__device__ __forceinline__ unsigned long long gtimer()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
constexpr unsigned long long WAIT_LIMIT_NS = 1000000000ull;  // 1 s

// relaxed, L1-bypassing accesses for values other SMs write while we poll
__device__ __forceinline__ double ld_poll(const double *p)
{
    double v;
    asm volatile("ld.relaxed.gpu.global.f64 %0, [%1];" : "=d"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ float ld_poll(const float *p)
{
    float v;
    asm volatile("ld.relaxed.gpu.global.f32 %0, [%1];" : "=f"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_publish(double *p, double v)
{
    asm volatile("st.relaxed.gpu.global.f64 [%0], %1;" ::"l"(p), "d"(v) : "memory");
}
__device__ __forceinline__ void st_publish(float *p, float v)
{
    asm volatile("st.relaxed.gpu.global.f32 [%0], %1;" ::"l"(p), "f"(v) : "memory");
}
__device__ __forceinline__ int ld_acquire(const int *p)
{
    int v;
    asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release(int *p, int v)
{
    asm volatile("st.release.gpu.global.b32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// ---------------------------------------------------------------- factor value types
template <typename T>
struct FVal;
// ld: load one stored factor value and widen it; cvt: widen a loaded one
template <>
struct FVal<double> {
    __device__ static double ld(const double *p, long i) { return __ldg(p + i); }
    __device__ static double cvt(double v) { return v; }
};
template <>
struct FVal<float> {
    __device__ static float ld(const float *p, long i) { return __ldg(p + i); }
    __device__ static float cvt(float v) { return v; }
};
template <>
struct FVal<__nv_bfloat16> {
    __device__ static float ld(const __nv_bfloat16 *p, long i) { return __bfloat162float(__ldg(p + i)); }
    __device__ static float cvt(__nv_bfloat16 v) { return __bfloat162float(v); }
};
template <>
struct FVal<__half> {
    __device__ static float ld(const __half *p, long i) { return __half2float(__ldg(p + i)); }
    __device__ static float cvt(__half v) { return __half2float(v); }
};

// ---------------------------------------------------------------- deterministic reductions
// One "reduction slot": per-block partials for K values and a ticket counter.
struct RedSlot {
    double *part;      // [K][grid]
    unsigned *ticket;  // single counter, reset by the last block
};

template <int K>
__device__ __forceinline__ void warp_sum(double (&v)[K])
{
#pragma unroll
    for (int k = 0; k < K; k++) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_xor_sync(0xffffffffu, v[k], o);
    }
}

// Reduce v[K] over the block, publish the block partial, and let the last
// block (in ticket order) sum all partials in block order.  Returns true in
// every thread of the last block; the totals are then in tot[K] (shared).
// blockDim.x must be a multiple of 32 and <= 1024.
template <int K>
__device__ bool block_reduce_publish(double (&v)[K], RedSlot slot, double *tot /*shared, >= K*/)
{
    __shared__ double sred[32][K > 0 ? K : 1];
    __shared__ bool s_last;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    warp_sum<K>(v);
    if (lane == 0) {
#pragma unroll
        for (int k = 0; k < K; k++) sred[wid][k] = v[k];
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        const int G = gridDim.x;
#pragma unroll
        for (int k = 0; k < K; k++) {
            double s = 0.0;
            for (int w = 0; w < nw; w++) s += sred[w][k];
            slot.part[(long)k * G + blockIdx.x] = s;
        }
        __threadfence();
        unsigned t = atomicAdd(slot.ticket, 1u);
        s_last = (t == (unsigned)G - 1);
    }
    __syncthreads();
    if (!s_last) return false;
    __threadfence();
    // last block: sum partials in fixed order
    const int G = gridDim.x;
#pragma unroll
    for (int k = 0; k < K; k++) {
        double s = 0.0;
        for (int b = threadIdx.x; b < G; b += blockDim.x) s += __ldcg(slot.part + (long)k * G + b);
        v[k] = s;
    }
    warp_sum<K>(v);
    __syncthreads();
    if (lane == 0) {
#pragma unroll
        for (int k = 0; k < K; k++) sred[wid][k] = v[k];
    }
    __syncthreads();
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < K; k++) {
            double s = 0.0;
            for (int w = 0; w < nw; w++) s += sred[w][k];
            tot[k] = s;
        }
        *slot.ticket = 0u;
    }
    __syncthreads();
    return true;
}

// ---------------------------------------------------------------- CSR / plans
struct DevCsr {
    int n = 0;
    long nnz = 0;
    const int *rp = nullptr;
    const int *ci = nullptr;
    const double *v = nullptr;
    const float *v32 = nullptr;
};

// Row-block tiling of a CSR matrix for the staged SpMV kernel.  Block b covers
// rows [rb[b], rb[b+1]); its entries are copied to shared memory by one bulk
// copy of the 16-byte aligned range that contains them.
struct SpmvTiling {
    int nblocks = 0;
    int max_rows = 0;      // rows per block (<= threads per block)
    int cap = 0;           // max entries staged per block (aligned range)
    DBuf<int> rb;          // nblocks+1 row boundaries
    DBuf<int> longrow;     // 1 if the block is a single row longer than cap
};

struct DevEll {
    int n = 0, w = 0;
    const int *ci = nullptr;     // [w][n] column-major
    const double *v = nullptr;   // [w][n]
    const float *v32 = nullptr;  // [w][n]
};

// A triangular factor prepared for the sync-free solve: rows permuted into
// dependency-level order ("positions"), each position's entries stored
// contiguously in the order the row sum is accumulated.
template <typename FT>
struct TriPlan {
    int n = 0;
    long nnz = 0;
    int nlevels = 0;
    const int *perm = nullptr;  // position -> row
    const int *prp = nullptr;   // position row pointer (n+1)
    const int *pci = nullptr;   // dependency row of each entry
    const FT *pv = nullptr;     // entry values
    const void *dinv = nullptr; // per position (U solve only): double or float
};

}  // namespace xs
