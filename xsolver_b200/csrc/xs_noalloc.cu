// LU solve that allocates nothing.
//
// Some callers cannot call cudaMalloc: code running inside a memory pool or
// allocator that owns all device memory, applications that must not allocate
// after start-up (fixed memory budgets, real-time loops), and callers that
// only hand in buffers they already own.  xs_lusolve_noalloc serves them: it
// takes the ILU factors and the vectors as device pointers and keeps its
// scratch — the two readiness buffers of the sync-free solves, the block
// tickets and an error word — in one file-scope __device__ array of fixed
// size, so no call allocates device memory.
//
// Limits and sharing:
//   * n <= 262144 rows (NA_MAX_ROWS): the array holds 2 * 262144 doubles
//     (4 MiB) plus a few words; every GPU that loads the library holds it
//     until the process exits.
//   * Every call uses the same array.  Each call re-initialises what must
//     start from a known state (tickets, error word, readiness buffers), so
//     the contents left by an earlier call do not matter; but two calls that
//     overlap on the GPU (different streams, or different host threads
//     sharing a device) race on the array and must be serialised by the
//     caller.
//   * The first call on a device looks up the array's device address
//     (cudaGetSymbolAddress) with that device current and keeps it for the
//     rest of the process; make that first call before any stream capture.
//     The kept address belongs to the device's current context, so calls
//     must not span a cudaDeviceReset (or any destruction and re-creation of
//     the primary context) on that device.
//   * Every call waits for `stream` (cudaStreamSynchronize) before it
//     returns, and reads the kernels' error word back to the host.
//   * Every pointer must be a valid device pointer when n > 0, also the
//     column and value arrays of a factor without entries.
//
// The solve itself is the same row computation as the plan-based sync-free
// solve (L: increasing column, dinv scale, U': decreasing column, separate
// multiply and subtract), processed in natural row order instead of
// dependency-level order, so its result is bitwise identical.
#include <cuda_runtime.h>
#include <mutex>
#include <stdint.h>

#include "../../include/xsolver_c.h"

namespace {

constexpr int NA_THREADS = 128;
constexpr int NA_MAX_ROWS = 262144;
constexpr unsigned long long NA_LIMIT_NS = 1000000000ull;
constexpr uint64_t NA_SENTINEL = 0x7ff4dead5e17e1a1ull;

// [0, MAX) L readiness buffer, [MAX, 2*MAX) U readiness buffer,
// then 4 words (as doubles): L ticket, U ticket, error word, spare
constexpr size_t NA_WORDS = 2 * (size_t)NA_MAX_ROWS + 4;
static __device__ __align__(256) double xs_noalloc_scratch[NA_WORDS];

struct NaScratch {
    double *lbuf;
    double *ubuf;
    unsigned *ticket_l;
    unsigned *ticket_u;
    int *err;
};

__device__ __forceinline__ unsigned long long na_timer()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
__device__ __forceinline__ double na_poll(const double *p)
{
    double v;
    asm volatile("ld.relaxed.gpu.global.f64 %0, [%1];" : "=d"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void na_publish(double *p, double v)
{
    asm volatile("st.relaxed.gpu.global.f64 [%0], %1;" ::"l"(p), "d"(v) : "memory");
}
__device__ __forceinline__ bool na_is_sentinel(double v) { return (uint64_t)__double_as_longlong(v) == NA_SENTINEL; }

__global__ void k_na_init(int n, NaScratch s)
{
    const double sent = __longlong_as_double((long long)NA_SENTINEL);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        s.lbuf[i] = sent;
        s.ubuf[i] = sent;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        *s.ticket_l = 0u;
        *s.ticket_u = 0u;
        *s.err = 0;
    }
}

// UPPER = false: y = L^{-1} x into lbuf (unit lower, entries in increasing
// column order).  UPPER = true: z = U'^{-1} (dinv * y), rows in decreasing
// order, entries in decreasing column order, result into ubuf and z.
template <bool UPPER>
__global__ void __launch_bounds__(NA_THREADS) k_na_trsv(int n, const int *__restrict__ rp, const int *__restrict__ ci,
                                                        const double *__restrict__ v, const double *__restrict__ dinv,
                                                        const double *rhs, double *self, double *out, NaScratch s)
{
    __shared__ int s_blk;
    unsigned *ticket = UPPER ? s.ticket_u : s.ticket_l;
    if (threadIdx.x == 0) {
        const unsigned t = atomicAdd(ticket, 1u);
        s_blk = (int)t;
    }
    __syncthreads();
    const int p = s_blk * NA_THREADS + (int)threadIdx.x;
    if (p >= n) return;
    const int row = UPPER ? n - 1 - p : p;  // every dependency sits at a smaller position
    double acc;
    if (!UPPER) acc = rhs[row];
    else {
        const double yv = rhs[row];
        acc = yv * dinv[row];
    }
    const int k0 = rp[row], k1 = rp[row + 1];
    for (int q = 0; q < k1 - k0; q++) {
        const int k = UPPER ? k1 - 1 - q : k0 + q;
        const int c = ci[k];
        double y = na_poll(self + c);
        if (na_is_sentinel(y)) {
            const unsigned long long t0 = na_timer();
            long spins = 0;
            while (na_is_sentinel(y)) {
                __nanosleep(64);  // yield point: the producer may be a lane of this warp
                y = na_poll(self + c);
                if ((++spins & 255) == 0) {
                    if (na_timer() - t0 > NA_LIMIT_NS) {
                        atomicOr(s.err, 1);
                        return;
                    }
                    if (*(volatile int *)s.err) return;
                }
            }
        }
        acc = acc - y * v[k];
    }
    na_publish(self + row, acc);
    if (out) out[row] = acc;
}

std::mutex g_mu;
double *g_base[64] = {nullptr};  // device address of the array, per device ordinal

int scratch_for_current_device(NaScratch &s)
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return XS_ERR_CUDA;
    if (dev < 0 || dev >= 64) return XS_ERR_UNSUPPORTED;
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_base[dev]) {
        void *ptr = nullptr;
        if (cudaGetSymbolAddress(&ptr, xs_noalloc_scratch) != cudaSuccess || !ptr) return XS_ERR_CUDA;
        g_base[dev] = (double *)ptr;
    }
    double *b = g_base[dev];
    s.lbuf = b;
    s.ubuf = b + NA_MAX_ROWS;
    unsigned *w = (unsigned *)(b + 2 * (size_t)NA_MAX_ROWS);
    s.ticket_l = w;
    s.ticket_u = w + 2;
    s.err = (int *)(w + 4);
    return XS_OK;
}

}  // namespace

extern "C" int xs_lusolve_noalloc(int n, const int *lrp, const int *lci, const double *lv, const double *dinv,
                                  const int *urp, const int *uci, const double *uv, const double *x, double *z,
                                  void *stream)
{
    if (n < 0) return XS_ERR_INVALID;
    if (n > 0 && (!lrp || !lci || !lv || !dinv || !urp || !uci || !uv || !x || !z)) return XS_ERR_INVALID;
    if (n > NA_MAX_ROWS) return XS_ERR_CAPACITY;
    if (n == 0) return XS_OK;
    NaScratch s;
    int st = scratch_for_current_device(s);
    if (st != XS_OK) return st;
    cudaStream_t cs = (cudaStream_t)stream;
    const int blocks = (n + NA_THREADS - 1) / NA_THREADS;
    k_na_init<<<(n + 255) / 256, 256, 0, cs>>>(n, s);
    k_na_trsv<false><<<blocks, NA_THREADS, 0, cs>>>(n, lrp, lci, lv, nullptr, x, s.lbuf, nullptr, s);
    k_na_trsv<true><<<blocks, NA_THREADS, 0, cs>>>(n, urp, uci, uv, dinv, s.lbuf, s.ubuf, z, s);
    if (cudaGetLastError() != cudaSuccess) return XS_ERR_CUDA;
    int e = 0;
    if (cudaMemcpyAsync(&e, s.err, sizeof(int), cudaMemcpyDeviceToHost, cs) != cudaSuccess) return XS_ERR_CUDA;
    if (cudaStreamSynchronize(cs) != cudaSuccess) return XS_ERR_CUDA;
    return e ? XS_ERR_TRSV_TIMEOUT : XS_OK;
}
