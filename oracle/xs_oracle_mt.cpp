// Threaded timing variant of the oracle's BiCGSTAB + ILU(0) solve.
//
// TEST INFRASTRUCTURE, not the product: the benchmark's CPU reference arm
// times the reference algorithm with it on all host threads.  Parity tests
// use the single-threaded restatement in xs_oracle.cpp, which this file does
// not touch.
//
// Algorithm: right-preconditioned BiCGSTAB, intel/mpisolver-C-v1.cpp:365-482
// (phi kept in the preconditioned variable, sol = M^-1 phi at the end), with
// the ILU(0) apply of hip/HostMatrix/HostMatrixCSR.cpp:385-409 (L with unit
// diagonal forward, scale by dinv, U' row-scaled backward).  The reference
// runs its SpMV and BLAS-1 calls through a threaded BLAS and its triangular
// solves sequentially; so does this variant (a persistent pool of host
// threads, each taking one contiguous range of every loop):
//   * SpMV, axpy, scal and copy run rows / elements on the threads with each
//     element's arithmetic unchanged (results independent of the thread
//     count);
//   * dot products sum fixed blocks of ORCMT_DOT_BLOCK elements in parallel
//     and the block sums in order (deterministic for any thread count; the
//     order differs from the single-threaded oracle's, so iteration counts
//     may differ by a step or two);
//   * the LU apply is sequential, as in the reference.
#include <algorithm>
#include <cmath>
#include <condition_variable>
#include <functional>
#include <mutex>
#include <thread>
#include <vector>

namespace {

constexpr long ORCMT_DOT_BLOCK = 16384;

// Fork-join pool: run(f) calls f(t) for t = 0..T-1, f(0) on the caller, and
// returns when all are done.
class Pool {
  public:
    explicit Pool(int T) : T_(std::max(1, T))
    {
        for (int t = 1; t < T_; t++) th_.emplace_back([this, t] { loop(t); });
    }
    ~Pool()
    {
        {
            std::lock_guard<std::mutex> g(m_);
            quit_ = true;
            gen_++;
        }
        cv_.notify_all();
        for (auto &x : th_) x.join();
    }
    int size() const { return T_; }
    void run(const std::function<void(int)> &f)
    {
        {
            std::lock_guard<std::mutex> g(m_);
            job_ = &f;
            pending_ = T_ - 1;
            gen_++;
        }
        cv_.notify_all();
        f(0);
        std::unique_lock<std::mutex> lk(m_);
        done_.wait(lk, [this] { return pending_ == 0; });
    }
    // [lo, hi) of thread t's share of n items
    void range(long n, int t, long &lo, long &hi) const
    {
        lo = n * t / T_;
        hi = n * (t + 1) / T_;
    }

  private:
    void loop(int t)
    {
        long seen = 0;
        for (;;) {
            const std::function<void(int)> *f;
            {
                std::unique_lock<std::mutex> lk(m_);
                cv_.wait(lk, [&] { return gen_ != seen; });
                seen = gen_;
                if (quit_) return;
                f = job_;
            }
            (*f)(t);
            std::lock_guard<std::mutex> g(m_);
            if (--pending_ == 0) done_.notify_one();
        }
    }
    int T_;
    std::vector<std::thread> th_;
    std::mutex m_;
    std::condition_variable cv_, done_;
    const std::function<void(int)> *job_ = nullptr;
    long gen_ = 0;
    int pending_ = 0;
    bool quit_ = false;
};

// body(i) for i in [0, n) split over the pool
template <typename F>
void pfor(Pool &P, long n, F body)
{
    P.run([&](int t) {
        long lo, hi;
        P.range(n, t, lo, hi);
        for (long i = lo; i < hi; i++) body(i);
    });
}

struct Ctx {
    Pool *P;
    int n;
    const int *rp, *ci;
    const double *v;
    const int *lrp, *lci, *urp, *uci;
    const double *lv, *dinv, *uv;
    std::vector<double> part;
};

double dot(Ctx &c, const double *x, const double *y)
{
    const long n = c.n, nb = (n + ORCMT_DOT_BLOCK - 1) / ORCMT_DOT_BLOCK;
    c.part.assign(nb, 0.0);
    pfor(*c.P, nb, [&](long b) {
        const long k1 = std::min(n, (b + 1) * ORCMT_DOT_BLOCK);
        double s = 0.0;
        for (long k = b * ORCMT_DOT_BLOCK; k < k1; k++) s += x[k] * y[k];
        c.part[b] = s;
    });
    double s = 0.0;
    for (long b = 0; b < nb; b++) s += c.part[b];
    return s;
}

void axpy(Pool &P, int n, double a, const double *x, double *y)
{
    pfor(P, n, [&](long i) { y[i] = y[i] + a * x[i]; });
}

void scal(Pool &P, int n, double a, double *x)
{
    pfor(P, n, [&](long i) { x[i] = a * x[i]; });
}

void copy(Pool &P, int n, const double *x, double *y)
{
    pfor(P, n, [&](long i) { y[i] = x[i]; });
}

// y = A x (CSR order within each row)
void spmv(const Ctx &c, const double *x, double *y)
{
    pfor(*c.P, c.n, [&](long i) {
        double r = 0.0;
        for (int k = c.rp[i]; k < c.rp[i + 1]; k++) r = r + c.v[k] * x[c.ci[k]];
        y[i] = r;
    });
}

// y = b - A x
void bmax(const Ctx &c, const double *b, const double *x, double *y)
{
    pfor(*c.P, c.n, [&](long i) {
        double r = b[i];
        for (int k = c.rp[i]; k < c.rp[i + 1]; k++) r = r - c.v[k] * x[c.ci[k]];
        y[i] = r;
    });
}

// y = (LU)^-1 x, sequential (hip/HostMatrix/HostMatrixCSR.cpp:385-409)
void lusolve(const Ctx &c, const double *x, double *y)
{
    const int n = c.n;
    for (int i = 0; i < n; i++) {
        double sum = x[i];
        for (int ii = c.lrp[i]; ii < c.lrp[i + 1]; ii++) sum -= y[c.lci[ii]] * c.lv[ii];
        y[i] = sum;
    }
    for (int i = 0; i < n; i++) y[i] *= c.dinv[i];
    for (int i = n - 1; i >= 0; i--) {
        double sum = y[i];
        for (int ii = c.urp[i + 1] - 1; ii >= c.urp[i]; ii--) sum -= y[c.uci[ii]] * c.uv[ii];
        y[i] = sum;
    }
}

}  // namespace

// Returns the number of iterations run (the reference's usediter + 1), or -1
// for bad arguments.  sol holds x0 on entry and the solution on exit;
// *final_rsm receives the last relative residual.
extern "C" int orcmt_bicgstab(int n, const int *rp, const int *ci, const double *v, const int *lrp, const int *lci,
                              const double *lv, const double *dinv, const int *urp, const int *uci, const double *uv,
                              const double *rhs, double *sol, double tol, int maxiter, int threads,
                              double *final_rsm)
{
    if (n <= 0 || !rp || !ci || !v || !lrp || !dinv || !urp || !rhs || !sol || maxiter < 1) return -1;
    Pool P(threads > 0 ? threads : (int)std::max(1u, std::thread::hardware_concurrency()));
    Ctx c{&P, n, rp, ci, v, lrp, lci, urp, uci, lv, dinv, uv, {}};
    std::vector<double> zk(n, 0.0), phi(n), res(n), pk(n, 0.0), uk(n, 0.0), vk(n, 0.0), sk(n, 0.0), reso(n);
    const double small = 1e-20;
    double alpha = 1.0, beto = 1.0, gama = 1.0, rsm = 1.0;
    copy(P, n, sol, phi.data());
    bmax(c, rhs, phi.data(), res.data());
    const double res0 = std::sqrt(dot(c, res.data(), res.data()));
    copy(P, n, res.data(), reso.data());
    int it = 0;
    for (; it < maxiter; it++) {
        const double beta = dot(c, res.data(), reso.data());
        const double omega = (beta * gama) / (alpha * beto + small);
        beto = beta;
        axpy(P, n, -alpha, uk.data(), pk.data());
        scal(P, n, omega, pk.data());
        axpy(P, n, 1.0, res.data(), pk.data());
        lusolve(c, pk.data(), zk.data());
        spmv(c, zk.data(), uk.data());
        gama = beta / (dot(c, uk.data(), reso.data()) + small);
        copy(P, n, res.data(), sk.data());
        axpy(P, n, -gama, uk.data(), sk.data());
        lusolve(c, sk.data(), zk.data());
        spmv(c, zk.data(), vk.data());
        const double t0 = dot(c, vk.data(), sk.data()), t1 = dot(c, vk.data(), vk.data());
        alpha = t0 / (t1 + small);
        axpy(P, n, gama, pk.data(), phi.data());
        axpy(P, n, alpha, sk.data(), phi.data());
        copy(P, n, sk.data(), res.data());
        axpy(P, n, -alpha, vk.data(), res.data());
        rsm = std::sqrt(dot(c, res.data(), res.data())) / (res0 + small);
        if (rsm < tol) {
            it++;
            break;
        }
    }
    lusolve(c, phi.data(), sol);
    if (final_rsm) *final_rsm = rsm;
    return it;
}
