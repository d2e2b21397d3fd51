// The QZ kernels' bodies (xtgevc3_b200/csrc/qz_cplx.cuh: rb::zgges_cta, qz_real.cuh:
// rb::dgges_cta) compiled for the CPU (test harness, not a product path): on one thread, and
// on host threads with a std::barrier for the CTA barrier, so that the generalized Schur
// forms they compute can be checked without a GPU.  Built by tests/test_qz_host.py with g++ into tests/_build.
#include <barrier>
#include <thread>
#include <vector>

#include "../xtgevc3_b200/csrc/qz_real.cuh"

using namespace xtg::rb;

namespace {

struct CtaHost {
    int t, n;
    std::barrier<> *bar;
    int tid() const { return t; }
    int nth() const { return n; }
    int cta() const { return 0; }
    int ncta() const { return 1; }
    void sync() const { bar->arrive_and_wait(); }
};

template <class R>
int run(int nth, int wantq, int wantz, int n, R *A, R *B, R *Q, R *Z)
{
    QzPencil<R> p{n,
                  wantq,
                  wantz,
                  reinterpret_cast<zc<R> *>(A),
                  reinterpret_cast<zc<R> *>(B),
                  reinterpret_cast<zc<R> *>(Q),
                  reinterpret_cast<zc<R> *>(Z),
                  n,
                  n,
                  n,
                  n};
    int info = 0;
    std::barrier<> bar(nth);
    std::vector<std::thread> th;
    for (int t = 0; t < nth; t++)
        th.emplace_back([&, t] {
            const int i = zgges_cta(CtaHost{t, nth, &bar}, p);
            if (t == 0) info = i;
        });
    for (auto &x : th) x.join();
    return info;
}

template <class R>
int run_real(int nth, int wantq, int wantz, int n, R *A, R *B, R *Q, R *Z, R *ar, R *ai, R *be)
{
    QzPencilR<R> p{n, wantq, wantz, A, B, Q, Z, n, n, n, n, ar, ai, be};
    int info = 0;
    std::barrier<> bar(nth);
    std::vector<std::thread> th;
    for (int t = 0; t < nth; t++)
        th.emplace_back([&, t] {
            const int i = dgges_cta(CtaHost{t, nth, &bar}, p);
            if (t == 0) info = i;
        });
    for (auto &x : th) x.join();
    return info;
}

}  // namespace

extern "C" {

// real: n x n, leading dimension n; alphar, alphai, beta n each; returns INFO
int host_dgges(int nth, int wantq, int wantz, int n, double *A, double *B, double *Q, double *Z, double *ar, double *ai,
               double *be)
{
    return run_real(nth, wantq, wantz, n, A, B, Q, Z, ar, ai, be);
}

int host_sgges(int nth, int wantq, int wantz, int n, float *A, float *B, float *Q, float *Z, float *ar, float *ai,
               float *be)
{
    return run_real(nth, wantq, wantz, n, A, B, Q, Z, ar, ai, be);
}


// complex arrays interleaved, n x n, leading dimension n; returns INFO
int host_zgges(int nth, int wantq, int wantz, int n, double *A, double *B, double *Q, double *Z)
{
    return run(nth, wantq, wantz, n, A, B, Q, Z);
}

int host_cgges(int nth, int wantq, int wantz, int n, float *A, float *B, float *Q, float *Z)
{
    return run(nth, wantq, wantz, n, A, B, Q, Z);
}

}  // extern "C"
