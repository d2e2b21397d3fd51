// The real reordering kernel's arithmetic compiled for the CPU (test harness, not a product
// path): xtgevc3_b200/csrc/tgexc_real_blocks.cuh is host and device code, so the swaps and the
// walk that the GPU kernel runs can be compared with LAPACK D/STGEX2 and D/STGEXC on a machine
// without a GPU; the kernel's own body (walk_cta) also runs here on host threads.  Built by
// tests/test_tgexc_blocks_host.py with g++ into tests/_build.
#include <barrier>
#include <thread>
#include <vector>

#include "../xtgevc3_b200/csrc/tgexc_real_blocks.cuh"

using namespace xtg::rb;

namespace {

template <class R>
Pencil<R> pencil(int wantq, int wantz, int n, R *A, int lda, R *B, int ldb, R *Q, int ldq, R *Z, int ldz)
{
    return Pencil<R>{n, wantq, wantz, A, B, Q, Z, lda, ldb, ldq, ldz};
}

// one swap at j1 (1-based) of blocks n1 above n2: 0 done, 1 rejected (xTGEX2's INFO)
template <class R>
int swap_one(const Pencil<R> &p, int j1, int n1, int n2)
{
    Swap<R> s;
    s.j1 = j1 - 1;
    s.n1 = n1;
    s.n2 = n2;
    swap_prepare(p, s);
    if (s.ok == 1)
        for (int ph = 0; ph < 3; ph++) swap_apply(p, s, ph, 0, 1);
    return s.ok == 0 ? 1 : 0;
}

// The CTA context of walk_cta on host threads: one std::thread per GPU thread, the CTA
// barrier a std::barrier.
struct CtaHost {
    int t, n;
    std::barrier<> *bar;
    int tid() const { return t; }
    int nth() const { return n; }
    int cta() const { return 0; }
    int ncta() const { return 1; }
    void sync() const { bar->arrive_and_wait(); }
};

// the reordering kernel's body (walk_cta) on nth host threads: INFO, ifst / ilst as the kernel
// reports them
template <class R>
int walk_threads(int nth, const Pencil<R> &p, int *ifst, int *ilst)
{
    WalkShared<R> sh{};
    std::barrier<> bar(nth);
    std::vector<std::thread> th;
    for (int t = 0; t < nth; t++) th.emplace_back([&, t] { walk_cta(CtaHost{t, nth, &bar}, sh, p, *ifst, *ilst); });
    for (auto &x : th) x.join();
    if (p.n > 1) {
        *ifst = sh.ifst;
        *ilst = sh.ilst;
    }
    return sh.info;
}

}  // namespace

extern "C" {

int threads_dtgexc(int nth, int wantq, int wantz, int n, double *A, int lda, double *B, int ldb, double *Q, int ldq,
                   double *Z, int ldz, int *ifst, int *ilst)
{
    return walk_threads(nth, pencil(wantq, wantz, n, A, lda, B, ldb, Q, ldq, Z, ldz), ifst, ilst);
}

int host_dtgexc(int wantq, int wantz, int n, double *A, int lda, double *B, int ldb, double *Q, int ldq, double *Z,
                int ldz, int *ifst, int *ilst)
{
    return tgexc_serial(pencil(wantq, wantz, n, A, lda, B, ldb, Q, ldq, Z, ldz), *ifst, *ilst);
}

int host_stgexc(int wantq, int wantz, int n, float *A, int lda, float *B, int ldb, float *Q, int ldq, float *Z,
                int ldz, int *ifst, int *ilst)
{
    return tgexc_serial(pencil(wantq, wantz, n, A, lda, B, ldb, Q, ldq, Z, ldz), *ifst, *ilst);
}

int host_dtgex2(int wantq, int wantz, int n, double *A, int lda, double *B, int ldb, double *Q, int ldq, double *Z,
                int ldz, int j1, int n1, int n2)
{
    return swap_one(pencil(wantq, wantz, n, A, lda, B, ldb, Q, ldq, Z, ldz), j1, n1, n2);
}

int host_stgex2(int wantq, int wantz, int n, float *A, int lda, float *B, int ldb, float *Q, int ldq, float *Z,
                int ldz, int j1, int n1, int n2)
{
    return swap_one(pencil(wantq, wantz, n, A, lda, B, ldb, Q, ldq, Z, ldz), j1, n1, n2);
}

}  // extern "C"
