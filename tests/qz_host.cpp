// The QZ kernels' bodies (xtgevc3_b200/csrc/qz_cplx.cuh: rb::zgges_cta, qz_real.cuh:
// rb::dgges_cta) and the reordering kernels' bodies (tgsen.cuh: rb::tgsen_real_cta,
// rb::tgsen_cplx_cta, with xGGES's SDIM check) compiled for the CPU (test harness, not a product path): on one thread, and
// on host threads with a std::barrier for the CTA barrier, so that the generalized Schur
// forms they compute can be checked without a GPU.  Built by tests/test_qz_host.py with g++ into tests/_build.
#include <barrier>
#include <thread>
#include <vector>

#include "../xtgevc3_b200/csrc/qz_real.cuh"
#include "../xtgevc3_b200/csrc/tgsen.cuh"
#include "../xtgevc3_b200/csrc/tgsyl.cuh"
#include "../xtgevc3_b200/csrc/gges_scale.h"
#include "../xtgevc3_b200/csrc/ggbal.cuh"

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

template <class R>
int run_tgsen_real(int nth, int wantq, int wantz, int n, R *A, R *B, R *Q, R *Z, const int *sel, R *ar, R *ai, R *be)
{
    Pencil<R> p{n, wantq, wantz, A, B, wantq ? Q : A, wantz ? Z : A, n, n, n, n};
    WalkShared<R> sh{};
    int info = 0;
    std::barrier<> bar(nth);
    std::vector<std::thread> th;
    for (int t = 0; t < nth; t++)
        th.emplace_back([&, t] {
            const int i = tgsen_real_cta(CtaHost{t, nth, &bar}, sh, p, sel, ar, ai, be);
            if (t == 0) info = i;
        });
    for (auto &x : th) x.join();
    return info;
}

template <class R>
int run_tgsen_cplx(int nth, int wantq, int wantz, int n, R *A, R *B, R *Q, R *Z, const int *sel, R *al, R *be)
{
    using C = zc<R>;
    C *a = reinterpret_cast<C *>(A), *b = reinterpret_cast<C *>(B);
    ZPencil<R> p{n, wantq, wantz, a, b, wantq ? reinterpret_cast<C *>(Q) : a, wantz ? reinterpret_cast<C *>(Z) : a,
                 n, n, n, n};
    ZSortShared<R> sh{};
    int info = 0;
    std::barrier<> bar(nth);
    std::vector<std::thread> th;
    for (int t = 0; t < nth; t++)
        th.emplace_back([&, t] {
            const int i = tgsen_cplx_cta(CtaHost{t, nth, &bar}, sh, p, sel, reinterpret_cast<C *>(al),
                                         reinterpret_cast<C *>(be));
            if (t == 0) info = i;
        });
    for (auto &x : th) x.join();
    return info;
}

template <class R>
int run_tgsyl(int nth, int ijob, int m, int n, const R *A, const R *B, R *C, const R *D, const R *E, R *F, R *scale,
              R *dif)
{
    SylvShared<R> sh{};
    SylvG<R> &y = sh.y;
    y.m = m;
    y.n = n;
    y.A = A;
    y.D = D;
    y.B = B;
    y.E = E;
    y.lda = y.ldd = y.ldc = y.ldf = m;
    y.ldb = y.lde = n;
    y.C = C;
    y.F = F;
    std::vector<int> cuts(m / 2 + n / 2 + 4);
    std::vector<R> work(2 * (size_t)m * n);
    std::barrier<> bar(nth);
    std::vector<std::thread> th;
    for (int t = 0; t < nth; t++)
        th.emplace_back([&, t] { tgsyl_cta(CtaHost{t, nth, &bar}, sh, ijob, cuts.data(), work.data(), dif); });
    for (auto &x : th) x.join();
    *scale = sh.scale;
    return sh.info;
}

template <class R>
int run_tgsen_full(int nth, int ijob, int n, R *A, R *B, R *Q, R *Z, const int *sel, R *ar, R *ai, R *be, R *est,
                   int *m)
{
    Pencil<R> p{n, 1, 1, A, B, Q, Z, n, n, n, n};
    WalkShared<R> shw{};
    SylvShared<R> shs{};
    std::vector<R> work((size_t)n * n + 2);
    std::vector<int> iwork((size_t)n * n / 2 + 2), cuts(n / 2 + 4);
    int info = 0;
    std::barrier<> bar(nth);
    std::vector<std::thread> th;
    for (int t = 0; t < nth; t++)
        th.emplace_back([&, t] {
            const int i = tgsen_real_full_cta(CtaHost{t, nth, &bar}, shw, shs, p, sel, ijob, ar, ai, be, work.data(),
                                              iwork.data(), cuts.data(), est, m);
            if (t == 0) info = i;
        });
    for (auto &x : th) x.join();
    return info;
}

template <class R>
int run_ztgsyl(int nth, int ijob, int m, int n, const R *A, const R *B, R *C, const R *D, const R *E, R *F, R *scale,
               R *dif)
{
    using Cx = zc<R>;
    ZSylvShared<R> sh{};
    ZSylvG<R> &y = sh.y;
    y.m = m;
    y.n = n;
    y.A = reinterpret_cast<const Cx *>(A);
    y.D = reinterpret_cast<const Cx *>(D);
    y.B = reinterpret_cast<const Cx *>(B);
    y.E = reinterpret_cast<const Cx *>(E);
    y.lda = y.ldd = y.ldc = y.ldf = m;
    y.ldb = y.lde = n;
    y.C = reinterpret_cast<Cx *>(C);
    y.F = reinterpret_cast<Cx *>(F);
    std::vector<int> cuts(m / 2 + n / 2 + 4);
    std::vector<Cx> work(2 * (size_t)m * n);
    std::barrier<> bar(nth);
    std::vector<std::thread> th;
    for (int t = 0; t < nth; t++)
        th.emplace_back([&, t] { ztgsyl_cta(CtaHost{t, nth, &bar}, sh, ijob, cuts.data(), work.data(), dif); });
    for (auto &x : th) x.join();
    *scale = sh.scale;
    return sh.info;
}

template <class R>
int run_ztgsen_full(int nth, int ijob, int n, R *A, R *B, R *Q, R *Z, const int *sel, R *al, R *be, R *est, int *m)
{
    using Cx = zc<R>;
    Cx *a = reinterpret_cast<Cx *>(A), *b = reinterpret_cast<Cx *>(B);
    ZPencil<R> p{n, 1, 1, a, b, reinterpret_cast<Cx *>(Q), reinterpret_cast<Cx *>(Z), n, n, n, n};
    ZSortShared<R> shs{};
    ZSylvShared<R> shy{};
    std::vector<Cx> work((size_t)n * n + 2);
    std::vector<int> cuts(n / 2 + 4);
    int info = 0;
    std::barrier<> bar(nth);
    std::vector<std::thread> th;
    for (int t = 0; t < nth; t++)
        th.emplace_back([&, t] {
            const int i = tgsen_cplx_full_cta(CtaHost{t, nth, &bar}, shs, shy, p, sel, ijob, reinterpret_cast<Cx *>(al),
                                              reinterpret_cast<Cx *>(be), work.data(), cuts.data(), est, m);
            if (t == 0) info = i;
        });
    for (auto &x : th) x.join();
    return info;
}

template <class R>
int run_tgsyl_t(int nth, int m, int n, const R *A, const R *B, R *C, const R *D, const R *E, R *F, R *scale)
{
    SylvShared<R> sh{};
    SylvG<R> &y = sh.y;
    y.m = m;
    y.n = n;
    y.A = A;
    y.D = D;
    y.B = B;
    y.E = E;
    y.lda = y.ldd = y.ldc = y.ldf = m;
    y.ldb = y.lde = n;
    y.C = C;
    y.F = F;
    std::vector<int> cuts(m / 2 + n / 2 + 4);
    std::barrier<> bar(nth);
    std::vector<std::thread> th;
    for (int t = 0; t < nth; t++) th.emplace_back([&, t] { tgsyl_t_cta(CtaHost{t, nth, &bar}, sh, cuts.data()); });
    for (auto &x : th) x.join();
    *scale = sh.scale;
    return sh.info;
}

template <class R>
int run_ztgsyl_c(int nth, int m, int n, const R *A, const R *B, R *C, const R *D, const R *E, R *F, R *scale)
{
    using Cx = zc<R>;
    ZSylvShared<R> sh{};
    ZSylvG<R> &y = sh.y;
    y.m = m;
    y.n = n;
    y.A = reinterpret_cast<const Cx *>(A);
    y.D = reinterpret_cast<const Cx *>(D);
    y.B = reinterpret_cast<const Cx *>(B);
    y.E = reinterpret_cast<const Cx *>(E);
    y.lda = y.ldd = y.ldc = y.ldf = m;
    y.ldb = y.lde = n;
    y.C = reinterpret_cast<Cx *>(C);
    y.F = reinterpret_cast<Cx *>(F);
    std::vector<int> cuts(m / 2 + n / 2 + 4);
    std::barrier<> bar(nth);
    std::vector<std::thread> th;
    for (int t = 0; t < nth; t++) th.emplace_back([&, t] { ztgsyl_c_cta(CtaHost{t, nth, &bar}, sh, cuts.data()); });
    for (auto &x : th) x.join();
    *scale = sh.scale;
    return sh.info;
}

template <class E, class R>
int run_ggbal(int nth, int n, E *A, E *B, R *ls, R *rs, int *ilo, int *ihi)
{
    BalPencil<E> p{n, A, B, n, n};
    BalShared sh{};
    std::vector<int> red(2 * (size_t)nth);
    std::barrier<> bar(nth);
    std::vector<std::thread> th;
    for (int t = 0; t < nth; t++)
        th.emplace_back([&, t] { ggbal_cta(CtaHost{t, nth, &bar}, sh, p, ls, rs, ilo, ihi, red.data()); });
    for (auto &x : th) x.join();
    return 0;
}

template <class E, class R>
int run_ggbak(int nth, int n, int ilo, int ihi, const R *scale, E *V, int m = -1)
{
    std::barrier<> bar(nth);
    std::vector<std::thread> th;
    for (int t = 0; t < nth; t++)
        th.emplace_back([&, t] { ggbak_cta(CtaHost{t, nth, &bar}, n, ilo, ihi, scale, V, n, m); });
    for (auto &x : th) x.join();
    return 0;
}

// SELCTG from flags: the test passes the selection that LAPACK's SELCTG made, one flag per
// eigenvalue in order, and the check reads them back in the same order
struct FlagSel {
    const int *flags;
    mutable int i = 0;
    template <class T>
    int operator()(const T *, const T *, const T *) const { return flags[i++]; }
    template <class T>
    int operator()(const T *, const T *) const { return flags[i++]; }
};

}  // namespace

extern "C" {

// xTGSEN (IJOB = 0) bodies: n x n, leading dimension n; returns INFO
int host_dtgsen0(int nth, int wantq, int wantz, int n, double *A, double *B, double *Q, double *Z, const int *sel,
                 double *ar, double *ai, double *be)
{
    return run_tgsen_real(nth, wantq, wantz, n, A, B, Q, Z, sel, ar, ai, be);
}

int host_stgsen0(int nth, int wantq, int wantz, int n, float *A, float *B, float *Q, float *Z, const int *sel,
                 float *ar, float *ai, float *be)
{
    return run_tgsen_real(nth, wantq, wantz, n, A, B, Q, Z, sel, ar, ai, be);
}

int host_ztgsen0(int nth, int wantq, int wantz, int n, double *A, double *B, double *Q, double *Z, const int *sel,
                 double *al, double *be)
{
    return run_tgsen_cplx(nth, wantq, wantz, n, A, B, Q, Z, sel, al, be);
}

int host_ctgsen0(int nth, int wantq, int wantz, int n, float *A, float *B, float *Q, float *Z, const int *sel,
                 float *al, float *be)
{
    return run_tgsen_cplx(nth, wantq, wantz, n, A, B, Q, Z, sel, al, be);
}

// DTGSEN (IJOB 0, 1, 2, 4) body with Q and Z: est = PL, PR, DIF(1), DIF(2); returns INFO
int host_dtgsen(int nth, int ijob, int n, double *A, double *B, double *Q, double *Z, const int *sel, double *ar,
                double *ai, double *be, double *est, int *m)
{
    return run_tgsen_full(nth, ijob, n, A, B, Q, Z, sel, ar, ai, be, est, m);
}

int host_stgsen(int nth, int ijob, int n, float *A, float *B, float *Q, float *Z, const int *sel, float *ar, float *ai,
                float *be, float *est, int *m)
{
    return run_tgsen_full(nth, ijob, n, A, B, Q, Z, sel, ar, ai, be, est, m);
}

// xTGSYL (TRANS = 'N', IJOB 0 / 1 / 3) body: A, D m x m, B, E n x n, C, F m x n (leading
// dimensions m, n, m); returns INFO
int host_dtgsyl(int nth, int ijob, int m, int n, const double *A, const double *B, double *C, const double *D,
                const double *E, double *F, double *scale, double *dif)
{
    return run_tgsyl(nth, ijob, m, n, A, B, C, D, E, F, scale, dif);
}

int host_stgsyl(int nth, int ijob, int m, int n, const float *A, const float *B, float *C, const float *D,
                const float *E, float *F, float *scale, float *dif)
{
    return run_tgsyl(nth, ijob, m, n, A, B, C, D, E, F, scale, dif);
}

// ZTGSEN (IJOB 0, 1, 2, 4) body with Q and Z (interleaved complex arrays); est = PL, PR,
// DIF(1), DIF(2); returns INFO
int host_ztgsen(int nth, int ijob, int n, double *A, double *B, double *Q, double *Z, const int *sel, double *al,
                double *be, double *est, int *m)
{
    return run_ztgsen_full(nth, ijob, n, A, B, Q, Z, sel, al, be, est, m);
}

int host_ctgsen(int nth, int ijob, int n, float *A, float *B, float *Q, float *Z, const int *sel, float *al, float *be,
                float *est, int *m)
{
    return run_ztgsen_full(nth, ijob, n, A, B, Q, Z, sel, al, be, est, m);
}

// D/STGSYL with TRANS = 'T' body
int host_dtgsyl_t(int nth, int m, int n, const double *A, const double *B, double *C, const double *D,
                  const double *E, double *F, double *scale)
{
    return run_tgsyl_t(nth, m, n, A, B, C, D, E, F, scale);
}

int host_stgsyl_t(int nth, int m, int n, const float *A, const float *B, float *C, const float *D, const float *E,
                  float *F, float *scale)
{
    return run_tgsyl_t(nth, m, n, A, B, C, D, E, F, scale);
}

// Z/CTGSYL with TRANS = 'C' body
int host_ztgsyl_c(int nth, int m, int n, const double *A, const double *B, double *C, const double *D,
                  const double *E, double *F, double *scale)
{
    return run_ztgsyl_c(nth, m, n, A, B, C, D, E, F, scale);
}

int host_ctgsyl_c(int nth, int m, int n, const float *A, const float *B, float *C, const float *D, const float *E,
                  float *F, float *scale)
{
    return run_ztgsyl_c(nth, m, n, A, B, C, D, E, F, scale);
}

// Z/CTGSYL body (interleaved complex arrays)
int host_ztgsyl(int nth, int ijob, int m, int n, const double *A, const double *B, double *C, const double *D,
                const double *E, double *F, double *scale, double *dif)
{
    return run_ztgsyl(nth, ijob, m, n, A, B, C, D, E, F, scale, dif);
}

int host_ctgsyl(int nth, int ijob, int m, int n, const float *A, const float *B, float *C, const float *D,
                const float *E, float *F, float *scale, float *dif)
{
    return run_ztgsyl(nth, ijob, m, n, A, B, C, D, E, F, scale, dif);
}

// xLASCL's steps (gges_scale.h) applied to x[0, count): returns the number of factors
int host_dlascl(double cfrom, double cto, int count, double *x)
{
    double mul[8];
    const int k = xtg::gs::lascl_steps(cfrom, cto, mul);
    xtg::gs::lascl_apply(k, mul, x, (size_t)count);
    return k;
}

// xGGES's scaling decision for a norm (gges_scale.h): 1 and *to when the pencil is scaled
int host_gges_needs_scaling(double nrm, double *to) { return xtg::gs::needs_scaling(nrm, to) ? 1 : 0; }

// xGGES's scaling back on host arrays (the steps of gges_scale_out without the device):
// DGGES's pair guard, the eigenvalues, A upper Hessenberg (real) / upper triangular (complex,
// cplx = 1: interleaved arrays), B upper triangular
int host_gges_scale_out(int cplx, int n, double *A, double *B, double *ev0, double *ev1, double *ev2, int ilascl,
                        double anrm, double anrmto, int ilbscl, double bnrm, double bnrmto)
{
    const int cw = cplx ? 2 : 1;
    if (!cplx && (ilascl || ilbscl)) {
        std::vector<double> aii(n), aii1(n), bii(n);
        for (int i = 0; i < n; i++) {
            aii[i] = A[i + (size_t)i * n];
            aii1[i] = i + 1 < n ? A[i + (size_t)(i + 1) * n] : 0.0;
            bii[i] = B[i + (size_t)i * n];
        }
        xtg::gs::pair_guard(n, ilascl != 0, anrm, anrmto, ilbscl != 0, bnrm, bnrmto, aii.data(), aii1.data(),
                            bii.data(), ev0, ev1, ev2);
    }
    double f[8];
    for (int w = 0; w < 2; w++) {
        if (!(w == 0 ? ilascl : ilbscl)) continue;
        const int k = xtg::gs::lascl_steps(w == 0 ? anrmto : bnrmto, w == 0 ? anrm : bnrm, f);
        double *M = w == 0 ? A : B;
        const int kind = (w == 0 && !cplx) ? 2 : 1;
        for (int j = 0; j < n; j++)
            for (int i = 0; i < n; i++) {
                if ((kind == 1 && i > j) || (kind == 2 && i > j + 1)) continue;
                xtg::gs::lascl_apply(k, f, M + ((size_t)i + (size_t)j * n) * cw, cw);
            }
        if (w == 0) {
            xtg::gs::lascl_apply(k, f, ev0, (size_t)n * cw);
            if (!cplx) xtg::gs::lascl_apply(k, f, ev1, (size_t)n);
        } else {
            xtg::gs::lascl_apply(k, f, cplx ? ev1 : ev2, (size_t)n * cw);
        }
    }
    return 0;
}

// xGGBAL 'P' / xGGBAK 'P' bodies (d: real double, z: complex double, interleaved)
int host_dggbal(int nth, int n, double *A, double *B, double *ls, double *rs, int *ilo, int *ihi)
{
    return run_ggbal(nth, n, A, B, ls, rs, ilo, ihi);
}

int host_zggbal(int nth, int n, double *A, double *B, double *ls, double *rs, int *ilo, int *ihi)
{
    return run_ggbal(nth, n, reinterpret_cast<zc<double> *>(A), reinterpret_cast<zc<double> *>(B), ls, rs, ilo, ihi);
}

int host_dggbak(int nth, int n, int ilo, int ihi, const double *scale, double *V)
{
    return run_ggbak(nth, n, ilo, ihi, scale, V);
}

// V n x m (leading dimension n)
int host_dggbak_m(int nth, int n, int m, int ilo, int ihi, const double *scale, double *V)
{
    return run_ggbak(nth, n, ilo, ihi, scale, V, m);
}

int host_zggbak(int nth, int n, int ilo, int ihi, const double *scale, double *V)
{
    return run_ggbak(nth, n, ilo, ihi, scale, reinterpret_cast<zc<double> *>(V));
}

// xGGES's check: SELCTG's answers as flags in order; returns SDIM, *info as the check leaves it
int host_dgges_sdim(int n, const int *flags, const double *ar, const double *ai, const double *be, int *info)
{
    return gges_sdim_real(n, FlagSel{flags}, ar, ai, be, info);
}

int host_zgges_sdim(int n, const int *flags, const double *al, const double *be, int *info)
{
    return gges_sdim_cplx(n, FlagSel{flags}, reinterpret_cast<const zc<double> *>(al),
                          reinterpret_cast<const zc<double> *>(be), info);
}

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
