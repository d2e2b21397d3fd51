// The DIF arithmetic of the xTGSNA kernels (real and complex) compiled for the CPU (test harness, not a
// product path): xtgevc3_b200/csrc/tgsna_dif.cuh and tgexc_real_blocks.cuh are host and
// device code, so the estimate the GPU kernel computes per eigenvalue (reorder a copy, then
// xTGSYL's Frobenius-norm estimate) can be compared with LAPACK D/STGSNA on a machine
// without a GPU.  Built by tests/test_tgsna_dif_host.py with g++ into tests/_build.
#include <barrier>
#include <thread>
#include <vector>

#include "../xtgevc3_b200/csrc/tgsna_dif.cuh"
#include "../xtgevc3_b200/csrc/tgsna_dif_cplx.cuh"

using namespace xtg::rb;

namespace {

// DTGSNA's DIF for every selected eigenvalue (howmny 'A' or 'S' with select), dif[0 .. m)
template <class R>
int dif_all(char howmny, const int *select, int n, const R *A, int lda, const R *B, int ldb, R *dif, int mm, int *m)
{
    auto a = [&](int i, int k) { return A[(size_t)i + (size_t)k * lda]; };
    auto b = [&](int i, int k) { return B[(size_t)i + (size_t)k * ldb]; };
    std::vector<R> wa((size_t)n * n), wb((size_t)n * n), c(2 * (size_t)n), f(2 * (size_t)n);
    std::vector<int> starts(n / 2 + 4);
    int ks = 0;
    for (int k = 0; k < n;) {
        const bool pair = k + 1 < n && a(k + 1, k) != R(0);
        const bool sel = howmny == 'A' || (select[k] != 0 || (pair && select[k + 1] != 0));
        if (sel) {
            if (ks + (pair ? 2 : 1) > mm) return -15;
            R d;
            if (n == 1) {
                d = lapy2(a(0, 0), b(0, 0));
            } else {
                R cond = R(0);
                if (pair) cond = pair_cond(a(k, k), a(k + 1, k), a(k, k + 1), a(k + 1, k + 1), b(k, k), b(k + 1, k),
                                           b(k, k + 1), b(k + 1, k + 1));
                for (int j = 0; j < n; j++)
                    for (int i = 0; i < n; i++) {
                        wa[i + (size_t)j * n] = a(i, j);
                        wb[i + (size_t)j * n] = b(i, j);
                    }
                Pencil<R> p{n, 0, 0, wa.data(), wb.data(), nullptr, nullptr, n, n, 1, 1};
                int ifst = k + 1, ilst = 1;
                if (tgexc_serial(p, ifst, ilst) > 0) {
                    d = R(0);
                } else {
                    const int n1 = wa[1] != R(0) ? 2 : 1;
                    d = (n - n1 == 0) ? cond
                                      : dif_reordered_serial(n, wa.data(), wb.data(), n, c.data(), f.data(), n,
                                                             starts.data());
                    if (pair && n - n1 > 0) d = xmin(d, cond);
                }
            }
            dif[ks] = d;
            if (pair) dif[ks + 1] = d;
            ks += pair ? 2 : 1;
        }
        k += pair ? 2 : 1;
    }
    *m = ks;
    return 0;
}

// ZTGSNA's DIF for every selected eigenvalue (complex A, B interleaved)
template <class R>
int zdif_all(char howmny, const int *select, int n, const R *A_, const R *B_, R *dif, int mm, int *m)
{
    const zc<R> *A = reinterpret_cast<const zc<R> *>(A_), *B = reinterpret_cast<const zc<R> *>(B_);
    std::vector<zc<R>> wa((size_t)n * n), wb((size_t)n * n), c(n), f(n);
    std::vector<int> starts(n / 2 + 4);
    int ks = 0;
    for (int k = 0; k < n; k++) {
        if (howmny != 'A' && !select[k]) continue;
        if (ks >= mm) return -15;
        dif[ks++] = zdif_serial(n, A, n, B, n, k, wa.data(), wb.data(), c.data(), f.data(), starts.data());
    }
    *m = ks;
    return 0;
}

// The CTA context of the kernel bodies on host threads: one std::thread per GPU thread, the
// CTA barrier a std::barrier.  Emulated CTAs run one after another.
struct CtaHost {
    int t, n, b, nb;
    std::barrier<> *bar;
    int tid() const { return t; }
    int nth() const { return n; }
    int cta() const { return b; }
    int ncta() const { return nb; }
    void sync() const { bar->arrive_and_wait(); }
};

// the selected blocks as the kernels take them (xTGSNA's selection rule)
template <class E, class IsPair>
std::vector<DifItem> dif_items(char howmny, const int *select, int n, IsPair is_pair, int *m)
{
    std::vector<DifItem> items;
    int ks = 0;
    for (int k = 0; k < n;) {
        const bool pair = is_pair(k);
        if (howmny == 'A' || select[k] != 0 || (pair && select[k + 1] != 0)) {
            items.push_back(DifItem{k, ks, pair ? 1 : 0});
            ks += pair ? 2 : 1;
        }
        k += pair ? 2 : 1;
    }
    *m = ks;
    return items;
}

template <class Body>
void run_grid(int nth, int grid, Body body)
{
    for (int b = 0; b < grid; b++) {
        std::barrier<> bar(nth);
        std::vector<std::thread> th;
        for (int t = 0; t < nth; t++) th.emplace_back([&, t] { body(CtaHost{t, nth, b, grid, &bar}); });
        for (auto &x : th) x.join();
    }
}

}  // namespace

extern "C" {

// the real DIF kernel's body (rb::dif_cta) on nth host threads per CTA and grid CTAs; returns
// the kernel's error flag
int threads_ddif(int nth, int grid, char howmny, const int *select, int n, const double *A, const double *B,
                 double *dif, int *m)
{
    auto items = dif_items<double>(howmny, select, n, [&](int k) { return k + 1 < n && A[k + 1 + (size_t)k * n] != 0.0; }, m);
    const size_t per = dif_work_elems(n);
    std::vector<double> work(per * grid);
    int err = 0;
    std::vector<DifShared<double>> sh(grid);
    run_grid(nth, grid, [&](const CtaHost &c) {
        dif_cta(c, sh[c.b], n, A, n, B, n, items.data(), (int)items.size(), dif, work.data(), per, &err);
    });
    return err;
}

// the complex DIF kernel's body (rb::zdif_cta) likewise
int threads_zdif(int nth, int grid, char howmny, const int *select, int n, const double *A, const double *B,
                 double *dif, int *m)
{
    auto items = dif_items<zc<double>>(howmny, select, n, [](int) { return false; }, m);
    const size_t per = zdif_work_elems(n);
    std::vector<zc<double>> work(per * grid);
    std::vector<ZDifShared<double>> sh(grid);
    run_grid(nth, grid, [&](const CtaHost &c) {
        zdif_cta(c, sh[c.b], n, reinterpret_cast<const zc<double> *>(A), n, reinterpret_cast<const zc<double> *>(B), n,
                 items.data(), (int)items.size(), dif, work.data(), per);
    });
    return 0;
}


int host_zdif(char howmny, const int *select, int n, const double *A, const double *B, double *dif, int mm, int *m)
{
    return zdif_all(howmny, select, n, A, B, dif, mm, m);
}

int host_cdif(char howmny, const int *select, int n, const float *A, const float *B, float *dif, int mm, int *m)
{
    return zdif_all(howmny, select, n, A, B, dif, mm, m);
}


int host_ddif(char howmny, const int *select, int n, const double *A, int lda, const double *B, int ldb, double *dif,
              int mm, int *m)
{
    return dif_all(howmny, select, n, A, lda, B, ldb, dif, mm, m);
}

int host_sdif(char howmny, const int *select, int n, const float *A, int lda, const float *B, int ldb, float *dif,
              int mm, int *m)
{
    return dif_all(howmny, select, n, A, lda, B, ldb, dif, mm, m);
}

// the estimate alone, on a pencil whose first block is the eigenvalue's (already reordered)
double host_ddif_reordered(int n, const double *A, const double *B)
{
    std::vector<double> c(2 * (size_t)n), f(2 * (size_t)n);
    std::vector<int> starts(n / 2 + 4);
    return dif_reordered_serial(n, A, B, n, c.data(), f.data(), n, starts.data());
}

// a complex pair's own bound from its 2x2 block (column-major a[4], b[4])
double host_dpair_cond(const double *a, const double *b)
{
    return pair_cond(a[0], a[1], a[2], a[3], b[0], b[1], b[2], b[3]);
}

}  // extern "C"
