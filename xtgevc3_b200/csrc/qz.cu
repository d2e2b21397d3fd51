// The generalized Schur form of a pencil on the GPU (LAPACK Z/C/D/SGGES), in xGGES's order:
// A and B scaled into range where their largest entries lie outside it (gges_scale.h;
// maxabs_kernel, lascl_kernel), balanced by permutations (ggbal.cuh: xGGBAL 'P'), the QZ step
// (rb::zgges_cta of qz_cplx.cuh or rb::dgges_cta of qz_real.cuh on one CTA; complex alpha =
// diag(S), beta = diag(T), real alphar / alphai / beta as DHGEQZ returns them), with SORT = 'S'
// the ordering (SELCTG on the host over the 2-3 n eigenvalue numbers read back, the
// reordering kernel of tgsen.cuh on one CTA), VSL / VSR permuted back (xGGBAK 'P'), the form
// and eigenvalues scaled back, and xGGES's check of the reordered eigenvalues (SDIM, INFO =
// n + 2 / n + 3) on the host.  Also here: xTGSEN with IJOB 0-5 (tgsen.cuh) and xTGSYL
// (tgsyl.cuh) as entry points of their own.  The stages are chains of dependent plane
// rotations, swaps or small systems, so one CTA runs each (the O(n) rows or columns of a step
// spread over its threads); the result stays on the device for the eigenvector solve that
// follows (xtgevc3_ztgevc3_dev).
#include "../../include/xtgevc3.h"
#include "common.cuh"
#include "engine.cuh"
#include "ggbal.cuh"
#include "gges_scale.h"
#include "qz_real.cuh"
#include "tgsen.cuh"

#include <algorithm>
#include <cctype>
#include <cstring>
#include <string>
#include <vector>

namespace xtg {
namespace {

constexpr int kQzThreads = 512;

template <class R>
__global__ void __launch_bounds__(kQzThreads, 1)
    zgges_kernel(rb::QzPencil<R> p, rb::zc<R> *alpha, rb::zc<R> *beta, int *info)
{
    const int i = rb::zgges_cta(rb::CtaDev{}, p);  // ends with a barrier
    for (int j = threadIdx.x; j < p.n; j += blockDim.x) {
        alpha[j] = p.A[j + (size_t)j * p.lda];
        beta[j] = p.B[j + (size_t)j * p.ldb];
    }
    if (threadIdx.x == 0) *info = i;
}

template <class R>
__global__ void __launch_bounds__(kQzThreads, 1) dgges_kernel(rb::QzPencilR<R> p, int *info)
{
    const int i = rb::dgges_cta(rb::CtaDev{}, p);
    if (threadIdx.x == 0) *info = i;
}

// The reordering kernels: rb::tgsen_real_cta / rb::tgsen_cplx_cta on one CTA; info: 0, 1 (a
// swap was rejected) or 3 (a walk reached its bound)
template <class R>
__global__ void __launch_bounds__(kQzThreads, 1)
    tgsen_real_kernel(rb::Pencil<R> p, const int *select, R *alphar, R *alphai, R *beta, int *info)
{
    __shared__ rb::WalkShared<R> sh;
    const int i = rb::tgsen_real_cta(rb::CtaDev{}, sh, p, select, alphar, alphai, beta);
    if (threadIdx.x == 0) *info = i;
}

// DTGSEN with IJOB 0 to 5 (rb::tgsen_real_full_cta): status = {INFO, M}; est = PL, PR,
// DIF(1), DIF(2); work 4 M (n - M) elements, iwork 2 M (n - M) ints, cuts n / 2 + 4 ints
template <class R>
__global__ void __launch_bounds__(kQzThreads, 1)
    tgsen_real_full_kernel(rb::Pencil<R> p, const int *select, int ijob, R *alphar, R *alphai, R *beta, R *work,
                           int *iwork, int *cuts, R *est, int *status)
{
    __shared__ rb::WalkShared<R> shw;
    __shared__ rb::SylvShared<R> shs;
    const int i = rb::tgsen_real_full_cta(rb::CtaDev{}, shw, shs, p, select, ijob, alphar, alphai, beta, work, iwork,
                                          cuts, est, status + 1);
    if (threadIdx.x == 0) status[0] = i;
}

// ZTGSEN with IJOB 0, 1, 2, 4 (rb::tgsen_cplx_full_cta): as tgsen_real_full_kernel
template <class R>
__global__ void __launch_bounds__(kQzThreads, 1)
    tgsen_cplx_full_kernel(rb::ZPencil<R> p, const int *select, int ijob, rb::zc<R> *alpha, rb::zc<R> *beta,
                           rb::zc<R> *work, int *cuts, R *est, int *status)
{
    __shared__ rb::ZSortShared<R> shs;
    __shared__ rb::ZSylvShared<R> shy;
    const int i =
        rb::tgsen_cplx_full_cta(rb::CtaDev{}, shs, shy, p, select, ijob, alpha, beta, work, cuts, est, status + 1);
    if (threadIdx.x == 0) status[0] = i;
}

// Z/CTGSYL (TRANS = 'N', IJOB 0, 1, 3: rb::ztgsyl_cta; trans: TRANS = 'C', rb::ztgsyl_c_cta):
// as tgsyl_kernel
template <class R>
__global__ void __launch_bounds__(kQzThreads, 1)
    ztgsyl_kernel(rb::ZSylvG<R> y, int trans, int ijob, int *cuts, rb::zc<R> *work, R *out, int *status)
{
    __shared__ rb::ZSylvShared<R> sh;
    if (threadIdx.x == 0) sh.y = y;
    __syncthreads();
    R dif = out[1];
    if (trans) rb::ztgsyl_c_cta(rb::CtaDev{}, sh, cuts);
    else rb::ztgsyl_cta(rb::CtaDev{}, sh, ijob, cuts, work, &dif);
    if (threadIdx.x == 0) {
        status[0] = sh.info;
        out[0] = sh.scale;
        out[1] = dif;
    }
}

// xTGSYL (TRANS = 'N' with IJOB 0, 1, 3: rb::tgsyl_cta; trans: TRANS = 'T', rb::tgsyl_t_cta):
// status = {INFO}, out = {SCALE, DIF}
template <class R>
__global__ void __launch_bounds__(kQzThreads, 1)
    tgsyl_kernel(rb::SylvG<R> y, int trans, int ijob, int *cuts, R *work, R *out, int *status)
{
    __shared__ rb::SylvShared<R> sh;
    if (threadIdx.x == 0) sh.y = y;
    __syncthreads();
    R dif = out[1];
    if (trans) rb::tgsyl_t_cta(rb::CtaDev{}, sh, cuts);
    else rb::tgsyl_cta(rb::CtaDev{}, sh, ijob, cuts, work, &dif);
    if (threadIdx.x == 0) {
        status[0] = sh.info;
        out[0] = sh.scale;
        out[1] = dif;
    }
}

template <class R>
__global__ void __launch_bounds__(kQzThreads, 1)
    tgsen_cplx_kernel(rb::ZPencil<R> p, const int *select, rb::zc<R> *alpha, rb::zc<R> *beta, int *info)
{
    __shared__ rb::ZSortShared<R> sh;
    const int i = rb::tgsen_cplx_cta(rb::CtaDev{}, sh, p, select, alpha, beta);
    if (threadIdx.x == 0) *info = i;
}

// ---- xGGES's scaling of the pencil (gges_scale.h) on the device ------------------------------

__device__ __forceinline__ double modulus_(double x) { return fabs(x); }
__device__ __forceinline__ double modulus_(float x) { return (double)fabsf(x); }
template <class R>
__device__ __forceinline__ double modulus_(rb::zc<R> x) { return (double)rb::cabs(x); }

// Largest modulus of the n x n matrix A (xLANGE 'M') as the bits of a non-negative double
// (integer order of those bits is their numeric order) into *bits; any NaN sets *nan
template <class E>
__global__ void __launch_bounds__(256) maxabs_kernel(const E *A, int lda, int n, unsigned long long *bits, int *nan)
{
    double mx = 0.0;
    int bad = 0;
    const size_t total = (size_t)n * n;
    for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < total; t += (size_t)gridDim.x * blockDim.x) {
        const double v = modulus_(A[(t % n) + (t / n) * (size_t)lda]);
        if (v != v) bad = 1;
        else if (v > mx) mx = v;
    }
    for (int o = 16; o > 0; o >>= 1) {
        mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
        bad |= __shfl_xor_sync(0xffffffffu, bad, o);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicMax(bits, (unsigned long long)__double_as_longlong(mx));
        if (bad) atomicExch(nan, 1);
    }
}

template <class R>
struct Muls {
    R f[8];
    int k;
};

__device__ __forceinline__ void scale_(double &x, double f) { x *= f; }
__device__ __forceinline__ void scale_(float &x, float f) { x *= f; }
template <class R>
__device__ __forceinline__ void scale_(rb::zc<R> &x, R f)
{
    x.re *= f;
    x.im *= f;
}

// xLASCL's multiplications of the entries of A in region kind (0 all, 1 upper triangle, 2 upper
// Hessenberg), factor after factor
template <class E, class R>
__global__ void __launch_bounds__(256) lascl_kernel(E *A, int lda, int n, int kind, Muls<R> m)
{
    const size_t total = (size_t)n * n;
    for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < total; t += (size_t)gridDim.x * blockDim.x) {
        const int i = (int)(t % n), j = (int)(t / n);
        if ((kind == 1 && i > j) || (kind == 2 && i > j + 1)) continue;
        E v = A[(size_t)i + (size_t)j * lda];
        for (int s = 0; s < m.k; s++) scale_(v, m.f[s]);
        A[(size_t)i + (size_t)j * lda] = v;
    }
}

// xGGBAL 'P' (rb::ggbal_cta): lscale, rscale n each; ilohi = {ILO, IHI}; red 2 kQzThreads ints
template <class E, class R>
__global__ void __launch_bounds__(kQzThreads, 1)
    ggbal_kernel(rb::BalPencil<E> p, R *lscale, R *rscale, int *ilohi, int *red)
{
    __shared__ rb::BalShared sh;
    rb::ggbal_cta(rb::CtaDev{}, sh, p, lscale, rscale, ilohi, ilohi + 1, red);
}

// xGGBAK 'P' (rb::ggbak_cta) of the Schur vectors V with xGGBAL's ILO, IHI and scale
template <class E, class R>
__global__ void __launch_bounds__(kQzThreads, 1) ggbak_kernel(int n, const int *ilohi, const R *scale, E *V, int ldv)
{
    rb::ggbak_cta(rb::CtaDev{}, n, ilohi[0], ilohi[1], scale, V, ldv);
}

// xGGBAK 'P' of an n x m V with host ILO, IHI (the entry point xtgevc3_*ggbak)
template <class E, class R>
__global__ void __launch_bounds__(kQzThreads, 1)
    ggbak_m_kernel(int n, int ilo, int ihi, const R *scale, E *V, int ldv, int m)
{
    rb::ggbak_cta(rb::CtaDev{}, n, ilo, ihi, scale, V, ldv, m);
}

// xGGES's permutation balancing around the QZ step: gges_balance_in permutes A and B (ILO, IHI,
// LSCALE, RSCALE stay on the device in bal), gges_balance_out permutes the rows of VSL / VSR
// back (after the ordering, before the scaling back, as xGGES)
template <class R>
struct GgesBalance {
    R *scale = nullptr;  // lscale (n), rscale (n)
    int *ints = nullptr;  // ILO, IHI, then the reduction scratch
};

template <class E, class R>
cudaError_t gges_balance_in(cudaStream_t st, int n, E *A, int lda, E *B, int ldb, GgesBalance<R> &bal)
{
    cudaError_t e = cudaMallocAsync(&bal.scale, 2 * (size_t)n * sizeof(R), st);
    if (e == cudaSuccess) e = cudaMallocAsync(&bal.ints, (2 + 2 * kQzThreads) * sizeof(int), st);
    if (e == cudaSuccess) e = cudaMemsetAsync(bal.scale, 0, 2 * (size_t)n * sizeof(R), st);
    if (e != cudaSuccess) return e;
    const rb::BalPencil<E> p{n, A, B, lda, ldb};
    ggbal_kernel<E, R><<<1, kQzThreads, 0, st>>>(p, bal.scale, bal.scale + n, bal.ints, bal.ints + 2);
    count_launches(1);
    return cudaGetLastError();
}

template <class E, class R>
cudaError_t gges_balance_out(cudaStream_t st, int n, E *VSL, int ldvsl, E *VSR, int ldvsr, const GgesBalance<R> &bal)
{
    cudaError_t e = cudaSuccess;
    if (VSL) {
        ggbak_kernel<E, R><<<1, kQzThreads, 0, st>>>(n, bal.ints, bal.scale, VSL, ldvsl);
        count_launches(1);
        e = cudaGetLastError();
    }
    if (VSR && e == cudaSuccess) {
        ggbak_kernel<E, R><<<1, kQzThreads, 0, st>>>(n, bal.ints, bal.scale + n, VSR, ldvsr);
        count_launches(1);
        e = cudaGetLastError();
    }
    return e;
}

template <class R>
void gges_balance_free(cudaStream_t st, GgesBalance<R> &bal)
{
    if (bal.scale) cudaFreeAsync(bal.scale, st);
    if (bal.ints) cudaFreeAsync(bal.ints, st);
    bal.scale = nullptr;
    bal.ints = nullptr;
}

// The scaling decisions of xGGES for one run
template <class R>
struct GgesScale {
    bool ilascl = false, ilbscl = false;
    R anrm = R(0), anrmto = R(0), bnrm = R(0), bnrmto = R(0);
};

constexpr int kScaleGrid = 4 * 148;

// xGGES's first step: the largest moduli of A and B; A, B scaled into [smlnum, bignum] where
// they lie outside it (a NaN anywhere leaves the pencil as it is, as xLANGE's NaN does)
template <class E, class R>
cudaError_t gges_scale_in(cudaStream_t st, int n, E *A, int lda, E *B, int ldb, GgesScale<R> &g)
{
    unsigned long long *d = nullptr;  // bits of |A|max, |B|max, then the two NaN flags
    cudaError_t e = cudaMallocAsync(&d, 3 * sizeof(unsigned long long), st);
    if (e != cudaSuccess) return e;
    unsigned long long h[3] = {0, 0, 0};
    e = cudaMemsetAsync(d, 0, 3 * sizeof(unsigned long long), st);
    if (e == cudaSuccess) {
        int *nan = reinterpret_cast<int *>(d + 2);
        maxabs_kernel<E><<<kScaleGrid, 256, 0, st>>>(A, lda, n, d, nan);
        maxabs_kernel<E><<<kScaleGrid, 256, 0, st>>>(B, ldb, n, d + 1, nan + 1);
        count_launches(2);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(h, d, sizeof(h), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    cudaFreeAsync(d, st);
    if (e != cudaSuccess) return e;
    const int *nan = reinterpret_cast<const int *>(h + 2);
    double an, bn;
    memcpy(&an, &h[0], sizeof(double));
    memcpy(&bn, &h[1], sizeof(double));
    g.anrm = (R)an;
    g.bnrm = (R)bn;
    g.ilascl = !nan[0] && gs::needs_scaling(g.anrm, &g.anrmto);
    g.ilbscl = !nan[1] && gs::needs_scaling(g.bnrm, &g.bnrmto);
    for (int w = 0; w < 2 && e == cudaSuccess; w++) {
        if (!(w == 0 ? g.ilascl : g.ilbscl)) continue;
        Muls<R> m;
        m.k = gs::lascl_steps(w == 0 ? g.anrm : g.bnrm, w == 0 ? g.anrmto : g.bnrmto, m.f);
        lascl_kernel<E, R><<<kScaleGrid, 256, 0, st>>>(w == 0 ? A : B, w == 0 ? lda : ldb, n, 0, m);
        count_launches(1);
        e = cudaGetLastError();
    }
    return e;
}

// the scaled-back eigenvalue copies SELCTG sees (xGGES undoes the scaling before selecting)
template <class R>
void gges_unscale_host(const GgesScale<R> &g, int n, R *a0, R *a1, R *b, int cw)
{
    R f[8];
    if (g.ilascl) {
        const int k = gs::lascl_steps(g.anrmto, g.anrm, f);
        gs::lascl_apply(k, f, a0, (size_t)n * cw);
        if (a1) gs::lascl_apply(k, f, a1, (size_t)n * cw);
    }
    if (g.ilbscl) {
        const int k = gs::lascl_steps(g.bnrmto, g.bnrm, f);
        gs::lascl_apply(k, f, b, (size_t)n * cw);
    }
}

// xGGES's last step: the Schur form and the eigenvalues scaled back (real: A upper Hessenberg,
// after DGGES's guard of complex pairs; complex: A upper triangular); B upper triangular
template <class E, class R>
cudaError_t gges_scale_out(cudaStream_t st, int n, E *A, int lda, E *B, int ldb, E *ev0, E *ev1, E *ev2,
                           const GgesScale<R> &g)
{
    if (!g.ilascl && !g.ilbscl) return cudaSuccess;
    constexpr bool cplx = sizeof(E) == 2 * sizeof(R);
    constexpr int cw = cplx ? 2 : 1;
    const int nev = cplx ? 2 : 3;
    std::vector<R> h((size_t)3 * n * cw);
    E *dv[3] = {ev0, ev1, ev2};
    cudaError_t e = cudaSuccess;
    for (int k = 0; k < nev && e == cudaSuccess; k++)
        e = cudaMemcpyAsync(h.data() + (size_t)k * n * cw, dv[k], n * sizeof(E), cudaMemcpyDeviceToHost, st);
    std::vector<R> aii(n), aii1(n), bii(n);
    if (!cplx && e == cudaSuccess) {  // A(i, i), A(i, i + 1), B(i, i) for DGGES's guard
        e = cudaMemcpy2DAsync(aii.data(), sizeof(R), A, (size_t)(lda + 1) * sizeof(R), sizeof(R), n,
                              cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess && n > 1)
            e = cudaMemcpy2DAsync(aii1.data(), sizeof(R), reinterpret_cast<const R *>(A) + lda,
                                  (size_t)(lda + 1) * sizeof(R), sizeof(R), n - 1, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess)
            e = cudaMemcpy2DAsync(bii.data(), sizeof(R), B, (size_t)(ldb + 1) * sizeof(R), sizeof(R), n,
                                  cudaMemcpyDeviceToHost, st);
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return e;
    R *a0 = h.data(), *a1 = cplx ? nullptr : h.data() + n, *b = h.data() + (size_t)(cplx ? 1 : 2) * n * cw;
    if (!cplx) gs::pair_guard(n, g.ilascl, g.anrm, g.anrmto, g.ilbscl, g.bnrm, g.bnrmto, aii.data(), aii1.data(),
                              bii.data(), a0, a1, b);
    gges_unscale_host(g, n, a0, a1, b, cw);
    for (int k = 0; k < nev && e == cudaSuccess; k++)
        e = cudaMemcpyAsync(dv[k], h.data() + (size_t)k * n * cw, n * sizeof(E), cudaMemcpyHostToDevice, st);
    for (int w = 0; w < 2 && e == cudaSuccess; w++) {
        if (!(w == 0 ? g.ilascl : g.ilbscl)) continue;
        Muls<R> m;
        m.k = gs::lascl_steps(w == 0 ? g.anrmto : g.bnrmto, w == 0 ? g.anrm : g.bnrm, m.f);
        lascl_kernel<E, R><<<kScaleGrid, 256, 0, st>>>(w == 0 ? A : B, w == 0 ? lda : ldb, n,
                                                       (w == 0 && !cplx) ? 2 : 1, m);
        count_launches(1);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    return e;
}

// SELCTG of real and complex xGGES (nonzero: selected); complex values as (re, im) pairs
template <class R>
using SelReal = int (*)(const R *, const R *, const R *);
template <class R>
using SelCplx = int (*)(const R *, const R *);

// LAPACK xGGES's argument checks, numbered by its argument list (JOBVSL, JOBVSR, SORT,
// SELCTG, N, A, LDA, B, LDB, SDIM, ALPHA, BETA, VSL, LDVSL, VSR, LDVSR, ... complex; real
// pencils have ALPHAR, ALPHAI in place of ALPHA, one argument more before VSL).  A null
// SELCTG with SORT = 'S' is argument 4.
int gges_check(char jobvsl, char jobvsr, char sort, bool have_sel, int n, int lda, int ldb, int ldvsl, int ldvsr,
               bool real = false)
{
    const bool wl = jobvsl == 'V', wr = jobvsr == 'V';
    if (!wl && jobvsl != 'N') return -1;
    if (!wr && jobvsr != 'N') return -2;
    if (sort != 'N' && sort != 'S') return -3;
    if (sort == 'S' && !have_sel) return -4;
    if (n < 0) return -5;
    if (lda < std::max(1, n)) return -7;
    if (ldb < std::max(1, n)) return -9;
    if (ldvsl < 1 || (wl && ldvsl < n)) return real ? -15 : -14;
    if (ldvsr < 1 || (wr && ldvsr < n)) return real ? -17 : -16;
    return 0;
}

// The selection flags to the device, the reordering kernel, the status back (stream st, then
// synchronised): the common part of the real and complex ordering steps.
template <class LAUNCH>
cudaError_t run_tgsen(cudaStream_t st, const std::vector<int> &bw, int *status, LAUNCH launch)
{
    const int n = (int)bw.size();
    int *d_sel = nullptr;  // n flags, then the status word
    cudaError_t e = cudaMallocAsync(&d_sel, (n + 1) * sizeof(int), st);
    if (e != cudaSuccess) return e;
    e = cudaMemcpyAsync(d_sel, bw.data(), n * sizeof(int), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) {
        launch(d_sel, d_sel + n);
        count_launches(1);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(status, d_sel + n, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    cudaFreeAsync(d_sel, st);
    return e;
}

// xGGES's ordering step for real pencils (QZ done, INFO 0): SELCTG over the QZ eigenvalues
// (scaled back first, as DGGES does), DTGSEN (IJOB = 0) on the device (INFO = n + 3 when a
// swap was rejected).  DGGES's check of the new eigenvalues (gges_check_real) follows the
// scaling back of the Schur form.
template <class R>
cudaError_t gges_sort_real(cudaStream_t st, SelReal<R> sel, const rb::Pencil<R> &p, R *alphar, R *alphai, R *beta,
                           const GgesScale<R> &g, int *info)
{
    const int n = p.n;
    std::vector<R> h(3 * (size_t)n);
    R *dv[3] = {alphar, alphai, beta};
    cudaError_t e = cudaSuccess;
    for (int k = 0; k < 3 && e == cudaSuccess; k++)
        e = cudaMemcpyAsync(h.data() + (size_t)k * n, dv[k], n * sizeof(R), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return e;
    gges_unscale_host(g, n, h.data(), h.data() + n, h.data() + 2 * (size_t)n, 1);
    std::vector<int> bw(n);
    for (int i = 0; i < n; i++) bw[i] = sel(&h[i], &h[n + i], &h[2 * (size_t)n + i]) != 0 ? 1 : 0;
    int status = 0;
    e = run_tgsen(st, bw, &status, [&](int *d_sel, int *d_status) {
        tgsen_real_kernel<R><<<1, kQzThreads, 0, st>>>(p, d_sel, alphar, alphai, beta, d_status);
    });
    if (e != cudaSuccess) return e;
    if (status != 0) *info = n + 3;
    if (status == 3) set_last_error("xGGES: the reordering walk did not end within its swap bound");
    return cudaSuccess;
}

// DGGES's check of the final eigenvalues: SDIM counts the selected ones (a pair counts 2 when
// either of its values is selected), INFO = n + 2 when a selected eigenvalue follows one that
// is not (rounding in the reordering changed a selection)
template <class R>
cudaError_t gges_check_real(cudaStream_t st, SelReal<R> sel, int n, const R *alphar, const R *alphai, const R *beta,
                            int *sdim, int *info)
{
    std::vector<R> h(3 * (size_t)n);
    const R *dv[3] = {alphar, alphai, beta};
    cudaError_t e = cudaSuccess;
    for (int k = 0; k < 3 && e == cudaSuccess; k++)
        e = cudaMemcpyAsync(h.data() + (size_t)k * n, dv[k], n * sizeof(R), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return e;
    *sdim = rb::gges_sdim_real(n, sel, h.data(), h.data() + n, h.data() + 2 * (size_t)n, info);
    return cudaSuccess;
}

// The same for complex pencils: ZTGSEN (IJOB = 0) on the device (INFO = n + 3 as for real
// pencils); ZGGES's check (gges_check_cplx) after the scaling back.
template <class R>
cudaError_t gges_sort_cplx(cudaStream_t st, SelCplx<R> sel, const rb::ZPencil<R> &p, rb::zc<R> *alpha,
                           rb::zc<R> *beta, const GgesScale<R> &g, int *info)
{
    using C = rb::zc<R>;
    const int n = p.n;
    std::vector<C> h(2 * (size_t)n);
    cudaError_t e = cudaMemcpyAsync(h.data(), alpha, n * sizeof(C), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(h.data() + n, beta, n * sizeof(C), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return e;
    gges_unscale_host(g, n, &h[0].re, (R *)nullptr, &h[n].re, 2);
    std::vector<int> bw(n);
    for (int i = 0; i < n; i++) bw[i] = sel(&h[i].re, &h[n + i].re) != 0 ? 1 : 0;
    int status = 0;
    e = run_tgsen(st, bw, &status, [&](int *d_sel, int *d_status) {
        tgsen_cplx_kernel<R><<<1, kQzThreads, 0, st>>>(p, d_sel, alpha, beta, d_status);
    });
    if (e != cudaSuccess) return e;
    if (status != 0) *info = n + 3;
    return cudaSuccess;
}

template <class R>
cudaError_t gges_check_cplx(cudaStream_t st, SelCplx<R> sel, int n, const rb::zc<R> *alpha, const rb::zc<R> *beta,
                            int *sdim, int *info)
{
    using C = rb::zc<R>;
    std::vector<C> h(2 * (size_t)n);
    cudaError_t e = cudaMemcpyAsync(h.data(), alpha, n * sizeof(C), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(h.data() + n, beta, n * sizeof(C), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return e;
    *sdim = rb::gges_sdim_cplx(n, sel, h.data(), h.data() + n, info);
    return cudaSuccess;
}

// Real pencils, device pointers (alphar, alphai, beta n each).  Returns 0, or 1 when a CUDA
// call failed.  sdim may be null when sort is 'N' (it is set to 0 otherwise).
template <class R>
int gges_device_real(cudaStream_t st, char jobvsl, char jobvsr, char sort, SelReal<R> sel, int n, R *A, int lda,
                     R *B, int ldb, int *sdim, R *alphar, R *alphai, R *beta, R *VSL, int ldvsl, R *VSR, int ldvsr,
                     int *info)
{
    set_last_error("");
    jobvsl = (char)std::toupper((unsigned char)jobvsl);
    jobvsr = (char)std::toupper((unsigned char)jobvsr);
    sort = (char)std::toupper((unsigned char)sort);
    *info = gges_check(jobvsl, jobvsr, sort, sel != nullptr, n, lda, ldb, ldvsl, ldvsr, true);
    if (*info) {
        set_last_error("xGGES: argument " + std::to_string(-*info) + " has an illegal value");
        return 0;
    }
    if (sdim) *sdim = 0;
    if (n == 0) return 0;
    const int wl = jobvsl == 'V', wr = jobvsr == 'V';
    int *d_info = nullptr, h_info = 0;
    GgesScale<R> g;
    GgesBalance<R> bal;
    cudaError_t e = gges_scale_in<R, R>(st, n, A, lda, B, ldb, g);
    if (e == cudaSuccess) e = gges_balance_in<R, R>(st, n, A, lda, B, ldb, bal);
    if (e == cudaSuccess) e = cudaMallocAsync(&d_info, sizeof(int), st);
    if (e == cudaSuccess) {
        // Q and Z are not referenced when not wanted
        rb::QzPencilR<R> p{n,   wl,  wr,  A,      B,      wl ? VSL : A, wr ? VSR : A, lda, ldb, wl ? ldvsl : lda,
                           wr ? ldvsr : lda, alphar, alphai, beta};
        dgges_kernel<R><<<1, kQzThreads, 0, st>>>(p, d_info);
        count_launches(1);
        e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaMemcpyAsync(&h_info, d_info, sizeof(int), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        cudaFreeAsync(d_info, st);
        *info = h_info;
        if (e == cudaSuccess && h_info == 0) {  // a QZ failure leaves the pencil scaled, as DGGES
            if (sort == 'S') {
                const rb::Pencil<R> q{n, wl, wr, A, B, p.Q, p.Z, lda, ldb, p.ldq, p.ldz};
                e = gges_sort_real<R>(st, sel, q, alphar, alphai, beta, g, info);
            }
            if (e == cudaSuccess)
                e = gges_balance_out<R, R>(st, n, wl ? VSL : nullptr, ldvsl, wr ? VSR : nullptr, ldvsr, bal);
            if (e == cudaSuccess) e = gges_scale_out<R, R>(st, n, A, lda, B, ldb, alphar, alphai, beta, g);
            if (e == cudaSuccess && sort == 'S') {
                int sd = 0;
                e = gges_check_real<R>(st, sel, n, alphar, alphai, beta, &sd, info);
                if (sdim) *sdim = sd;
            }
        }
    }
    gges_balance_free(st, bal);  // stream-ordered after the kernels that read it
    if (e != cudaSuccess) {
        set_last_error(std::string("xGGES: ") + cudaGetErrorString(e));
        *info = n + 1;
        return 1;
    }
    return 0;
}

// Real pencils, host pointers
template <class R>
void gges_host_real(char jobvsl, char jobvsr, char sort, SelReal<R> sel, int n, R *A, int lda, R *B, int ldb, int *sdim,
                    R *alphar, R *alphai, R *beta, R *VSL, int ldvsl, R *VSR, int ldvsr, int *info)
{
    set_last_error("");
    const char jl = (char)std::toupper((unsigned char)jobvsl), jr = (char)std::toupper((unsigned char)jobvsr);
    const char so = (char)std::toupper((unsigned char)sort);
    *info = gges_check(jl, jr, so, sel != nullptr, n, lda, ldb, ldvsl, ldvsr, true);
    if (*info) {
        set_last_error("xGGES: argument " + std::to_string(-*info) + " has an illegal value");
        return;
    }
    if (sdim) *sdim = 0;
    if (n == 0) return;
    const bool wl = jl == 'V', wr = jr == 'V';
    cudaStream_t st = nullptr;
    R *dA = nullptr, *dB = nullptr, *dL = nullptr, *dR = nullptr, *dv = nullptr;
    const size_t mat = (size_t)n * n * sizeof(R);
    cudaError_t e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
    for (R **q : {&dA, &dB})
        if (e == cudaSuccess) e = cudaMallocAsync(q, mat, st);
    if (wl && e == cudaSuccess) e = cudaMallocAsync(&dL, mat, st);
    if (wr && e == cudaSuccess) e = cudaMallocAsync(&dR, mat, st);
    if (e == cudaSuccess) e = cudaMallocAsync(&dv, 3 * (size_t)n * sizeof(R), st);
    if (e == cudaSuccess)
        e = cudaMemcpy2DAsync(dA, n * sizeof(R), A, (size_t)lda * sizeof(R), n * sizeof(R), n, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess)
        e = cudaMemcpy2DAsync(dB, n * sizeof(R), B, (size_t)ldb * sizeof(R), n * sizeof(R), n, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) {
        const int rc = gges_device_real<R>(st, jl, jr, so, sel, n, dA, n, dB, n, sdim, dv, dv + n, dv + 2 * n, dL,
                                           wl ? n : 1, dR, wr ? n : 1, info);
        if (rc == 0) {
            e = cudaMemcpy2DAsync(A, (size_t)lda * sizeof(R), dA, n * sizeof(R), n * sizeof(R), n, cudaMemcpyDeviceToHost, st);
            if (e == cudaSuccess)
                e = cudaMemcpy2DAsync(B, (size_t)ldb * sizeof(R), dB, n * sizeof(R), n * sizeof(R), n,
                                      cudaMemcpyDeviceToHost, st);
            if (wl && e == cudaSuccess)
                e = cudaMemcpy2DAsync(VSL, (size_t)ldvsl * sizeof(R), dL, n * sizeof(R), n * sizeof(R), n,
                                      cudaMemcpyDeviceToHost, st);
            if (wr && e == cudaSuccess)
                e = cudaMemcpy2DAsync(VSR, (size_t)ldvsr * sizeof(R), dR, n * sizeof(R), n * sizeof(R), n,
                                      cudaMemcpyDeviceToHost, st);
            R *outs[3] = {alphar, alphai, beta};
            for (int k = 0; k < 3 && e == cudaSuccess; k++)
                e = cudaMemcpyAsync(outs[k], dv + (size_t)k * n, n * sizeof(R), cudaMemcpyDeviceToHost, st);
            if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        } else {
            e = cudaErrorUnknown;
        }
    }
    for (R *q : {dA, dB, dL, dR, dv})
        if (q) cudaFreeAsync(q, st);
    if (st) {
        cudaStreamSynchronize(st);
        cudaStreamDestroy(st);
    }
    if (e != cudaSuccess && *info <= n) {
        set_last_error(std::string("xGGES staging: ") + cudaGetErrorString(e));
        *info = n + 1;
    }
}

// Device pointers (alpha, beta interleaved complex, n each).  Returns 0, or 1 when a CUDA call
// failed (message in last_error()).  sdim may be null when sort is 'N'.
template <class R>
int gges_device(cudaStream_t st, char jobvsl, char jobvsr, char sort, SelCplx<R> sel, int n, rb::zc<R> *A, int lda,
                rb::zc<R> *B, int ldb, int *sdim, rb::zc<R> *alpha, rb::zc<R> *beta, rb::zc<R> *VSL, int ldvsl,
                rb::zc<R> *VSR, int ldvsr, int *info)
{
    set_last_error("");
    jobvsl = (char)std::toupper((unsigned char)jobvsl);
    jobvsr = (char)std::toupper((unsigned char)jobvsr);
    sort = (char)std::toupper((unsigned char)sort);
    *info = gges_check(jobvsl, jobvsr, sort, sel != nullptr, n, lda, ldb, ldvsl, ldvsr);
    if (*info) {
        set_last_error("xGGES: argument " + std::to_string(-*info) + " has an illegal value");
        return 0;
    }
    if (sdim) *sdim = 0;
    if (n == 0) return 0;
    const int wl = jobvsl == 'V', wr = jobvsr == 'V';
    int *d_info = nullptr, h_info = 0;
    GgesScale<R> g;
    GgesBalance<R> bal;
    cudaError_t e = gges_scale_in<rb::zc<R>, R>(st, n, A, lda, B, ldb, g);
    if (e == cudaSuccess) e = gges_balance_in<rb::zc<R>, R>(st, n, A, lda, B, ldb, bal);
    if (e == cudaSuccess) e = cudaMallocAsync(&d_info, sizeof(int), st);
    if (e == cudaSuccess) {
        // Q and Z are not referenced when not wanted
        rb::QzPencil<R> p{n, wl, wr, A, B, wl ? VSL : A, wr ? VSR : A, lda, ldb, wl ? ldvsl : lda, wr ? ldvsr : lda};
        zgges_kernel<R><<<1, kQzThreads, 0, st>>>(p, alpha, beta, d_info);
        count_launches(1);
        e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaMemcpyAsync(&h_info, d_info, sizeof(int), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        cudaFreeAsync(d_info, st);
        *info = h_info;
        if (e == cudaSuccess && h_info == 0) {  // a QZ failure leaves the pencil scaled, as ZGGES
            if (sort == 'S') {
                const rb::ZPencil<R> q{n, wl, wr, A, B, p.Q, p.Z, lda, ldb, p.ldq, p.ldz};
                e = gges_sort_cplx<R>(st, sel, q, alpha, beta, g, info);
            }
            if (e == cudaSuccess)
                e = gges_balance_out<rb::zc<R>, R>(st, n, wl ? VSL : nullptr, ldvsl, wr ? VSR : nullptr, ldvsr, bal);
            if (e == cudaSuccess)
                e = gges_scale_out<rb::zc<R>, R>(st, n, A, lda, B, ldb, alpha, beta, (rb::zc<R> *)nullptr, g);
            if (e == cudaSuccess && sort == 'S') {
                int sd = 0;
                e = gges_check_cplx<R>(st, sel, n, alpha, beta, &sd, info);
                if (sdim) *sdim = sd;
            }
        }
    }
    gges_balance_free(st, bal);  // stream-ordered after the kernels that read it
    if (e != cudaSuccess) {
        set_last_error(std::string("xGGES: ") + cudaGetErrorString(e));
        *info = n + 1;
        return 1;
    }
    return 0;
}

// Host pointers: A, B (and VSL, VSR when wanted) go to the device and come back with alpha, beta.
template <class R>
void gges_host(char jobvsl, char jobvsr, char sort, SelCplx<R> sel, int n, rb::zc<R> *A, int lda, rb::zc<R> *B, int ldb,
               int *sdim, rb::zc<R> *alpha, rb::zc<R> *beta, rb::zc<R> *VSL, int ldvsl, rb::zc<R> *VSR, int ldvsr,
               int *info)
{
    using C = rb::zc<R>;
    set_last_error("");
    const char jl = (char)std::toupper((unsigned char)jobvsl), jr = (char)std::toupper((unsigned char)jobvsr);
    const char so = (char)std::toupper((unsigned char)sort);
    *info = gges_check(jl, jr, so, sel != nullptr, n, lda, ldb, ldvsl, ldvsr);
    if (*info) {
        set_last_error("xGGES: argument " + std::to_string(-*info) + " has an illegal value");
        return;
    }
    if (sdim) *sdim = 0;
    if (n == 0) return;
    const bool wl = jl == 'V', wr = jr == 'V';
    cudaStream_t st = nullptr;
    C *dA = nullptr, *dB = nullptr, *dL = nullptr, *dR = nullptr, *dab = nullptr;
    const size_t mat = (size_t)n * n * sizeof(C);
    cudaError_t e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
    for (C **q : {&dA, &dB})
        if (e == cudaSuccess) e = cudaMallocAsync(q, mat, st);
    if (wl && e == cudaSuccess) e = cudaMallocAsync(&dL, mat, st);
    if (wr && e == cudaSuccess) e = cudaMallocAsync(&dR, mat, st);
    if (e == cudaSuccess) e = cudaMallocAsync(&dab, 2 * (size_t)n * sizeof(C), st);
    if (e == cudaSuccess)
        e = cudaMemcpy2DAsync(dA, n * sizeof(C), A, (size_t)lda * sizeof(C), n * sizeof(C), n, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess)
        e = cudaMemcpy2DAsync(dB, n * sizeof(C), B, (size_t)ldb * sizeof(C), n * sizeof(C), n, cudaMemcpyHostToDevice, st);
    int rc = 0;
    if (e == cudaSuccess) {
        rc = gges_device<R>(st, jl, jr, so, sel, n, dA, n, dB, n, sdim, dab, dab + n, dL, wl ? n : 1, dR, wr ? n : 1,
                            info);
        if (rc == 0) {
            e = cudaMemcpy2DAsync(A, (size_t)lda * sizeof(C), dA, n * sizeof(C), n * sizeof(C), n, cudaMemcpyDeviceToHost, st);
            if (e == cudaSuccess)
                e = cudaMemcpy2DAsync(B, (size_t)ldb * sizeof(C), dB, n * sizeof(C), n * sizeof(C), n,
                                      cudaMemcpyDeviceToHost, st);
            if (wl && e == cudaSuccess)
                e = cudaMemcpy2DAsync(VSL, (size_t)ldvsl * sizeof(C), dL, n * sizeof(C), n * sizeof(C), n,
                                      cudaMemcpyDeviceToHost, st);
            if (wr && e == cudaSuccess)
                e = cudaMemcpy2DAsync(VSR, (size_t)ldvsr * sizeof(C), dR, n * sizeof(C), n * sizeof(C), n,
                                      cudaMemcpyDeviceToHost, st);
            if (e == cudaSuccess) e = cudaMemcpyAsync(alpha, dab, n * sizeof(C), cudaMemcpyDeviceToHost, st);
            if (e == cudaSuccess) e = cudaMemcpyAsync(beta, dab + n, n * sizeof(C), cudaMemcpyDeviceToHost, st);
            if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        }
    }
    for (C *q : {dA, dB, dL, dR, dab})
        if (q) cudaFreeAsync(q, st);
    if (st) {
        cudaStreamSynchronize(st);
        cudaStreamDestroy(st);
    }
    if (e != cudaSuccess) {
        set_last_error(std::string("xGGES staging: ") + cudaGetErrorString(e));
        *info = n + 1;
    }
}

// xTGSEN's argument checks (IJOB 0 to 5); sets last_error for a bad one
int tgsen_check(int ijob, int wantq, int wantz, int n, int lda, int ldb, int ldq, int ldz, bool cplx)
{
    int info = 0;
    const bool built = ijob >= 0 && ijob <= 5;
    (void)cplx;
    if (!built) info = -1;
    else if (n < 0) info = -5;
    else if (lda < std::max(1, n)) info = -7;
    else if (ldb < std::max(1, n)) info = -9;
    else if (ldq < 1 || (wantq && ldq < n)) info = cplx ? -13 : -14;
    else if (ldz < 1 || (wantz && ldz < n)) info = cplx ? -15 : -16;
    if (info == -1)
        set_last_error("xTGSEN: argument 1 has an illegal value");
    else if (info)
        set_last_error("xTGSEN: argument " + std::to_string(-info) + " has an illegal value");
    return info;
}

// LAPACK xTGSEN, device pointers, SELECT on the host: the reordering, the eigenvalues, M and
// (IJOB 1 to 5) PL, PR, DIF(1:2) (pl, pr, dif may be null).  INFO as LAPACK
// numbers its arguments (-1 IJOB, -5 N, -7 LDA, -9 LDB, -14 / -13 LDQ, -16 / -15 LDZ for real /
// complex pencils), 1 when a swap was rejected.  Returns 0, or 1 when a CUDA call failed.
template <class R, bool CPLX>
int tgsen_device(cudaStream_t st, int ijob, int wantq, int wantz, const int *select, int n, R *A, int lda, R *B,
                 int ldb, R *ev0, R *ev1, R *ev2, R *Q, int ldq, R *Z, int ldz, int *m, R *pl, R *pr, R *dif,
                 int *info)
{
    set_last_error("");
    *info = tgsen_check(ijob, wantq, wantz, n, lda, ldb, ldq, ldz, CPLX);
    if (*info) return 0;
    if (m) *m = 0;
    if (n == 0) return 0;
    std::vector<int> bw(n);
    for (int i = 0; i < n; i++) bw[i] = select[i] != 0 ? 1 : 0;
    int h[2] = {0, 0};
    R est[4] = {R(0), R(0), R(0), R(0)};
    size_t nwork = 0;  // IJOB >= 1: 2 M (n - M) elements for xTGSYL's right-hand sides
    cudaError_t e = cudaSuccess;
    if (CPLX && ijob != 0) {
        int mm = 0;
        for (int k = 0; k < n; k++) mm += bw[k];
        nwork = (ijob == 3 || ijob == 5 ? 4 : 2) * (size_t)mm * (n - mm) * 2;  // complex elements as reals
    }
    if (!CPLX && ijob != 0) {  // M from the subdiagonal (DTGSEN's count), to size the workspace
        std::vector<R> sub(n > 1 ? n - 1 : 1);
        if (n > 1)
            e = cudaMemcpy2DAsync(sub.data(), sizeof(R), A + 1, (size_t)(lda + 1) * sizeof(R), sizeof(R), n - 1,
                                  cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        int mm = 0;
        for (int k = 0; k < n; k++) {
            if (k + 1 < n && sub[k] != R(0)) {
                mm += (bw[k] || bw[k + 1]) ? 2 : 0;
                k++;
            } else {
                mm += bw[k];
            }
        }
        nwork = (ijob == 3 || ijob == 5 ? 4 : 2) * (size_t)mm * (n - mm);
    }
    const int ncuts = n / 2 + 4;
    const size_t niwork = (!CPLX && (ijob == 3 || ijob == 5)) ? nwork / 2 : 0;  // xLACN2's signs
    int *d = nullptr;  // n flags, the status (INFO, M), the cuts, the signs
    R *w = nullptr;    // PL, PR, DIF(1), DIF(2), then the workspace
    if (e == cudaSuccess) e = cudaMallocAsync(&d, (n + 2 + ncuts + niwork) * sizeof(int), st);
    if (e == cudaSuccess) e = cudaMallocAsync(&w, (4 + nwork) * sizeof(R), st);
    if (e == cudaSuccess) {
        e = cudaMemcpyAsync(d, bw.data(), n * sizeof(int), cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess) {
            if constexpr (CPLX) {
                using C = rb::zc<R>;
                C *a = reinterpret_cast<C *>(A), *b = reinterpret_cast<C *>(B);
                const rb::ZPencil<R> p{n, wantq, wantz, a, b, wantq ? reinterpret_cast<C *>(Q) : a,
                                       wantz ? reinterpret_cast<C *>(Z) : a, lda, ldb, wantq ? ldq : lda,
                                       wantz ? ldz : lda};
                tgsen_cplx_full_kernel<R><<<1, kQzThreads, 0, st>>>(p, d, ijob, reinterpret_cast<C *>(ev0),
                                                                     reinterpret_cast<C *>(ev1),
                                                                     reinterpret_cast<C *>(w + 4), d + n + 2, w, d + n);
            } else {
                const rb::Pencil<R> p{n, wantq, wantz, A, B, wantq ? Q : A, wantz ? Z : A, lda, ldb,
                                      wantq ? ldq : lda, wantz ? ldz : lda};
                tgsen_real_full_kernel<R><<<1, kQzThreads, 0, st>>>(p, d, ijob, ev0, ev1, ev2, w + 4,
                                                                     d + n + 2 + ncuts, d + n + 2, w, d + n);
            }
            count_launches(1);
            e = cudaGetLastError();
        }
        if (e == cudaSuccess) e = cudaMemcpyAsync(h, d + n, 2 * sizeof(int), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaMemcpyAsync(est, w, 4 * sizeof(R), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    }
    if (d) cudaFreeAsync(d, st);
    if (w) cudaFreeAsync(w, st);
    if (e != cudaSuccess) {
        set_last_error(std::string("xTGSEN: ") + cudaGetErrorString(e));
        return 1;
    }
    if (h[0] == 3) {
        set_last_error("xTGSEN: the reordering walk did not end within its swap bound");
        return 1;
    }
    *info = h[0];
    if (m) *m = h[1];
    if (ijob == 1 || ijob == 4 || ijob == 5) {
        if (pl) *pl = est[0];
        if (pr) *pr = est[1];
    }
    if (ijob >= 2 && dif) {
        dif[0] = est[2];
        dif[1] = est[3];
    }
    return 0;
}

// Host pointers: A, B (and Q, Z when wanted) go to the device and come back with the
// eigenvalues.  INFO = n + 1 (not a LAPACK value) when a CUDA call failed.
template <class R, bool CPLX>
void tgsen_host(int ijob, int wantq, int wantz, const int *select, int n, R *A, int lda, R *B, int ldb, R *ev0,
                R *ev1, R *ev2, R *Q, int ldq, R *Z, int ldz, int *m, R *pl, R *pr, R *dif, int *info)
{
    constexpr int w = CPLX ? 2 : 1;  // reals per element
    const int nev = CPLX ? 2 : 3;
    set_last_error("");
    *info = tgsen_check(ijob, wantq, wantz, n, lda, ldb, ldq, ldz, CPLX);  // before any data moves
    if (*info) return;
    if (m) *m = 0;
    if (n == 0) return;
    cudaStream_t st = nullptr;
    R *dA = nullptr, *dB = nullptr, *dQ = nullptr, *dZ = nullptr, *dv = nullptr;
    const size_t row = (size_t)n * w * sizeof(R), mat = row * n;
    cudaError_t e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
    for (R **q : {&dA, &dB})
        if (e == cudaSuccess) e = cudaMallocAsync(q, mat, st);
    if (wantq && e == cudaSuccess) e = cudaMallocAsync(&dQ, mat, st);
    if (wantz && e == cudaSuccess) e = cudaMallocAsync(&dZ, mat, st);
    if (e == cudaSuccess) e = cudaMallocAsync(&dv, nev * row, st);
    struct M2 {
        R *h, *d;
        int ld;
    } mats[4] = {{A, dA, lda}, {B, dB, ldb}, {Q, dQ, ldq}, {Z, dZ, ldz}};
    for (const M2 &x : mats)
        if (x.d && e == cudaSuccess)
            e = cudaMemcpy2DAsync(x.d, row, x.h, (size_t)x.ld * w * sizeof(R), row, n, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) {
        const int rc = tgsen_device<R, CPLX>(st, ijob, wantq, wantz, select, n, dA, n, dB, n, dv, dv + (size_t)n * w,
                                             dv + 2 * (size_t)n * w, dQ ? dQ : dA, n, dZ ? dZ : dA, n, m, pl, pr, dif,
                                             info);
        if (rc == 0) {
            for (const M2 &x : mats)
                if (x.d && e == cudaSuccess)
                    e = cudaMemcpy2DAsync(x.h, (size_t)x.ld * w * sizeof(R), x.d, row, row, n, cudaMemcpyDeviceToHost,
                                          st);
            R *outs[3] = {ev0, ev1, ev2};
            for (int k = 0; k < nev && e == cudaSuccess; k++)
                e = cudaMemcpyAsync(outs[k], dv + (size_t)k * n * w, row, cudaMemcpyDeviceToHost, st);
            if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        } else {
            e = cudaErrorUnknown;
        }
    }
    for (R *q : {dA, dB, dQ, dZ, dv})
        if (q) cudaFreeAsync(q, st);
    if (st) {
        cudaStreamSynchronize(st);
        cudaStreamDestroy(st);
    }
    if (e != cudaSuccess) {
        if (e != cudaErrorUnknown) set_last_error(std::string("xTGSEN staging: ") + cudaGetErrorString(e));
        *info = n + 1;
    }
}

// LAPACK xTGSYL's argument checks (TRANS = 'N' with IJOB 0, 1, 3, and TRANS = 'T' (real) /
// 'C' (complex) with IJOB not referenced, as LAPACK; the xGECON-based IJOB 2, 4 are refused with
// INFO = -2); sets last_error for a bad one
int tgsyl_check(char trans, int ijob, int m, int n, int lda, int ldb, int ldc, int ldd, int lde, int ldf,
                bool cplx = false)
{
    int info = 0;
    if (trans != 'N' && trans != (cplx ? 'C' : 'T')) info = -1;
    else if (trans == 'N' && ijob != 0 && ijob != 1 && ijob != 3) info = -2;
    else if (m <= 0) info = -3;
    else if (n <= 0) info = -4;
    else if (lda < std::max(1, m)) info = -6;
    else if (ldb < std::max(1, n)) info = -8;
    else if (ldc < std::max(1, m)) info = -10;
    else if (ldd < std::max(1, m)) info = -12;
    else if (lde < std::max(1, n)) info = -14;
    else if (ldf < std::max(1, m)) info = -16;
    if (info == -2 && (ijob == 2 || ijob == 4))
        set_last_error("xTGSYL: IJOB 2 and 4 (DGECON-based estimates) are not built");
    else if (info)
        set_last_error("xTGSYL: argument " + std::to_string(-info) + " has an illegal value");
    return info;
}

// xTGSYL, device pointers: C, F overwritten by R, L; *scale, *dif (IJOB 1, 3; left as given
// when the estimate's accumulator stayed 0).  Returns 0, or 1 when a CUDA call failed.
template <class R, bool CPLX = false>
int tgsyl_device(cudaStream_t st, char trans, int ijob, int m, int n, const R *A, int lda, const R *B, int ldb, R *C,
                 int ldc, const R *D, int ldd, const R *E, int lde, R *F, int ldf, R *scale, R *dif, int *info)
{
    set_last_error("");
    trans = (char)std::toupper((unsigned char)trans);
    *info = tgsyl_check(trans, ijob, m, n, lda, ldb, ldc, ldd, lde, ldf, CPLX);
    if (*info) return 0;
    if (trans != 'N') ijob = 0;  // not referenced by the transposed solve
    const int ncuts = m / 2 + n / 2 + 4;
    const size_t nwork = ijob == 1 ? 2 * (size_t)m * n * (CPLX ? 2 : 1) : 0;
    int *d = nullptr;  // the status, then the cuts
    R *w = nullptr;    // SCALE, DIF, then the saved solution (IJOB 1)
    R out[2] = {R(1), dif ? *dif : R(0)};
    int h = 0;
    cudaError_t e = cudaMallocAsync(&d, (1 + ncuts) * sizeof(int), st);
    if (e == cudaSuccess) e = cudaMallocAsync(&w, (2 + nwork) * sizeof(R), st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(w, out, 2 * sizeof(R), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess && CPLX) {
        using Cx = rb::zc<R>;
        rb::ZSylvG<R> y{};
        y.m = m;
        y.n = n;
        y.A = reinterpret_cast<const Cx *>(A);
        y.D = reinterpret_cast<const Cx *>(D);
        y.B = reinterpret_cast<const Cx *>(B);
        y.E = reinterpret_cast<const Cx *>(E);
        y.lda = lda;
        y.ldd = ldd;
        y.ldb = ldb;
        y.lde = lde;
        y.C = reinterpret_cast<Cx *>(C);
        y.F = reinterpret_cast<Cx *>(F);
        y.ldc = ldc;
        y.ldf = ldf;
        ztgsyl_kernel<R><<<1, kQzThreads, 0, st>>>(y, trans == 'C' ? 1 : 0, ijob, d + 1, reinterpret_cast<Cx *>(w + 2),
                                                    w, d);
        count_launches(1);
        e = cudaGetLastError();
    } else if (e == cudaSuccess) {
        rb::SylvG<R> y{};
        y.m = m;
        y.n = n;
        y.A = A;
        y.D = D;
        y.B = B;
        y.E = E;
        y.lda = lda;
        y.ldd = ldd;
        y.ldb = ldb;
        y.lde = lde;
        y.C = C;
        y.F = F;
        y.ldc = ldc;
        y.ldf = ldf;
        tgsyl_kernel<R><<<1, kQzThreads, 0, st>>>(y, trans == 'T' ? 1 : 0, ijob, d + 1, w + 2, w, d);
        count_launches(1);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(&h, d, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(out, w, 2 * sizeof(R), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (d) cudaFreeAsync(d, st);
    if (w) cudaFreeAsync(w, st);
    if (e != cudaSuccess) {
        set_last_error(std::string("xTGSYL: ") + cudaGetErrorString(e));
        return 1;
    }
    *info = h;
    if (scale) *scale = out[0];
    if (dif && ijob != 0) *dif = out[1];
    return 0;
}

// Host pointers.  INFO = m + n + 1 (not a LAPACK value) when a CUDA call failed.
template <class R, bool CPLX = false>
void tgsyl_host(char trans, int ijob, int m, int n, const R *A, int lda, const R *B, int ldb, R *C, int ldc,
                const R *D, int ldd, const R *E, int lde, R *F, int ldf, R *scale, R *dif, int *info)
{
    set_last_error("");
    *info = tgsyl_check((char)std::toupper((unsigned char)trans), ijob, m, n, lda, ldb, ldc, ldd, lde, ldf, CPLX);
    if (*info) return;
    constexpr int w = CPLX ? 2 : 1;  // reals per element
    cudaStream_t st = nullptr;
    R *buf = nullptr;
    const size_t mm = (size_t)m * m * w, nn = (size_t)n * n * w, mn = (size_t)m * n * w;
    cudaError_t e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaMallocAsync(&buf, (2 * mm + 2 * nn + 2 * mn) * sizeof(R), st);
    R *dA = buf, *dD = buf + mm, *dB = buf + 2 * mm, *dE = dB + nn, *dC = dE + nn, *dF = dC + mn;
    struct M2 {
        const R *h;
        R *d;
        int ld, rows, cols;
    } ins[6] = {{A, dA, lda, m, m}, {D, dD, ldd, m, m}, {B, dB, ldb, n, n},
                {E, dE, lde, n, n}, {C, dC, ldc, m, n}, {F, dF, ldf, m, n}};
    for (const M2 &x : ins)
        if (e == cudaSuccess)
            e = cudaMemcpy2DAsync(x.d, x.rows * w * sizeof(R), x.h, (size_t)x.ld * w * sizeof(R), x.rows * w * sizeof(R),
                                  x.cols, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) {
        const int rc =
            tgsyl_device<R, CPLX>(st, trans, ijob, m, n, dA, m, dB, n, dC, m, dD, m, dE, n, dF, m, scale, dif, info);
        if (rc == 0) {
            const size_t col = (size_t)m * w * sizeof(R);
            e = cudaMemcpy2DAsync(C, (size_t)ldc * w * sizeof(R), dC, col, col, n, cudaMemcpyDeviceToHost, st);
            if (e == cudaSuccess)
                e = cudaMemcpy2DAsync(F, (size_t)ldf * w * sizeof(R), dF, col, col, n, cudaMemcpyDeviceToHost, st);
            if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        } else {
            e = cudaErrorUnknown;
        }
    }
    if (buf) cudaFreeAsync(buf, st);
    if (st) {
        cudaStreamSynchronize(st);
        cudaStreamDestroy(st);
    }
    if (e != cudaSuccess) {
        if (e != cudaErrorUnknown) set_last_error(std::string("xTGSYL staging: ") + cudaGetErrorString(e));
        *info = m + n + 1;
    }
}

// ---- xGGBAL / xGGBAK as entry points of their own (JOB 'N' or 'P') ---------------------------

// LAPACK xGGBAL's checks: JOB (-1; 'S' and 'B', the scaling, are not built), N (-2), LDA (-4),
// LDB (-6)
int ggbal_check(char job, int n, int lda, int ldb)
{
    int info = 0;
    if (job != 'N' && job != 'P') info = -1;
    else if (n < 0) info = -2;
    else if (lda < std::max(1, n)) info = -4;
    else if (ldb < std::max(1, n)) info = -6;
    if (info == -1 && (job == 'S' || job == 'B'))
        set_last_error("xGGBAL: JOB = 'S' / 'B' (the scaling) is not built");
    else if (info)
        set_last_error("xGGBAL: argument " + std::to_string(-info) + " has an illegal value");
    return info;
}

// device pointers (lscale, rscale n each on the device); returns 0, or 1 when a CUDA call failed
template <class E, class R>
int ggbal_device(cudaStream_t st, char job, int n, E *A, int lda, E *B, int ldb, int *ilo, int *ihi, R *lscale,
                 R *rscale, int *info)
{
    set_last_error("");
    job = (char)std::toupper((unsigned char)job);
    *info = ggbal_check(job, n, lda, ldb);
    if (*info) return 0;
    *ilo = 1;
    *ihi = n;
    if (n == 0) return 0;
    cudaError_t e = cudaSuccess;
    if (job == 'N') {
        const std::vector<R> ones(n, R(1));
        e = cudaMemcpyAsync(lscale, ones.data(), n * sizeof(R), cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess) e = cudaMemcpyAsync(rscale, ones.data(), n * sizeof(R), cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    } else {
        int *d = nullptr, h[2] = {1, n};
        e = cudaMallocAsync(&d, (2 + 2 * kQzThreads) * sizeof(int), st);
        if (e == cudaSuccess) {
            const rb::BalPencil<E> p{n, A, B, lda, ldb};
            ggbal_kernel<E, R><<<1, kQzThreads, 0, st>>>(p, lscale, rscale, d, d + 2);
            count_launches(1);
            e = cudaGetLastError();
            if (e == cudaSuccess) e = cudaMemcpyAsync(h, d, 2 * sizeof(int), cudaMemcpyDeviceToHost, st);
            if (e == cudaSuccess) e = cudaStreamSynchronize(st);
            cudaFreeAsync(d, st);
        }
        *ilo = h[0];
        *ihi = h[1];
    }
    if (e != cudaSuccess) {
        set_last_error(std::string("xGGBAL: ") + cudaGetErrorString(e));
        return 1;
    }
    return 0;
}

// host pointers; INFO = n + 1 (not a LAPACK value) when a CUDA call failed
template <class E, class R>
void ggbal_host(char job, int n, E *A, int lda, E *B, int ldb, int *ilo, int *ihi, R *lscale, R *rscale, int *info)
{
    set_last_error("");
    *info = ggbal_check((char)std::toupper((unsigned char)job), n, lda, ldb);
    if (*info) return;
    *ilo = 1;
    *ihi = n;
    if (n == 0) return;
    cudaStream_t st = nullptr;
    E *dA = nullptr, *dB = nullptr;
    R *ds = nullptr;
    const size_t col = (size_t)n * sizeof(E);
    cudaError_t e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaMallocAsync(&dA, col * n, st);
    if (e == cudaSuccess) e = cudaMallocAsync(&dB, col * n, st);
    if (e == cudaSuccess) e = cudaMallocAsync(&ds, 2 * (size_t)n * sizeof(R), st);
    if (e == cudaSuccess) e = cudaMemcpy2DAsync(dA, col, A, (size_t)lda * sizeof(E), col, n, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpy2DAsync(dB, col, B, (size_t)ldb * sizeof(E), col, n, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) {
        if (ggbal_device<E, R>(st, job, n, dA, n, dB, n, ilo, ihi, ds, ds + n, info) != 0) {
            e = cudaErrorUnknown;
        } else {
            e = cudaMemcpy2DAsync(A, (size_t)lda * sizeof(E), dA, col, col, n, cudaMemcpyDeviceToHost, st);
            if (e == cudaSuccess)
                e = cudaMemcpy2DAsync(B, (size_t)ldb * sizeof(E), dB, col, col, n, cudaMemcpyDeviceToHost, st);
            if (e == cudaSuccess) e = cudaMemcpyAsync(lscale, ds, n * sizeof(R), cudaMemcpyDeviceToHost, st);
            if (e == cudaSuccess) e = cudaMemcpyAsync(rscale, ds + n, n * sizeof(R), cudaMemcpyDeviceToHost, st);
            if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        }
    }
    for (void *q : {(void *)dA, (void *)dB, (void *)ds})
        if (q) cudaFreeAsync(q, st);
    if (st) {
        cudaStreamSynchronize(st);
        cudaStreamDestroy(st);
    }
    if (e != cudaSuccess) {
        if (e != cudaErrorUnknown) set_last_error(std::string("xGGBAL staging: ") + cudaGetErrorString(e));
        *info = n + 1;
    }
}

// LAPACK xGGBAK's checks: JOB (-1; 'S', 'B' not built), SIDE (-2), N (-3), ILO (-4), IHI (-5),
// M (-8), LDV (-10)
int ggbak_check(char job, char side, int n, int ilo, int ihi, int m, int ldv)
{
    int info = 0;
    if (job != 'N' && job != 'P') info = -1;
    else if (side != 'L' && side != 'R') info = -2;
    else if (n < 0) info = -3;
    else if (ilo < 1 || ilo > std::max(1, n)) info = -4;
    else if ((n == 0 && ihi != 0 && ilo != 1) || (n > 0 && (ihi < ilo || ihi > std::max(1, n)))) info = -5;
    else if (m < 0) info = -8;
    else if (ldv < std::max(1, n)) info = -10;
    if (info == -1 && (job == 'S' || job == 'B'))
        set_last_error("xGGBAK: JOB = 'S' / 'B' (the scaling) is not built");
    else if (info)
        set_last_error("xGGBAK: argument " + std::to_string(-info) + " has an illegal value");
    return info;
}

// device pointers (lscale, rscale and V on the device)
template <class E, class R>
int ggbak_device(cudaStream_t st, char job, char side, int n, int ilo, int ihi, const R *lscale, const R *rscale, int m,
                 E *V, int ldv, int *info)
{
    set_last_error("");
    job = (char)std::toupper((unsigned char)job);
    side = (char)std::toupper((unsigned char)side);
    *info = ggbak_check(job, side, n, ilo, ihi, m, ldv);
    if (*info || n == 0 || m == 0 || job == 'N') return 0;
    ggbak_m_kernel<E, R><<<1, kQzThreads, 0, st>>>(n, ilo, ihi, side == 'L' ? lscale : rscale, V, ldv, m);
    count_launches(1);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
        set_last_error(std::string("xGGBAK: ") + cudaGetErrorString(e));
        return 1;
    }
    return 0;
}

template <class E, class R>
void ggbak_host(char job, char side, int n, int ilo, int ihi, const R *lscale, const R *rscale, int m, E *V, int ldv,
                int *info)
{
    set_last_error("");
    const char jb = (char)std::toupper((unsigned char)job), sd = (char)std::toupper((unsigned char)side);
    *info = ggbak_check(jb, sd, n, ilo, ihi, m, ldv);
    if (*info || n == 0 || m == 0 || jb == 'N') return;
    cudaStream_t st = nullptr;
    E *dV = nullptr;
    R *ds = nullptr;
    const size_t col = (size_t)n * sizeof(E);
    cudaError_t e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaMallocAsync(&dV, col * m, st);
    if (e == cudaSuccess) e = cudaMallocAsync(&ds, n * sizeof(R), st);
    if (e == cudaSuccess) e = cudaMemcpy2DAsync(dV, col, V, (size_t)ldv * sizeof(E), col, m, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(ds, sd == 'L' ? lscale : rscale, n * sizeof(R), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) {
        if (ggbak_device<E, R>(st, jb, sd, n, ilo, ihi, ds, ds, m, dV, n, info) != 0) {
            e = cudaErrorUnknown;
        } else {
            e = cudaMemcpy2DAsync(V, (size_t)ldv * sizeof(E), dV, col, col, m, cudaMemcpyDeviceToHost, st);
            if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        }
    }
    if (dV) cudaFreeAsync(dV, st);
    if (ds) cudaFreeAsync(ds, st);
    if (st) {
        cudaStreamSynchronize(st);
        cudaStreamDestroy(st);
    }
    if (e != cudaSuccess) {
        if (e != cudaErrorUnknown) set_last_error(std::string("xGGBAK staging: ") + cudaGetErrorString(e));
        *info = n + 1;
    }
}

}  // namespace
}  // namespace xtg

using xtg::rb::zc;

extern "C" {

void xtgevc3_zgges(char jobvsl, char jobvsr, int n, double *A, int lda, double *B, int ldb, double *alpha,
                   double *beta, double *VSL, int ldvsl, double *VSR, int ldvsr, int *info)
{
    xtgevc3_zgges_sort(jobvsl, jobvsr, 'N', nullptr, n, A, lda, B, ldb, nullptr, alpha, beta, VSL, ldvsl, VSR, ldvsr,
                       info);
}

void xtgevc3_cgges(char jobvsl, char jobvsr, int n, float *A, int lda, float *B, int ldb, float *alpha, float *beta,
                   float *VSL, int ldvsl, float *VSR, int ldvsr, int *info)
{
    xtgevc3_cgges_sort(jobvsl, jobvsr, 'N', nullptr, n, A, lda, B, ldb, nullptr, alpha, beta, VSL, ldvsl, VSR, ldvsr,
                       info);
}

int xtgevc3_zgges_dev(void *stream, char jobvsl, char jobvsr, int n, double *A, int lda, double *B, int ldb,
                      double *alpha, double *beta, double *VSL, int ldvsl, double *VSR, int ldvsr, int *info)
{
    return xtgevc3_zgges_sort_dev(stream, jobvsl, jobvsr, 'N', nullptr, n, A, lda, B, ldb, nullptr, alpha, beta, VSL,
                                  ldvsl, VSR, ldvsr, info);
}

int xtgevc3_cgges_dev(void *stream, char jobvsl, char jobvsr, int n, float *A, int lda, float *B, int ldb, float *alpha,
                      float *beta, float *VSL, int ldvsl, float *VSR, int ldvsr, int *info)
{
    return xtgevc3_cgges_sort_dev(stream, jobvsl, jobvsr, 'N', nullptr, n, A, lda, B, ldb, nullptr, alpha, beta, VSL,
                                  ldvsl, VSR, ldvsr, info);
}

void xtgevc3_dgges(char jobvsl, char jobvsr, int n, double *A, int lda, double *B, int ldb, double *alphar,
                   double *alphai, double *beta, double *VSL, int ldvsl, double *VSR, int ldvsr, int *info)
{
    xtg::gges_host_real<double>(jobvsl, jobvsr, 'N', nullptr, n, A, lda, B, ldb, nullptr, alphar, alphai, beta, VSL,
                                ldvsl, VSR, ldvsr, info);
}

void xtgevc3_sgges(char jobvsl, char jobvsr, int n, float *A, int lda, float *B, int ldb, float *alphar, float *alphai,
                   float *beta, float *VSL, int ldvsl, float *VSR, int ldvsr, int *info)
{
    xtg::gges_host_real<float>(jobvsl, jobvsr, 'N', nullptr, n, A, lda, B, ldb, nullptr, alphar, alphai, beta, VSL,
                               ldvsl, VSR, ldvsr, info);
}

int xtgevc3_dgges_dev(void *stream, char jobvsl, char jobvsr, int n, double *A, int lda, double *B, int ldb,
                      double *alphar, double *alphai, double *beta, double *VSL, int ldvsl, double *VSR, int ldvsr,
                      int *info)
{
    return xtg::gges_device_real<double>(static_cast<cudaStream_t>(stream), jobvsl, jobvsr, 'N', nullptr, n, A, lda, B,
                                         ldb, nullptr, alphar, alphai, beta, VSL, ldvsl, VSR, ldvsr, info);
}

int xtgevc3_sgges_dev(void *stream, char jobvsl, char jobvsr, int n, float *A, int lda, float *B, int ldb,
                      float *alphar, float *alphai, float *beta, float *VSL, int ldvsl, float *VSR, int ldvsr, int *info)
{
    return xtg::gges_device_real<float>(static_cast<cudaStream_t>(stream), jobvsl, jobvsr, 'N', nullptr, n, A, lda, B,
                                        ldb, nullptr, alphar, alphai, beta, VSL, ldvsl, VSR, ldvsr, info);
}

// ---- with ordering (SORT, SELCTG, SDIM in LAPACK xGGES's positions) -------------------------

void xtgevc3_zgges_sort(char jobvsl, char jobvsr, char sort, xtgevc3_zselect2 selctg, int n, double *A, int lda,
                        double *B, int ldb, int *sdim, double *alpha, double *beta, double *VSL, int ldvsl, double *VSR,
                        int ldvsr, int *info)
{
    xtg::gges_host<double>(jobvsl, jobvsr, sort, selctg, n, reinterpret_cast<zc<double> *>(A), lda,
                           reinterpret_cast<zc<double> *>(B), ldb, sdim, reinterpret_cast<zc<double> *>(alpha),
                           reinterpret_cast<zc<double> *>(beta), reinterpret_cast<zc<double> *>(VSL), ldvsl,
                           reinterpret_cast<zc<double> *>(VSR), ldvsr, info);
}

void xtgevc3_cgges_sort(char jobvsl, char jobvsr, char sort, xtgevc3_cselect2 selctg, int n, float *A, int lda,
                        float *B, int ldb, int *sdim, float *alpha, float *beta, float *VSL, int ldvsl, float *VSR,
                        int ldvsr, int *info)
{
    xtg::gges_host<float>(jobvsl, jobvsr, sort, selctg, n, reinterpret_cast<zc<float> *>(A), lda,
                          reinterpret_cast<zc<float> *>(B), ldb, sdim, reinterpret_cast<zc<float> *>(alpha),
                          reinterpret_cast<zc<float> *>(beta), reinterpret_cast<zc<float> *>(VSL), ldvsl,
                          reinterpret_cast<zc<float> *>(VSR), ldvsr, info);
}

int xtgevc3_zgges_sort_dev(void *stream, char jobvsl, char jobvsr, char sort, xtgevc3_zselect2 selctg, int n, double *A,
                           int lda, double *B, int ldb, int *sdim, double *alpha, double *beta, double *VSL, int ldvsl,
                           double *VSR, int ldvsr, int *info)
{
    return xtg::gges_device<double>(static_cast<cudaStream_t>(stream), jobvsl, jobvsr, sort, selctg, n,
                                    reinterpret_cast<zc<double> *>(A), lda, reinterpret_cast<zc<double> *>(B), ldb,
                                    sdim, reinterpret_cast<zc<double> *>(alpha), reinterpret_cast<zc<double> *>(beta),
                                    reinterpret_cast<zc<double> *>(VSL), ldvsl, reinterpret_cast<zc<double> *>(VSR),
                                    ldvsr, info);
}

int xtgevc3_cgges_sort_dev(void *stream, char jobvsl, char jobvsr, char sort, xtgevc3_cselect2 selctg, int n, float *A,
                           int lda, float *B, int ldb, int *sdim, float *alpha, float *beta, float *VSL, int ldvsl,
                           float *VSR, int ldvsr, int *info)
{
    return xtg::gges_device<float>(static_cast<cudaStream_t>(stream), jobvsl, jobvsr, sort, selctg, n,
                                   reinterpret_cast<zc<float> *>(A), lda, reinterpret_cast<zc<float> *>(B), ldb, sdim,
                                   reinterpret_cast<zc<float> *>(alpha), reinterpret_cast<zc<float> *>(beta),
                                   reinterpret_cast<zc<float> *>(VSL), ldvsl, reinterpret_cast<zc<float> *>(VSR), ldvsr,
                                   info);
}

void xtgevc3_dgges_sort(char jobvsl, char jobvsr, char sort, xtgevc3_dselect3 selctg, int n, double *A, int lda,
                        double *B, int ldb, int *sdim, double *alphar, double *alphai, double *beta, double *VSL,
                        int ldvsl, double *VSR, int ldvsr, int *info)
{
    xtg::gges_host_real<double>(jobvsl, jobvsr, sort, selctg, n, A, lda, B, ldb, sdim, alphar, alphai, beta, VSL, ldvsl,
                                VSR, ldvsr, info);
}

void xtgevc3_sgges_sort(char jobvsl, char jobvsr, char sort, xtgevc3_sselect3 selctg, int n, float *A, int lda,
                        float *B, int ldb, int *sdim, float *alphar, float *alphai, float *beta, float *VSL, int ldvsl,
                        float *VSR, int ldvsr, int *info)
{
    xtg::gges_host_real<float>(jobvsl, jobvsr, sort, selctg, n, A, lda, B, ldb, sdim, alphar, alphai, beta, VSL, ldvsl,
                               VSR, ldvsr, info);
}

int xtgevc3_dgges_sort_dev(void *stream, char jobvsl, char jobvsr, char sort, xtgevc3_dselect3 selctg, int n,
                           double *A, int lda, double *B, int ldb, int *sdim, double *alphar, double *alphai,
                           double *beta, double *VSL, int ldvsl, double *VSR, int ldvsr, int *info)
{
    return xtg::gges_device_real<double>(static_cast<cudaStream_t>(stream), jobvsl, jobvsr, sort, selctg, n, A, lda, B,
                                         ldb, sdim, alphar, alphai, beta, VSL, ldvsl, VSR, ldvsr, info);
}

int xtgevc3_sgges_sort_dev(void *stream, char jobvsl, char jobvsr, char sort, xtgevc3_sselect3 selctg, int n, float *A,
                           int lda, float *B, int ldb, int *sdim, float *alphar, float *alphai, float *beta, float *VSL,
                           int ldvsl, float *VSR, int ldvsr, int *info)
{
    return xtg::gges_device_real<float>(static_cast<cudaStream_t>(stream), jobvsl, jobvsr, sort, selctg, n, A, lda, B,
                                        ldb, sdim, alphar, alphai, beta, VSL, ldvsl, VSR, ldvsr, info);
}

}  // extern "C"

// ---- xTGSEN (IJOB 0; real pencils also 1, 2, 4) and xTGSYL (TRANS = 'N', IJOB 0, 1, 3) ------

extern "C" {

void xtgevc3_dtgsen(int ijob, int wantq, int wantz, const int *select, int n, double *A, int lda, double *B, int ldb,
                    double *alphar, double *alphai, double *beta, double *Q, int ldq, double *Z, int ldz, int *m,
                    double *pl, double *pr, double *dif, int *info)
{
    xtg::tgsen_host<double, false>(ijob, wantq, wantz, select, n, A, lda, B, ldb, alphar, alphai, beta, Q, ldq, Z, ldz,
                                   m, pl, pr, dif, info);
}

void xtgevc3_stgsen(int ijob, int wantq, int wantz, const int *select, int n, float *A, int lda, float *B, int ldb,
                    float *alphar, float *alphai, float *beta, float *Q, int ldq, float *Z, int ldz, int *m, float *pl,
                    float *pr, float *dif, int *info)
{
    xtg::tgsen_host<float, false>(ijob, wantq, wantz, select, n, A, lda, B, ldb, alphar, alphai, beta, Q, ldq, Z, ldz,
                                  m, pl, pr, dif, info);
}

void xtgevc3_ztgsen(int ijob, int wantq, int wantz, const int *select, int n, double *A, int lda, double *B, int ldb,
                    double *alpha, double *beta, double *Q, int ldq, double *Z, int ldz, int *m, double *pl,
                    double *pr, double *dif, int *info)
{
    xtg::tgsen_host<double, true>(ijob, wantq, wantz, select, n, A, lda, B, ldb, alpha, beta, nullptr, Q, ldq, Z, ldz,
                                  m, pl, pr, dif, info);
}

void xtgevc3_ctgsen(int ijob, int wantq, int wantz, const int *select, int n, float *A, int lda, float *B, int ldb,
                    float *alpha, float *beta, float *Q, int ldq, float *Z, int ldz, int *m, float *pl, float *pr,
                    float *dif, int *info)
{
    xtg::tgsen_host<float, true>(ijob, wantq, wantz, select, n, A, lda, B, ldb, alpha, beta, nullptr, Q, ldq, Z, ldz, m,
                                 pl, pr, dif, info);
}

int xtgevc3_dtgsen_dev(void *stream, int ijob, int wantq, int wantz, const int *select, int n, double *A, int lda,
                       double *B, int ldb, double *alphar, double *alphai, double *beta, double *Q, int ldq, double *Z,
                       int ldz, int *m, double *pl, double *pr, double *dif, int *info)
{
    return xtg::tgsen_device<double, false>(static_cast<cudaStream_t>(stream), ijob, wantq, wantz, select, n, A, lda, B,
                                            ldb, alphar, alphai, beta, Q, ldq, Z, ldz, m, pl, pr, dif, info);
}

int xtgevc3_stgsen_dev(void *stream, int ijob, int wantq, int wantz, const int *select, int n, float *A, int lda,
                       float *B, int ldb, float *alphar, float *alphai, float *beta, float *Q, int ldq, float *Z,
                       int ldz, int *m, float *pl, float *pr, float *dif, int *info)
{
    return xtg::tgsen_device<float, false>(static_cast<cudaStream_t>(stream), ijob, wantq, wantz, select, n, A, lda, B,
                                           ldb, alphar, alphai, beta, Q, ldq, Z, ldz, m, pl, pr, dif, info);
}

int xtgevc3_ztgsen_dev(void *stream, int ijob, int wantq, int wantz, const int *select, int n, double *A, int lda,
                       double *B, int ldb, double *alpha, double *beta, double *Q, int ldq, double *Z, int ldz, int *m,
                       double *pl, double *pr, double *dif, int *info)
{
    return xtg::tgsen_device<double, true>(static_cast<cudaStream_t>(stream), ijob, wantq, wantz, select, n, A, lda, B,
                                           ldb, alpha, beta, nullptr, Q, ldq, Z, ldz, m, pl, pr, dif, info);
}

int xtgevc3_ctgsen_dev(void *stream, int ijob, int wantq, int wantz, const int *select, int n, float *A, int lda,
                       float *B, int ldb, float *alpha, float *beta, float *Q, int ldq, float *Z, int ldz, int *m,
                       float *pl, float *pr, float *dif, int *info)
{
    return xtg::tgsen_device<float, true>(static_cast<cudaStream_t>(stream), ijob, wantq, wantz, select, n, A, lda, B,
                                          ldb, alpha, beta, nullptr, Q, ldq, Z, ldz, m, pl, pr, dif, info);
}

void xtgevc3_dtgsyl(char trans, int ijob, int m, int n, const double *A, int lda, const double *B, int ldb, double *C,
                    int ldc, const double *D, int ldd, const double *E, int lde, double *F, int ldf, double *scale,
                    double *dif, int *info)
{
    xtg::tgsyl_host<double>(trans, ijob, m, n, A, lda, B, ldb, C, ldc, D, ldd, E, lde, F, ldf, scale, dif, info);
}

void xtgevc3_stgsyl(char trans, int ijob, int m, int n, const float *A, int lda, const float *B, int ldb, float *C,
                    int ldc, const float *D, int ldd, const float *E, int lde, float *F, int ldf, float *scale,
                    float *dif, int *info)
{
    xtg::tgsyl_host<float>(trans, ijob, m, n, A, lda, B, ldb, C, ldc, D, ldd, E, lde, F, ldf, scale, dif, info);
}

int xtgevc3_dtgsyl_dev(void *stream, char trans, int ijob, int m, int n, const double *A, int lda, const double *B,
                       int ldb, double *C, int ldc, const double *D, int ldd, const double *E, int lde, double *F,
                       int ldf, double *scale, double *dif, int *info)
{
    return xtg::tgsyl_device<double>(static_cast<cudaStream_t>(stream), trans, ijob, m, n, A, lda, B, ldb, C, ldc, D,
                                     ldd, E, lde, F, ldf, scale, dif, info);
}

int xtgevc3_stgsyl_dev(void *stream, char trans, int ijob, int m, int n, const float *A, int lda, const float *B,
                       int ldb, float *C, int ldc, const float *D, int ldd, const float *E, int lde, float *F, int ldf,
                       float *scale, float *dif, int *info)
{
    return xtg::tgsyl_device<float>(static_cast<cudaStream_t>(stream), trans, ijob, m, n, A, lda, B, ldb, C, ldc, D,
                                    ldd, E, lde, F, ldf, scale, dif, info);
}

}  // extern "C"

// ---- Z/CTGSYL (TRANS = 'N', IJOB 0, 1, 3), interleaved complex arrays -------------------------

extern "C" {

void xtgevc3_ztgsyl(char trans, int ijob, int m, int n, const double *A, int lda, const double *B, int ldb, double *C,
                    int ldc, const double *D, int ldd, const double *E, int lde, double *F, int ldf, double *scale,
                    double *dif, int *info)
{
    xtg::tgsyl_host<double, true>(trans, ijob, m, n, A, lda, B, ldb, C, ldc, D, ldd, E, lde, F, ldf, scale, dif, info);
}

void xtgevc3_ctgsyl(char trans, int ijob, int m, int n, const float *A, int lda, const float *B, int ldb, float *C,
                    int ldc, const float *D, int ldd, const float *E, int lde, float *F, int ldf, float *scale,
                    float *dif, int *info)
{
    xtg::tgsyl_host<float, true>(trans, ijob, m, n, A, lda, B, ldb, C, ldc, D, ldd, E, lde, F, ldf, scale, dif, info);
}

int xtgevc3_ztgsyl_dev(void *stream, char trans, int ijob, int m, int n, const double *A, int lda, const double *B,
                       int ldb, double *C, int ldc, const double *D, int ldd, const double *E, int lde, double *F,
                       int ldf, double *scale, double *dif, int *info)
{
    return xtg::tgsyl_device<double, true>(static_cast<cudaStream_t>(stream), trans, ijob, m, n, A, lda, B, ldb, C, ldc,
                                           D, ldd, E, lde, F, ldf, scale, dif, info);
}

int xtgevc3_ctgsyl_dev(void *stream, char trans, int ijob, int m, int n, const float *A, int lda, const float *B,
                       int ldb, float *C, int ldc, const float *D, int ldd, const float *E, int lde, float *F, int ldf,
                       float *scale, float *dif, int *info)
{
    return xtg::tgsyl_device<float, true>(static_cast<cudaStream_t>(stream), trans, ijob, m, n, A, lda, B, ldb, C, ldc,
                                          D, ldd, E, lde, F, ldf, scale, dif, info);
}

}  // extern "C"

// ---- xGGBAL / xGGBAK (JOB 'N' or 'P') -----------------------------------------------------------

using xtg::rb::zc;

extern "C" {

#define XTG_GGBAL(P, E, R)                                                                                          \
    void xtgevc3_##P##ggbal(char job, int n, R *A, int lda, R *B, int ldb, int *ilo, int *ihi, R *lscale, R *rscale, \
                            int *info)                                                                              \
    {                                                                                                               \
        xtg::ggbal_host<E, R>(job, n, reinterpret_cast<E *>(A), lda, reinterpret_cast<E *>(B), ldb, ilo, ihi,       \
                              lscale, rscale, info);                                                                \
    }                                                                                                               \
    int xtgevc3_##P##ggbal_dev(void *stream, char job, int n, R *A, int lda, R *B, int ldb, int *ilo, int *ihi,      \
                               R *lscale, R *rscale, int *info)                                                     \
    {                                                                                                               \
        return xtg::ggbal_device<E, R>(static_cast<cudaStream_t>(stream), job, n, reinterpret_cast<E *>(A), lda,    \
                                       reinterpret_cast<E *>(B), ldb, ilo, ihi, lscale, rscale, info);              \
    }                                                                                                               \
    void xtgevc3_##P##ggbak(char job, char side, int n, int ilo, int ihi, const R *lscale, const R *rscale, int m,   \
                            R *V, int ldv, int *info)                                                               \
    {                                                                                                               \
        xtg::ggbak_host<E, R>(job, side, n, ilo, ihi, lscale, rscale, m, reinterpret_cast<E *>(V), ldv, info);      \
    }                                                                                                               \
    int xtgevc3_##P##ggbak_dev(void *stream, char job, char side, int n, int ilo, int ihi, const R *lscale,          \
                               const R *rscale, int m, R *V, int ldv, int *info)                                    \
    {                                                                                                               \
        return xtg::ggbak_device<E, R>(static_cast<cudaStream_t>(stream), job, side, n, ilo, ihi, lscale, rscale, m, \
                                       reinterpret_cast<E *>(V), ldv, info);                                        \
    }

XTG_GGBAL(d, double, double)
XTG_GGBAL(s, float, float)
XTG_GGBAL(z, zc<double>, double)
XTG_GGBAL(c, zc<float>, float)

#undef XTG_GGBAL

}  // extern "C"
