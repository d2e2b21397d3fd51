// DIF of LAPACK D/STGSNA (JOB = 'V' / 'B') on the GPU: one CTA per selected eigenvalue (1x1
// block) or complex pair (2x2 block) at a time, over a grid sized by the workspace:
//   1. the CTA copies (A, B) into its workspace and moves the block to the top with the real
//      reordering walk (tgexc_real_blocks.cuh: thread 0 computes each swap, the CTA applies it;
//      the same loop as the reordering kernel, bounded by 4 n + 16 swaps);
//   2. xTGSYL's Frobenius-norm estimate over the rest of the pencil (tgsna_dif.cuh): thread 0
//      solves each xTGSYL block's small Kronecker systems (xGETC2, xLATDF's +-1 look-ahead),
//      the CTA updates the rows above the block;
//   3. DIF = sqrt(2 n1 n2) / ||solutions||_F, a pair's own bound (xLAG2) taken as well; a
//      rejected swap gives DIF = 0, as in LAPACK.
// Complex pencils (Z/CTGSNA, tgsna_dif_cplx.cuh): the same steps with ZTGEX2's rotation swaps
// (at most n - 1 of them) and ZTGSYL's estimate over the diagonal entries.
#include "../../include/xtgevc3.h"
#include "common.cuh"
#include "engine.cuh"
#include "tgsna_dif.cuh"
#include "tgsna_dif_cplx.cuh"

#include <algorithm>
#include <string>
#include <vector>

namespace xtg {
namespace {

constexpr int kDifThreads = 256;

struct DifItem {
    int k, ks, pair;  // first row of the block (0-based), index of its DIF, complex pair
};

// workspace of one CTA, in elements of R: the reordered copy (2 n^2), C and F (n x 2 each),
// xTGSYL's block starts (n / 2 + 4 ints, n + 8 elements of room)
inline size_t dif_work_elems(int n) { return 2 * (size_t)n * n + 4 * (size_t)n + (size_t)n + 8; }

template <class R>
__global__ void __launch_bounds__(kDifThreads)
    tgsna_dif_kernel(int n, const R *A, int lda, const R *B, int ldb, const DifItem *items, int count, R *dif,
                     R *work, size_t per_cta, int *err)
{
    __shared__ rb::Swap<R> s;
    __shared__ rb::Walk w;
    __shared__ rb::Sylv<R> y;
    __shared__ int s_go, s_info, s_nbk;
    __shared__ R s_cond, s_d;
    R *Aw = work + blockIdx.x * per_cta;
    R *Bw = Aw + (size_t)n * n;
    R *Cw = Bw + (size_t)n * n;
    R *Fw = Cw + 2 * (size_t)n;
    int *starts = reinterpret_cast<int *>(Fw + 2 * (size_t)n);
    for (int it = blockIdx.x; it < count; it += gridDim.x) {
        const DifItem item = items[it];
        if (n == 1) {
            if (threadIdx.x == 0) dif[item.ks] = rb::lapy2(A[0], B[0]);
            continue;
        }
        for (size_t e = threadIdx.x; e < (size_t)n * n; e += blockDim.x) {
            const size_t i = e % n, j = e / n;
            Aw[e] = A[i + j * lda];
            Bw[e] = B[i + j * ldb];
        }
        for (int e = threadIdx.x; e < 2 * n; e += blockDim.x) {
            Cw[e] = R(0);
            Fw[e] = R(0);
        }
        const rb::Pencil<R> p{n, 0, 0, Aw, Bw, nullptr, nullptr, n, n, 1, 1};
        if (threadIdx.x == 0) {
            const int k = item.k;
            s_cond = R(0);
            if (item.pair)
                s_cond = rb::pair_cond(A[k + (size_t)k * lda], A[k + 1 + (size_t)k * lda], A[k + (size_t)(k + 1) * lda],
                                       A[k + 1 + (size_t)(k + 1) * lda], B[k + (size_t)k * ldb],
                                       B[k + 1 + (size_t)k * ldb], B[k + (size_t)(k + 1) * ldb],
                                       B[k + 1 + (size_t)(k + 1) * ldb]);
        }
        __syncthreads();  // the copy is complete before thread 0 reads it
        if (threadIdx.x == 0) {
            int f = item.k + 1, l = 1;
            s_go = rb::walk_begin(p, w, f, l) ? 1 : 0;
            s_info = 0;
            s.ok = 0;
            s.n1 = s.n2 = 1;
        }
        const int limit = 4 * n + 16;
        for (int step = 0;; step++) {  // the reordering kernel's walk loop
            if (threadIdx.x == 0 && s_go) {
                int j1, n1, n2;
                if (step >= limit) {
                    s_go = 0;
                    s_info = 3;
                } else if (!rb::walk_next(p, w, j1, n1, n2)) {
                    s_go = 0;
                } else {
                    s.j1 = j1 - 1;
                    s.n1 = n1;
                    s.n2 = n2;
                    rb::swap_prepare(p, s);
                    if (s.ok == 0) {
                        s_go = 0;
                        s_info = 1;
                    }
                }
            }
            __syncthreads();
            const int go = s_go, ok = s.ok, m = s.n1 + s.n2;
            if (!go) break;
            if (ok == 1) {
                rb::swap_apply(p, s, 0, threadIdx.x, blockDim.x);
                if (m == 2) {
                    __syncthreads();
                    rb::swap_apply(p, s, 1, threadIdx.x, blockDim.x);
                    __syncthreads();
                    rb::swap_apply(p, s, 2, threadIdx.x, blockDim.x);
                }
            }
            __syncthreads();
            if (threadIdx.x == 0) rb::walk_after(p, w);
        }
        __syncthreads();  // every thread has left the walk before its state is reused
        if (threadIdx.x == 0) {
            s_nbk = 0;
            s_d = R(0);  // a rejected swap: DIF = 0
            if (s_info == 3) atomicExch(err, 1);
            if (s_info == 0) {
                const int n1 = Aw[1] != R(0) ? 2 : 1;
                if (n - n1 == 0) {
                    s_d = s_cond;
                } else {
                    y.n1 = n1;
                    y.n2 = n - n1;
                    y.ld = n;
                    y.ldc = n;
                    y.A22 = Aw + n1 + (size_t)n1 * n;
                    y.B22 = Bw + n1 + (size_t)n1 * n;
                    for (int q = 0; q < 16; q++) {
                        y.A11s[q] = R(0);
                        y.B11s[q] = R(0);
                    }
                    for (int j = 0; j < n1; j++)
                        for (int i = 0; i < n1; i++) {
                            y.A11s[i + rb::LD * j] = Aw[i + (size_t)j * n];
                            y.B11s[i + rb::LD * j] = Bw[i + (size_t)j * n];
                        }
                    y.C = Cw;
                    y.F = Fw;
                    y.dsum = R(1);
                    y.dscale = R(0);
                    s_nbk = rb::tgsyl_blocks(y, starts);
                }
            }
        }
        __syncthreads();
        const int nbk = s_nbk;
        for (int b = nbk - 1; b >= 0; b--) {
            if (threadIdx.x == 0) rb::tgsyl_block(y, starts[b], starts[b + 1] - 1);
            __syncthreads();
            rb::tgsyl_update_above(y, starts[b], starts[b + 1] - 1, (int)threadIdx.x, (int)blockDim.x);
            __syncthreads();
        }
        if (threadIdx.x == 0) {
            R d = s_d;
            if (nbk > 0) {
                d = rb::xsqrt(R(2 * y.n1 * y.n2)) / (y.dscale * rb::xsqrt(y.dsum));
                if (item.pair) d = rb::xmin(d, s_cond);
            }
            dif[item.ks] = d;
            if (item.pair) dif[item.ks + 1] = d;
        }
        __syncthreads();  // the workspace is reused by the next item
    }
}

// Complex pencils: one CTA per eigenvalue, as above.  status: none needed (the walk is at most
// k swaps).  Workspace of one CTA in complex elements: the copy (2 n^2), C and F (n each),
// ZTGSYL's block starts (n / 2 + 4 ints, n + 8 elements of room).
inline size_t zdif_work_elems(int n) { return 2 * (size_t)n * n + 3 * (size_t)n + 8; }

template <class R>
__global__ void __launch_bounds__(kDifThreads)
    tgsna_dif_cplx_kernel(int n, const rb::zc<R> *A, int lda, const rb::zc<R> *B, int ldb, const DifItem *items,
                          int count, R *dif, rb::zc<R> *work, size_t per_cta)
{
    using C = rb::zc<R>;
    __shared__ rb::ZSwap<R> s;
    __shared__ rb::ZSylv<R> y;
    __shared__ int s_rej, s_nbk;
    C *Aw = work + blockIdx.x * per_cta;
    C *Bw = Aw + (size_t)n * n;
    C *Cw = Bw + (size_t)n * n;
    C *Fw = Cw + n;
    int *starts = reinterpret_cast<int *>(Fw + n);
    for (int it = blockIdx.x; it < count; it += gridDim.x) {
        const DifItem item = items[it];
        if (n == 1) {
            if (threadIdx.x == 0) dif[item.ks] = rb::lapy2(rb::cabs(A[0]), rb::cabs(B[0]));
            continue;
        }
        for (size_t e = threadIdx.x; e < (size_t)n * n; e += blockDim.x) {
            const size_t i = e % n, j = e / n;
            Aw[e] = A[i + j * lda];
            Bw[e] = B[i + j * ldb];
        }
        for (int e = threadIdx.x; e < n; e += blockDim.x) {
            Cw[e] = rb::mk(R(0), R(0));
            Fw[e] = rb::mk(R(0), R(0));
        }
        if (threadIdx.x == 0) s_rej = 0;
        __syncthreads();  // the copy is complete before thread 0 reads it
        for (int here = item.k; here > 0; here--) {  // the eigenvalue moves up one row per swap
            if (threadIdx.x == 0) {
                s.j = here - 1;
                rb::zswap_prepare(Aw, Bw, n, s);
                s_rej = s.ok ? 0 : 1;
            }
            __syncthreads();
            if (s_rej) break;
            rb::zswap_apply(Aw, Bw, n, n, s, 0, (int)threadIdx.x, (int)blockDim.x);
            __syncthreads();  // the 2x2 block takes the column rotation before the row rotation
            rb::zswap_apply(Aw, Bw, n, n, s, 1, (int)threadIdx.x, (int)blockDim.x);
            __syncthreads();
            rb::zswap_apply(Aw, Bw, n, n, s, 2, (int)threadIdx.x, (int)blockDim.x);
            __syncthreads();
        }
        __syncthreads();  // every thread has left the walk
        if (threadIdx.x == 0) {
            s_nbk = 0;
            if (!s_rej) {
                y.n2 = n - 1;
                y.ld = n;
                y.A22 = Aw + 1 + (size_t)n;
                y.B22 = Bw + 1 + (size_t)n;
                y.a11 = Aw[0];
                y.b11 = Bw[0];
                y.C = Cw;
                y.F = Fw;
                y.dsum = R(1);
                y.dscale = R(0);
                s_nbk = rb::ztgsyl_blocks(n - 1, starts);
            }
        }
        __syncthreads();
        const int nbk = s_nbk;
        for (int b = nbk - 1; b >= 0; b--) {
            if (threadIdx.x == 0) rb::ztgsyl_block(y, starts[b], starts[b + 1] - 1);
            __syncthreads();
            rb::ztgsyl_update_above(y, starts[b], starts[b + 1] - 1, (int)threadIdx.x, (int)blockDim.x);
            __syncthreads();
        }
        if (threadIdx.x == 0)  // a rejected swap: DIF = 0
            dif[item.ks] = nbk > 0 ? rb::xsqrt(R(2 * y.n2)) / (y.dscale * rb::xsqrt(y.dsum)) : R(0);
        __syncthreads();  // the workspace is reused by the next item
    }
}

}  // namespace

template <class R>
int dif_device(int n, const R *A, int lda, const R *B, int ldb, const std::vector<int> &rows,
               const std::vector<int> &outs, const std::vector<uint8_t> &pairs, R *dif_dev, cudaStream_t st)
{
    const int count = (int)rows.size();
    if (count == 0) return 0;
    std::vector<DifItem> h(count);
    for (int i = 0; i < count; i++) h[i] = DifItem{rows[i], outs[i], pairs[i] ? 1 : 0};
    const size_t per = dif_work_elems(n);
    // CTAs: up to four per SM, within a 4 GiB workspace (at least one)
    const size_t budget = (size_t)4 << 30;
    const size_t cap = std::max<size_t>(1, budget / (per * sizeof(R)));
    const int grid = (int)std::min<size_t>({(size_t)count, cap, (size_t)4 * 148});
    DifItem *d_items = nullptr;
    R *d_work = nullptr;
    int *d_err = nullptr;
    int h_err = 0;
    cudaError_t e = cudaMallocAsync(&d_items, count * sizeof(DifItem), st);
    if (e == cudaSuccess) e = cudaMallocAsync(&d_work, (size_t)grid * per * sizeof(R), st);
    if (e == cudaSuccess) e = cudaMallocAsync(&d_err, sizeof(int), st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_items, h.data(), count * sizeof(DifItem), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(d_err, 0, sizeof(int), st);
    if (e == cudaSuccess) {
        tgsna_dif_kernel<R><<<grid, kDifThreads, 0, st>>>(n, A, lda, B, ldb, d_items, count, dif_dev, d_work, per,
                                                           d_err);
        count_launches(1);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(&h_err, d_err, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    for (void *q : {(void *)d_items, (void *)d_work, (void *)d_err})
        if (q) cudaFreeAsync(q, st);
    if (e != cudaSuccess) {
        set_last_error(std::string("xTGSNA DIF: ") + cudaGetErrorString(e));
        return 1;
    }
    if (h_err) {
        set_last_error("xTGSNA DIF: a reordering walk did not end within its swap bound");
        return 1;
    }
    return 0;
}

template <class R>
int dif_device_cplx(int n, const R *A, int lda, const R *B, int ldb, const std::vector<int> &rows,
                    const std::vector<int> &outs, R *dif_dev, cudaStream_t st)
{
    using C = rb::zc<R>;
    const int count = (int)rows.size();
    if (count == 0) return 0;
    std::vector<DifItem> h(count);
    for (int i = 0; i < count; i++) h[i] = DifItem{rows[i], outs[i], 0};
    const size_t per = zdif_work_elems(n);
    const size_t budget = (size_t)4 << 30;
    const size_t cap = std::max<size_t>(1, budget / (per * sizeof(C)));
    const int grid = (int)std::min<size_t>({(size_t)count, cap, (size_t)4 * 148});
    DifItem *d_items = nullptr;
    C *d_work = nullptr;
    cudaError_t e = cudaMallocAsync(&d_items, count * sizeof(DifItem), st);
    if (e == cudaSuccess) e = cudaMallocAsync(&d_work, (size_t)grid * per * sizeof(C), st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_items, h.data(), count * sizeof(DifItem), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) {
        tgsna_dif_cplx_kernel<R><<<grid, kDifThreads, 0, st>>>(n, reinterpret_cast<const C *>(A), lda,
                                                                reinterpret_cast<const C *>(B), ldb, d_items, count,
                                                                dif_dev, d_work, per);
        count_launches(1);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    for (void *q : {(void *)d_items, (void *)d_work})
        if (q) cudaFreeAsync(q, st);
    if (e != cudaSuccess) {
        set_last_error(std::string("xTGSNA DIF: ") + cudaGetErrorString(e));
        return 1;
    }
    return 0;
}

template int dif_device<double>(int, const double *, int, const double *, int, const std::vector<int> &,
                                const std::vector<int> &, const std::vector<uint8_t> &, double *, cudaStream_t);
template int dif_device<float>(int, const float *, int, const float *, int, const std::vector<int> &,
                               const std::vector<int> &, const std::vector<uint8_t> &, float *, cudaStream_t);

template int dif_device_cplx<double>(int, const double *, int, const double *, int, const std::vector<int> &,
                                     const std::vector<int> &, double *, cudaStream_t);
template int dif_device_cplx<float>(int, const float *, int, const float *, int, const std::vector<int> &,
                                    const std::vector<int> &, float *, cudaStream_t);

}  // namespace xtg
