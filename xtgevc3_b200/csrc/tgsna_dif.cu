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

using rb::DifItem;
using rb::dif_work_elems;
using rb::zdif_work_elems;

template <class R>
__global__ void __launch_bounds__(kDifThreads)
    tgsna_dif_kernel(int n, const R *A, int lda, const R *B, int ldb, const DifItem *items, int count, R *dif,
                     R *work, size_t per_cta, int *err)
{
    __shared__ rb::DifShared<R> sh;
    rb::dif_cta(rb::CtaDev{}, sh, n, A, lda, B, ldb, items, count, dif, work, per_cta, err);
}

template <class R>
__global__ void __launch_bounds__(kDifThreads)
    tgsna_dif_cplx_kernel(int n, const rb::zc<R> *A, int lda, const rb::zc<R> *B, int ldb, const DifItem *items,
                          int count, R *dif, rb::zc<R> *work, size_t per_cta)
{
    __shared__ rb::ZDifShared<R> sh;
    rb::zdif_cta(rb::CtaDev{}, sh, n, A, lda, B, ldb, items, count, dif, work, per_cta);
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
