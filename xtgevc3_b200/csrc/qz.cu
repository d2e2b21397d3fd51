// The generalized Schur form of a pencil on the GPU (LAPACK Z/C/D/SGGES without ordering):
// rb::zgges_cta (qz_cplx.cuh) or rb::dgges_cta (qz_real.cuh) on one CTA; complex alpha =
// diag(S), beta = diag(T), real alphar / alphai / beta as DHGEQZ returns them.
// The three stages are chains of dependent plane rotations, so one CTA runs them (each
// rotation's O(n) rows or columns spread over its threads); the result stays on the device
// for the eigenvector solve that follows (xtgevc3_ztgevc3_dev).
#include "../../include/xtgevc3.h"
#include "common.cuh"
#include "engine.cuh"
#include "qz_real.cuh"

#include <algorithm>
#include <cctype>
#include <string>

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

// LAPACK xGGES's argument checks, numbered by its argument list (JOBVSL, JOBVSR, SORT,
// SELCTG, N, A, LDA, B, LDB, SDIM, ALPHA, BETA, VSL, LDVSL, VSR, LDVSR, ... complex; real
// pencils have ALPHAR, ALPHAI in place of ALPHA, one argument more before VSL)
int gges_check(char jobvsl, char jobvsr, int n, int lda, int ldb, int ldvsl, int ldvsr, bool real = false)
{
    const bool wl = jobvsl == 'V', wr = jobvsr == 'V';
    if (!wl && jobvsl != 'N') return -1;
    if (!wr && jobvsr != 'N') return -2;
    if (n < 0) return -5;
    if (lda < std::max(1, n)) return -7;
    if (ldb < std::max(1, n)) return -9;
    if (ldvsl < 1 || (wl && ldvsl < n)) return real ? -15 : -14;
    if (ldvsr < 1 || (wr && ldvsr < n)) return real ? -17 : -16;
    return 0;
}

// Real pencils, device pointers (alphar, alphai, beta n each).  Returns 0, or 1 when a CUDA
// call failed.
template <class R>
int gges_device_real(cudaStream_t st, char jobvsl, char jobvsr, int n, R *A, int lda, R *B, int ldb, R *alphar,
                     R *alphai, R *beta, R *VSL, int ldvsl, R *VSR, int ldvsr, int *info)
{
    set_last_error("");
    jobvsl = (char)std::toupper((unsigned char)jobvsl);
    jobvsr = (char)std::toupper((unsigned char)jobvsr);
    *info = gges_check(jobvsl, jobvsr, n, lda, ldb, ldvsl, ldvsr, true);
    if (*info) {
        set_last_error("xGGES: argument " + std::to_string(-*info) + " has an illegal value");
        return 0;
    }
    if (n == 0) return 0;
    const int wl = jobvsl == 'V', wr = jobvsr == 'V';
    int *d_info = nullptr, h_info = 0;
    cudaError_t e = cudaMallocAsync(&d_info, sizeof(int), st);
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
    }
    if (e != cudaSuccess) {
        set_last_error(std::string("xGGES: ") + cudaGetErrorString(e));
        *info = n + 1;
        return 1;
    }
    *info = h_info;
    return 0;
}

// Real pencils, host pointers
template <class R>
void gges_host_real(char jobvsl, char jobvsr, int n, R *A, int lda, R *B, int ldb, R *alphar, R *alphai, R *beta,
                    R *VSL, int ldvsl, R *VSR, int ldvsr, int *info)
{
    set_last_error("");
    const char jl = (char)std::toupper((unsigned char)jobvsl), jr = (char)std::toupper((unsigned char)jobvsr);
    *info = gges_check(jl, jr, n, lda, ldb, ldvsl, ldvsr, true);
    if (*info) {
        set_last_error("xGGES: argument " + std::to_string(-*info) + " has an illegal value");
        return;
    }
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
        const int rc = gges_device_real<R>(st, jl, jr, n, dA, n, dB, n, dv, dv + n, dv + 2 * n, dL, wl ? n : 1, dR,
                                           wr ? n : 1, info);
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
// failed (message in last_error()).
template <class R>
int gges_device(cudaStream_t st, char jobvsl, char jobvsr, int n, rb::zc<R> *A, int lda, rb::zc<R> *B, int ldb,
                rb::zc<R> *alpha, rb::zc<R> *beta, rb::zc<R> *VSL, int ldvsl, rb::zc<R> *VSR, int ldvsr, int *info)
{
    set_last_error("");
    jobvsl = (char)std::toupper((unsigned char)jobvsl);
    jobvsr = (char)std::toupper((unsigned char)jobvsr);
    *info = gges_check(jobvsl, jobvsr, n, lda, ldb, ldvsl, ldvsr);
    if (*info) {
        set_last_error("xGGES: argument " + std::to_string(-*info) + " has an illegal value");
        return 0;
    }
    if (n == 0) return 0;
    const int wl = jobvsl == 'V', wr = jobvsr == 'V';
    int *d_info = nullptr, h_info = 0;
    cudaError_t e = cudaMallocAsync(&d_info, sizeof(int), st);
    if (e == cudaSuccess) {
        // Q and Z are not referenced when not wanted
        rb::QzPencil<R> p{n, wl, wr, A, B, wl ? VSL : A, wr ? VSR : A, lda, ldb, wl ? ldvsl : lda, wr ? ldvsr : lda};
        zgges_kernel<R><<<1, kQzThreads, 0, st>>>(p, alpha, beta, d_info);
        count_launches(1);
        e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaMemcpyAsync(&h_info, d_info, sizeof(int), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        cudaFreeAsync(d_info, st);
    }
    if (e != cudaSuccess) {
        set_last_error(std::string("xGGES: ") + cudaGetErrorString(e));
        *info = n + 1;
        return 1;
    }
    *info = h_info;
    return 0;
}

// Host pointers: A, B (and VSL, VSR when wanted) go to the device and come back with alpha, beta.
template <class R>
void gges_host(char jobvsl, char jobvsr, int n, rb::zc<R> *A, int lda, rb::zc<R> *B, int ldb, rb::zc<R> *alpha,
               rb::zc<R> *beta, rb::zc<R> *VSL, int ldvsl, rb::zc<R> *VSR, int ldvsr, int *info)
{
    using C = rb::zc<R>;
    set_last_error("");
    const char jl = (char)std::toupper((unsigned char)jobvsl), jr = (char)std::toupper((unsigned char)jobvsr);
    *info = gges_check(jl, jr, n, lda, ldb, ldvsl, ldvsr);
    if (*info) {
        set_last_error("xGGES: argument " + std::to_string(-*info) + " has an illegal value");
        return;
    }
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
        rc = gges_device<R>(st, jl, jr, n, dA, n, dB, n, dab, dab + n, dL, wl ? n : 1, dR, wr ? n : 1, info);
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

}  // namespace
}  // namespace xtg

using xtg::rb::zc;

extern "C" {

void xtgevc3_zgges(char jobvsl, char jobvsr, int n, double *A, int lda, double *B, int ldb, double *alpha,
                   double *beta, double *VSL, int ldvsl, double *VSR, int ldvsr, int *info)
{
    xtg::gges_host<double>(jobvsl, jobvsr, n, reinterpret_cast<zc<double> *>(A), lda, reinterpret_cast<zc<double> *>(B),
                           ldb, reinterpret_cast<zc<double> *>(alpha), reinterpret_cast<zc<double> *>(beta),
                           reinterpret_cast<zc<double> *>(VSL), ldvsl, reinterpret_cast<zc<double> *>(VSR), ldvsr, info);
}

void xtgevc3_cgges(char jobvsl, char jobvsr, int n, float *A, int lda, float *B, int ldb, float *alpha, float *beta,
                   float *VSL, int ldvsl, float *VSR, int ldvsr, int *info)
{
    xtg::gges_host<float>(jobvsl, jobvsr, n, reinterpret_cast<zc<float> *>(A), lda, reinterpret_cast<zc<float> *>(B), ldb,
                          reinterpret_cast<zc<float> *>(alpha), reinterpret_cast<zc<float> *>(beta),
                          reinterpret_cast<zc<float> *>(VSL), ldvsl, reinterpret_cast<zc<float> *>(VSR), ldvsr, info);
}

int xtgevc3_zgges_dev(void *stream, char jobvsl, char jobvsr, int n, double *A, int lda, double *B, int ldb,
                      double *alpha, double *beta, double *VSL, int ldvsl, double *VSR, int ldvsr, int *info)
{
    return xtg::gges_device<double>(static_cast<cudaStream_t>(stream), jobvsl, jobvsr, n,
                                    reinterpret_cast<zc<double> *>(A), lda, reinterpret_cast<zc<double> *>(B), ldb,
                                    reinterpret_cast<zc<double> *>(alpha), reinterpret_cast<zc<double> *>(beta),
                                    reinterpret_cast<zc<double> *>(VSL), ldvsl, reinterpret_cast<zc<double> *>(VSR),
                                    ldvsr, info);
}

int xtgevc3_cgges_dev(void *stream, char jobvsl, char jobvsr, int n, float *A, int lda, float *B, int ldb, float *alpha,
                      float *beta, float *VSL, int ldvsl, float *VSR, int ldvsr, int *info)
{
    return xtg::gges_device<float>(static_cast<cudaStream_t>(stream), jobvsl, jobvsr, n,
                                   reinterpret_cast<zc<float> *>(A), lda, reinterpret_cast<zc<float> *>(B), ldb,
                                   reinterpret_cast<zc<float> *>(alpha), reinterpret_cast<zc<float> *>(beta),
                                   reinterpret_cast<zc<float> *>(VSL), ldvsl, reinterpret_cast<zc<float> *>(VSR), ldvsr,
                                   info);
}

void xtgevc3_dgges(char jobvsl, char jobvsr, int n, double *A, int lda, double *B, int ldb, double *alphar,
                   double *alphai, double *beta, double *VSL, int ldvsl, double *VSR, int ldvsr, int *info)
{
    xtg::gges_host_real<double>(jobvsl, jobvsr, n, A, lda, B, ldb, alphar, alphai, beta, VSL, ldvsl, VSR, ldvsr, info);
}

void xtgevc3_sgges(char jobvsl, char jobvsr, int n, float *A, int lda, float *B, int ldb, float *alphar, float *alphai,
                   float *beta, float *VSL, int ldvsl, float *VSR, int ldvsr, int *info)
{
    xtg::gges_host_real<float>(jobvsl, jobvsr, n, A, lda, B, ldb, alphar, alphai, beta, VSL, ldvsl, VSR, ldvsr, info);
}

int xtgevc3_dgges_dev(void *stream, char jobvsl, char jobvsr, int n, double *A, int lda, double *B, int ldb,
                      double *alphar, double *alphai, double *beta, double *VSL, int ldvsl, double *VSR, int ldvsr,
                      int *info)
{
    return xtg::gges_device_real<double>(static_cast<cudaStream_t>(stream), jobvsl, jobvsr, n, A, lda, B, ldb, alphar,
                                         alphai, beta, VSL, ldvsl, VSR, ldvsr, info);
}

int xtgevc3_sgges_dev(void *stream, char jobvsl, char jobvsr, int n, float *A, int lda, float *B, int ldb,
                      float *alphar, float *alphai, float *beta, float *VSL, int ldvsl, float *VSR, int ldvsr, int *info)
{
    return xtg::gges_device_real<float>(static_cast<cudaStream_t>(stream), jobvsl, jobvsr, n, A, lda, B, ldb, alphar,
                                        alphai, beta, VSL, ldvsl, VSR, ldvsr, info);
}

}  // extern "C"
