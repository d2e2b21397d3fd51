// Residual check of the split-precision form (real double): a randomised sketch of
//   r_c = (ac_c S - b_c P) x_c        (problem coordinates, the operator of column c's solve)
// for every computed eigenvector x_c, to flag the columns whose relative residual exceeds a
// bound; the flagged columns are solved again in FP64 (the refinement step).
//
// Sketch.  G is a 16 x n matrix of signs +-1 (bit r of a hash of the row index): with
// GS = G S and GP = G P (16 x n each), G r_c = ac (GS x_c) - b (GP x_c), and ||G r||^2 / 16 is
// an unbiased estimate of ||r||_2^2 (relative spread ~ sqrt(2/16)).  For a (Re, Im) pair the
// complex residual is (ac S - (br + i bi) P)(xr + i xi).  The column's relative residual
//   est_c = ||G r_c|| / 4 / ((|ac| anorm + |b| bnorm) ||x_c||_2)
// is flagged when it exceeds bound / 4 (a margin for the spread of the estimate) or is not
// finite.  Cost: S and P once (16 sums per entry); [GS; GP] X as one FP64 tensor-core GEMM
// (32 x n times the triangular X), and the column norms of X.
#pragma once
#include "common.cuh"

namespace xtg {
namespace refine {

constexpr int K = 16;  // sketch rows

// 16 sign bits for row i of the sketch (a 32-bit integer hash; bit r: sign of G(r, i))
__device__ __forceinline__ uint32_t sign_bits(uint32_t i)
{
    uint32_t h = i * 0x9E3779B1u + 0x7F4A7C15u;
    h ^= h >> 16;
    h *= 0x85EBCA6Bu;
    h ^= h >> 13;
    h *= 0xC2B2AE35u;
    h ^= h >> 16;
    return h;
}

// GA[j * ldg + r] = sum_{i <= min(n-1, j + hess)} G(r, i) A(i, j): one CTA of 256 threads
// per column j (A upper triangular, hess = 0, or upper Hessenberg, hess = 1); GA is the
// 16 x n sketch stored column-major with leading dimension ldg.
__global__ void __launch_bounds__(256) sketch_matrix_kernel(const double *A, int lda, int n, int hess, double *GA,
                                                            int ldg)
{
    __shared__ double part[8][K];
    const int j = blockIdx.x;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    double acc[K];
#pragma unroll
    for (int r = 0; r < K; r++) acc[r] = 0.0;
    const int rows = min(n, j + 1 + hess);
    const double *a = A + (size_t)j * lda;
    for (int i = threadIdx.x; i < rows; i += blockDim.x) {
        const double v = a[i];
        const uint32_t b = sign_bits((uint32_t)i);
#pragma unroll
        for (int r = 0; r < K; r++) acc[r] += ((b >> r) & 1u) ? v : -v;
    }
#pragma unroll
    for (int r = 0; r < K; r++)
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) acc[r] += __shfl_xor_sync(0xffffffffu, acc[r], o);
    if (lane < K) {
        double v = acc[0];
#pragma unroll
        for (int r = 1; r < K; r++)
            if (lane == r) v = acc[r];
        part[warp][lane] = v;
    }
    __syncthreads();
    if (threadIdx.x < K) {
        double v = 0.0;
        for (int w = 0; w < 8; w++) v += part[w][threadIdx.x];
        GA[(size_t)j * ldg + threadIdx.x] = v;
    }
}

// ||x_c||^2 over rows [0, kext_c) of each column of X: one warp per column.
__global__ void __launch_bounds__(256) column_sumsq_kernel(const double *X, int ldx, int m, const int *kext,
                                                           double *x2)
{
    const int c = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (c >= m) return;
    const double *xc = X + (size_t)c * ldx;
    double s = 0.0;
    for (int j = lane; j < kext[c]; j += 32) s = fma(xc[j], xc[j], s);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) x2[c] = s;
}

// Flags of the columns of each eigenvector (items: first column of each; a pair's two
// columns get one flag).  T: 2K x m, column c = {GS x_c, GP x_c}; x2: ||x_c||^2; coef: 4 per
// column (ac, b_re, b_im, smin); norms: {anorm, bnorm}.
__global__ void refine_flags_kernel(const double *T, const double *x2s, const int *items, int nitems,
                                    const uint8_t *kind, const double *coef, const double *norms, double bound,
                                    uint8_t *flags, int *count)
{
    const int it = blockIdx.x * blockDim.x + threadIdx.x;
    if (it >= nitems) return;
    const int c = items[it];
    const double ac = coef[4 * c + 0], br = coef[4 * c + 1], bi = coef[4 * c + 2];
    const double *t = T + (size_t)c * (2 * K);
    double r2 = 0.0, x2 = x2s[c];
    const bool pair = kind[c] == kPairRe;
    if (!pair) {
        for (int r = 0; r < K; r++) {
            const double v = ac * t[r] - br * t[K + r];
            r2 = fma(v, v, r2);
        }
    } else {
        const double *u = t + 2 * K;  // the Im column
        for (int r = 0; r < K; r++) {
            const double re = ac * t[r] - br * t[K + r] + bi * u[K + r];
            const double im = ac * u[r] - br * u[K + r] - bi * t[K + r];
            r2 = fma(re, re, fma(im, im, r2));
        }
        x2 += x2s[c + 1];
    }
    const double est = sqrt(r2 / K);
    const double den = (fabs(ac) * norms[0] + hypot(br, bi) * norms[1]) * sqrt(x2);
    const bool bad = !(est <= 0.25 * bound * den);
    flags[c] = bad ? 1 : 0;
    if (pair) flags[c + 1] = bad ? 1 : 0;
    if (bad) atomicAdd(count, pair ? 2 : 1);
}

}  // namespace refine
}  // namespace xtg
