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
// finite.  Cost: S and P once (16 sums per entry), X once (32 sums per entry).
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

// GA[j][r] = sum_{i <= min(n-1, j + hess)} G(r, i) A(i, j): one warp per column j (A upper
// triangular, hess = 0, or upper Hessenberg, hess = 1).
__global__ void __launch_bounds__(256) sketch_matrix_kernel(const double *A, int lda, int n, int hess, double *GA)
{
    const int j = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (j >= n) return;
    double acc[K];
#pragma unroll
    for (int r = 0; r < K; r++) acc[r] = 0.0;
    const int rows = min(n, j + 1 + hess);
    const double *a = A + (size_t)j * lda;
    for (int i = lane; i < rows; i += 32) {
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
        GA[(size_t)j * K + lane] = v;
    }
}

// Per column c of X (rows [0, kext_c)): T[c] = {GS x_c (16), GP x_c (16), ||x_c||^2}.  A CTA
// of 8 warps takes 8 consecutive columns; rows go in chunks of 32 whose GS / GP rows are
// staged in shared memory (transposed, one row of 32 per sketch row: conflict-free reads).
__global__ void __launch_bounds__(256) sketch_columns_kernel(const double *GS, const double *GP, const double *X,
                                                            int ldx, int m, const int *kext, double *T)
{
    __shared__ double gs[K][33], gp[K][33];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int c0 = blockIdx.x * 8, c = c0 + warp;
    const int kc = c < m ? kext[c] : 0;
    int kmax = 0;
    for (int q = 0; q < 8 && c0 + q < m; q++) kmax = max(kmax, kext[c0 + q]);
    double s[K], p[K], x2 = 0.0;
#pragma unroll
    for (int r = 0; r < K; r++) s[r] = p[r] = 0.0;
    const double *xc = X + (size_t)(c < m ? c : 0) * ldx;
    for (int j0 = 0; j0 < kmax; j0 += 32) {
        __syncthreads();
        for (int e = threadIdx.x; e < 32 * K; e += blockDim.x) {
            const int jj = e / K, r = e % K;
            const bool in = j0 + jj < kmax;
            gs[r][jj] = in ? GS[(size_t)(j0 + jj) * K + r] : 0.0;
            gp[r][jj] = in ? GP[(size_t)(j0 + jj) * K + r] : 0.0;
        }
        __syncthreads();
        const int j = j0 + lane;
        const double xv = (c < m && j < kc) ? xc[j] : 0.0;
        x2 = fma(xv, xv, x2);
#pragma unroll
        for (int r = 0; r < K; r++) {
            s[r] = fma(gs[r][lane], xv, s[r]);
            p[r] = fma(gp[r][lane], xv, p[r]);
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        x2 += __shfl_xor_sync(0xffffffffu, x2, o);
#pragma unroll
        for (int r = 0; r < K; r++) {
            s[r] += __shfl_xor_sync(0xffffffffu, s[r], o);
            p[r] += __shfl_xor_sync(0xffffffffu, p[r], o);
        }
    }
    if (c < m && lane == 0) {
        double *t = T + (size_t)c * (2 * K + 1);
#pragma unroll
        for (int r = 0; r < K; r++) {
            t[r] = s[r];
            t[K + r] = p[r];
        }
        t[2 * K] = x2;
    }
}

// Flags of the columns of each eigenvector (items: first column of each; a pair's two
// columns get one flag).  coef: 4 per column (ac, b_re, b_im, smin); norms: {anorm, bnorm}.
__global__ void refine_flags_kernel(const double *T, const int *items, int nitems, const uint8_t *kind,
                                    const double *coef, const double *norms, double bound, uint8_t *flags,
                                    int *count)
{
    const int it = blockIdx.x * blockDim.x + threadIdx.x;
    if (it >= nitems) return;
    const int c = items[it];
    const double ac = coef[4 * c + 0], br = coef[4 * c + 1], bi = coef[4 * c + 2];
    const double *t = T + (size_t)c * (2 * K + 1);
    double r2 = 0.0, x2 = t[2 * K];
    const bool pair = kind[c] == kPairRe;
    if (!pair) {
        for (int r = 0; r < K; r++) {
            const double v = ac * t[r] - br * t[K + r];
            r2 = fma(v, v, r2);
        }
    } else {
        const double *u = t + (2 * K + 1);  // the Im column
        for (int r = 0; r < K; r++) {
            const double re = ac * t[r] - br * t[K + r] + bi * u[K + r];
            const double im = ac * u[r] - br * u[K + r] - bi * t[K + r];
            r2 = fma(re, re, fma(im, im, r2));
        }
        x2 += u[2 * K];
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
