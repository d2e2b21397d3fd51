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
// finite.  Cost: S and P once (16 sums per entry each), X once (32 sums per entry).
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

// G2 = [G S; G P], 2K x n column-major (leading dimension 2K): one CTA of 256 threads per
// column j sums G(r, i) S(i, j) over rows i <= min(n-1, j+1) (S upper Hessenberg) and
// G(r, i) P(i, j) over i <= j (P upper triangular), one sign word per row.
__global__ void __launch_bounds__(256) sketch_matrix_kernel(const double *S, int lds, const double *P, int ldp, int n,
                                                            double *G2)
{
    __shared__ double part[8][2 * K];
    const int j = blockIdx.x;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    double acc[2 * K];
#pragma unroll
    for (int r = 0; r < 2 * K; r++) acc[r] = 0.0;
    const int rows = min(n, j + 2);
    const double *sc = S + (size_t)j * lds, *pc = P + (size_t)j * ldp;
    for (int i = threadIdx.x; i < rows; i += blockDim.x) {
        const double vs = sc[i], vp = i <= j ? pc[i] : 0.0;
        const uint32_t b = sign_bits((uint32_t)i);
#pragma unroll
        for (int r = 0; r < K; r++) {
            const bool plus = (b >> r) & 1u;
            acc[r] += plus ? vs : -vs;
            acc[K + r] += plus ? vp : -vp;
        }
    }
#pragma unroll
    for (int r = 0; r < 2 * K; r++)
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) acc[r] += __shfl_xor_sync(0xffffffffu, acc[r], o);
    double v = acc[0];
#pragma unroll
    for (int r = 1; r < 2 * K; r++)
        if (lane == r) v = acc[r];
    part[warp][lane] = v;
    __syncthreads();
    if (threadIdx.x < 2 * K) {
        double t = 0.0;
        for (int w = 0; w < 8; w++) t += part[w][threadIdx.x];
        G2[(size_t)j * 2 * K + threadIdx.x] = t;
    }
}

// T[:, c] = G2 X[:, c] (2K sums per column over its rows [0, kext_c)) and x2[c] = ||x_c||^2.
// A CTA of 256 threads takes 64 consecutive columns and walks their rows in chunks of 32,
// staged in shared memory with the chunk's 32 x 2K sketch entries; thread t computes 8 of
// the 2K sums (rows 8 (t / 64) .. +7 of T) of column t % 64 and, for t < 64, the norm.
__global__ void __launch_bounds__(256) sketch_columns_kernel(const double *G2, const double *X, int ldx, int m,
                                                            const int *kext, double *T, double *x2)
{
    __shared__ double xs[32][65];
    __shared__ double gs[32][2 * K + 1];
    const int c0 = blockIdx.x * 64, tc = threadIdx.x & 63, rg = threadIdx.x >> 6;
    const int c = c0 + tc;
    int kmax = 0;
    for (int q = 0; q < 64 && c0 + q < m; q++) kmax = max(kmax, kext[c0 + q]);
    double acc[8], nrm = 0.0;
#pragma unroll
    for (int r = 0; r < 8; r++) acc[r] = 0.0;
    for (int j0 = 0; j0 < kmax; j0 += 32) {
        __syncthreads();
        for (int e = threadIdx.x; e < 32 * 64; e += 256) {  // X chunk: 32 rows x 64 columns
            const int jj = e & 31, cc = e >> 5, col = c0 + cc, j = j0 + jj;
            xs[jj][cc] = (col < m && j < kext[col]) ? X[(size_t)col * ldx + j] : 0.0;
        }
        for (int e = threadIdx.x; e < 32 * 2 * K; e += 256) {  // sketch rows of the chunk
            const int jj = e / (2 * K), r = e % (2 * K), j = j0 + jj;
            gs[jj][r] = j < kmax ? G2[(size_t)j * 2 * K + r] : 0.0;
        }
        __syncthreads();
#pragma unroll 4
        for (int jj = 0; jj < 32; jj++) {
            const double xv = xs[jj][tc];
            if (rg == 0) nrm = fma(xv, xv, nrm);
#pragma unroll
            for (int r = 0; r < 8; r++) acc[r] = fma(gs[jj][8 * rg + r], xv, acc[r]);
        }
    }
    if (c < m) {
#pragma unroll
        for (int r = 0; r < 8; r++) T[(size_t)c * 2 * K + 8 * rg + r] = acc[r];
        if (rg == 0) x2[c] = nrm;
    }
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
