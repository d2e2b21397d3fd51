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

constexpr int ROWS = 512;  // rows of one chunk of a sketch

// Chunk c of the row-chunked sketches covers rows [c ROWS, (c + 1) ROWS); each chunk's partial
// sums go to their own slice of a [chunks][columns][2K] buffer (zeroed by the caller), summed
// afterwards in chunk order, so the sketch is the same from run to run.
inline int sketch_chunks(int rows) { return (rows + ROWS - 1) / ROWS; }

// Both sketches are products (2K or K rows) x (columns) of a row-chunk of sign or sketch
// entries with a column block of a matrix: a CTA of 256 threads takes 128 consecutive columns
// over one chunk of rows, in steps of JS rows; the step's matrix entries (JS x 128, column
// pairs adjacent) and its sketch entries sit in shared memory, and thread t sums 8 sketch
// rows for 2 adjacent columns (16 FMAs per row step against one 16-byte load of the column
// pair and four broadcast 16-byte loads of sketch entries).  Each thread holds the next
// step's global loads in registers while the current step is summed (one load latency per
// step, overlapped).
constexpr int SK_COLS = 128;

// Partial G2 = [G S; G P] (2K x n column-major, leading dimension 2K) of one row chunk.
// Grid (n / 128, chunks).  S(i, j) is read for i <= j + 1 (S upper Hessenberg), P(i, j) for
// i <= j (P upper triangular).  Thread t: column pair t % 64, 8 G2 rows (t / 64 = 0, 1: GS
// rows 0..7, 8..15; 2, 3: GP rows 0..7, 8..15).  The signs G(r, i) = +-1 are staged as doubles.
__global__ void __launch_bounds__(256, 2) sketch_matrix_kernel(const double *S, int lds, const double *P, int ldp, int n,
                                                            double *G2p)
{
    constexpr int JS = 16, NL = JS * SK_COLS / 256;  // loads per thread and matrix
    __shared__ __align__(16) double xs[2][JS][SK_COLS + 2];
    __shared__ __align__(16) double gs[JS][K];
    const int c0 = blockIdx.x * SK_COLS, tp = threadIdx.x & 63, grp = threadIdx.x >> 6;
    const int mat = grp >> 1, r0 = (grp & 1) * 8;
    const int jbeg = blockIdx.y * ROWS, jend = min(min(n, c0 + SK_COLS + 1), jbeg + ROWS);
    if (jbeg >= jend) return;
    // element q of a step: row jj = t % JS, column cc = t / JS + (256 / JS) q
    const int ljj = threadIdx.x % JS, lcc = threadIdx.x / JS;
    double vs[NL], vp[NL];
    auto load = [&](int j0) {
        const int j = j0 + ljj;
#pragma unroll
        for (int q = 0; q < NL; q++) {
            const int col = c0 + lcc + (256 / JS) * q;
            const bool in = col < n && j < jend;
            vs[q] = (in && j <= col + 1) ? S[(size_t)col * lds + j] : 0.0;
            vp[q] = (in && j <= col) ? P[(size_t)col * ldp + j] : 0.0;
        }
    };
    double acc[8][2];
#pragma unroll
    for (int r = 0; r < 8; r++) acc[r][0] = acc[r][1] = 0.0;
    load(jbeg);
    for (int j0 = jbeg; j0 < jend; j0 += JS) {
        __syncthreads();
#pragma unroll
        for (int q = 0; q < NL; q++) {
            xs[0][ljj][lcc + (256 / JS) * q] = vs[q];
            xs[1][ljj][lcc + (256 / JS) * q] = vp[q];
        }
        {
            const int jj = threadIdx.x / K, r = threadIdx.x % K;  // 256 = JS x K
            gs[jj][r] = (sign_bits((uint32_t)(j0 + jj)) >> r) & 1u ? 1.0 : -1.0;
        }
        __syncthreads();
        if (j0 + JS < jend) load(j0 + JS);
#pragma unroll
        for (int jj = 0; jj < JS; jj++) {
            const double2 x = *reinterpret_cast<const double2 *>(&xs[mat][jj][2 * tp]);
#pragma unroll
            for (int r = 0; r < 8; r += 2) {
                const double2 gv = *reinterpret_cast<const double2 *>(&gs[jj][r0 + r]);
                acc[r][0] = fma(gv.x, x.x, acc[r][0]);
                acc[r][1] = fma(gv.x, x.y, acc[r][1]);
                acc[r + 1][0] = fma(gv.y, x.x, acc[r + 1][0]);
                acc[r + 1][1] = fma(gv.y, x.y, acc[r + 1][1]);
            }
        }
    }
#pragma unroll
    for (int q = 0; q < 2; q++) {
        const int c = c0 + 2 * tp + q;
        if (c < n) {
            double *g = G2p + ((size_t)blockIdx.y * n + c) * 2 * K + mat * K + r0;
#pragma unroll
            for (int r = 0; r < 8; r++) g[r] = acc[r][q];
        }
    }
}

// out = sum over chunks of part (chunk order), len entries per chunk.
__global__ void sum_chunks_kernel(const double *part, int chunks, size_t len, double *out)
{
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < len; i += (size_t)gridDim.x * blockDim.x) {
        double t = 0.0;
        for (int ch = 0; ch < chunks; ch++) t += part[ch * len + i];
        out[i] = t;
    }
}

// Partial T[:, c] = G2 X[:, c] (2K sums per column over its rows [0, kext_c)) and x2[c] =
// ||x_c||^2 of one row chunk.  Grid (m / 128, chunks).  Thread t: column pair t % 64, T rows
// 8 (t / 64) .. +7; the threads with t < 64 also sum the pair's squares.
__global__ void __launch_bounds__(256, 2) sketch_columns_kernel(const double *G2, const double *X, int ldx, int m,
                                                            const int *kext, double *Tp, double *x2p)
{
    constexpr int JS = 32, NL = JS * SK_COLS / 256, NG = JS * 2 * K / 256;
    __shared__ __align__(16) double xs[JS][SK_COLS + 2];
    __shared__ __align__(16) double gs[JS][2 * K];
    __shared__ int kx[SK_COLS];
    __shared__ int wmax[8];
    const int c0 = blockIdx.x * SK_COLS, tp = threadIdx.x & 63, rg = threadIdx.x >> 6;
    int kmax = 0;
    if (threadIdx.x < SK_COLS) {
        const int k = c0 + threadIdx.x < m ? kext[c0 + threadIdx.x] : 0;
        kx[threadIdx.x] = k;
        kmax = k;
    }
    kmax = __reduce_max_sync(0xffffffffu, kmax);
    if ((threadIdx.x & 31) == 0) wmax[threadIdx.x >> 5] = kmax;
    __syncthreads();
    kmax = 0;
#pragma unroll
    for (int w = 0; w < 8; w++) kmax = max(kmax, wmax[w]);
    const int jbeg = blockIdx.y * ROWS, jend = min(kmax, jbeg + ROWS);
    if (jbeg >= jend) return;
    // X element q of a step: row jj = lane, column cc = warp + 8 q; sketch entry q: row
    // (t + 256 q) / 2K, entry (t + 256 q) % 2K
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    double vx[NL], vg[NG];
    auto load = [&](int j0) {
        const int j = j0 + lane;
#pragma unroll
        for (int q = 0; q < NL; q++) {
            const int cc = warp + 8 * q;
            vx[q] = (j < jend && j < kx[cc]) ? X[(size_t)(c0 + cc) * ldx + j] : 0.0;
        }
#pragma unroll
        for (int q = 0; q < NG; q++) {
            const int e = threadIdx.x + 256 * q, jr = j0 + e / (2 * K);
            vg[q] = jr < jend ? G2[(size_t)jr * 2 * K + e % (2 * K)] : 0.0;
        }
    };
    double acc[8][2], n0 = 0.0, n1 = 0.0;
#pragma unroll
    for (int r = 0; r < 8; r++) acc[r][0] = acc[r][1] = 0.0;
    load(jbeg);
    for (int j0 = jbeg; j0 < jend; j0 += JS) {
        __syncthreads();
#pragma unroll
        for (int q = 0; q < NL; q++) xs[lane][warp + 8 * q] = vx[q];
#pragma unroll
        for (int q = 0; q < NG; q++) {
            const int e = threadIdx.x + 256 * q;
            gs[e / (2 * K)][e % (2 * K)] = vg[q];
        }
        __syncthreads();
        if (j0 + JS < jend) load(j0 + JS);
#pragma unroll 8
        for (int jj = 0; jj < JS; jj++) {
            const double2 x = *reinterpret_cast<const double2 *>(&xs[jj][2 * tp]);
            if (rg == 0) {
                n0 = fma(x.x, x.x, n0);
                n1 = fma(x.y, x.y, n1);
            }
#pragma unroll
            for (int r = 0; r < 8; r += 2) {
                const double2 gv = *reinterpret_cast<const double2 *>(&gs[jj][8 * rg + r]);
                acc[r][0] = fma(gv.x, x.x, acc[r][0]);
                acc[r][1] = fma(gv.x, x.y, acc[r][1]);
                acc[r + 1][0] = fma(gv.y, x.x, acc[r + 1][0]);
                acc[r + 1][1] = fma(gv.y, x.y, acc[r + 1][1]);
            }
        }
    }
#pragma unroll
    for (int q = 0; q < 2; q++) {
        const int c = c0 + 2 * tp + q;
        if (c < m) {
            double *t = Tp + ((size_t)blockIdx.y * m + c) * 2 * K + 8 * rg;
#pragma unroll
            for (int r = 0; r < 8; r++) t[r] = acc[r][q];
            if (rg == 0) x2p[(size_t)blockIdx.y * m + c] = q ? n1 : n0;
        }
    }
}

// Flags of the columns of each eigenvector (items: first column of each; a pair's two
// columns get one flag), one warp per item, lane r holding sketch row r.  Tp: chunks x m x 2K
// partial sketches, column c of T = {GS x_c, GP x_c}; x2p: chunks x m partial ||x_c||^2;
// coef: 4 per column (ac, b_re, b_im, smin); norms: {anorm, bnorm}.
__global__ void __launch_bounds__(256) refine_flags_kernel(const double *Tp, const double *x2p, int chunks, int m,
                                                          const int *items, int nitems, const uint8_t *kind,
                                                          const double *coef, const double *norms, double bound,
                                                          uint8_t *flags, int *count)
{
    const int it = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (it >= nitems) return;
    const int c = items[it];
    const double ac = coef[4 * c + 0], br = coef[4 * c + 1], bi = coef[4 * c + 2];
    const bool pair = kind[c] == kPairRe;
    double t0 = 0.0, t1 = 0.0, x2 = 0.0;  // T(lane, c), T(lane, c + 1); lane 0, 1: ||x||^2 parts
    for (int ch = 0; ch < chunks; ch++) {
        const double *src = Tp + ((size_t)ch * m + c) * 2 * K;
        t0 += src[lane];
        if (pair) t1 += src[2 * K + lane];
        if (lane < (pair ? 2 : 1)) x2 += x2p[(size_t)ch * m + c + lane];
    }
    // lane r < K: residual sketch row r from {GS x}(r) (lane r) and {GP x}(r) (lane K + r)
    const double p0 = __shfl_down_sync(0xffffffffu, t0, K), p1 = __shfl_down_sync(0xffffffffu, t1, K);
    double r2 = 0.0;
    if (lane < K) {
        if (!pair) {
            const double v = ac * t0 - br * p0;
            r2 = v * v;
        } else {
            const double re = ac * t0 - br * p0 + bi * p1;
            const double im = ac * t1 - br * p1 - bi * p0;
            r2 = fma(re, re, im * im);
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        r2 += __shfl_xor_sync(0xffffffffu, r2, o);
        x2 += __shfl_xor_sync(0xffffffffu, x2, o);
    }
    if (lane) return;
    const double est = sqrt(r2 / K);
    const double den = (fabs(ac) * norms[0] + hypot(br, bi) * norms[1]) * sqrt(x2);
    const bool bad = !(est <= 0.25 * bound * den);
    flags[c] = bad ? 1 : 0;
    if (pair) flags[c + 1] = bad ? 1 : 0;
    if (bad) atomicAdd(count, pair ? 2 : 1);
}

}  // namespace refine
}  // namespace xtg
