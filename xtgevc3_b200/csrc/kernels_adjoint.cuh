// Kernels of the adjoint (reverse-mode derivative) of the right eigenvectors.
//
// Forward (HOWMNY = 'A', right side), per eigenvector column c of eigenvalue index k, with
// the shifted operator W = ac S - b P of that column:
//   real:  x = [xh; 1; 0],     W[0:k, 0:k] xh = -W[0:k, k]
//   pair:  x = [xh; s; 0],     s = (-W[k, k+1], W[k, k]),  W[0:k, 0:k] xh = -W[0:k, k:k+2] s
//          (complex x stored as the column pair (Re, Im); b = b_re + i b_im)
// (src/dtgevc3.cpp:616-822 and 1281-1470 for the solves, 727-740 for the seed.)  Given
// G = dL/dX (for a pair, G's two columns are dL/dRe x and dL/dIm x), with
//   mu = W[0:k, 0:k]^-T conj(g[0:k])          (the transposed shifted solve)
// the derivative with the eigenvalues and the per-column scale factors held fixed is
//   dL/dW[i, j] = -mu_i x_j   (i < k, j < k + w),   dW = ac dS - b dP,
// so dL/dS = -sum_c ac_c Re(mu_c x_c^T) and dL/dP = sum_c Re(b_c mu_c x_c^T): two GEMMs
// of an n x m operand built from mu and the eigenvector matrix, masked to the entries the
// forward reads: the upper Hessenberg band i <= j + 1 of a real S (the upstream solves are
// Hessenberg solves, so L depends smoothly on every subdiagonal entry of S, zero or not),
// the upper triangle of P (triangular by contract: the upstream realified pair solves
// drop the imaginary part of P's subdiagonal) and of complex pencils.  For a pair,
// the seed adds  sigma Re(nu^T ds)  with nu = conj(g[k:k+2]) - W[0:k, k:k+2]^T mu and
// sigma the column's accumulated overflow scale factor (recovered from x[k:k+2]), and the
// column scale kappa = ac / beta of a pair depends on the pencil norm that sets it
// (src/dtgevc3.cpp:716-725: 1 / ((|ar| + |ai|) bnorm) or 1 / (|beta| anorm)), which
// contributes -L_c / norm times the sign pattern of the column that attains the norm.
// Real columns and complex-arithmetic columns (x_k = 1) are scale invariant.
//
// The transposed solves run as the right problem of the reversed transposed pencil
// (F S^T F, F P^T F): in that orientation column c lives in rows [n - k, n), so it enters
// at the bottom row block and ends (is truncated) at row n - k, the mirror image of the
// forward, where a column starts at its seed and runs to row 0.
#pragma once
#include "common.cuh"
#include "kernels_diag.cuh"
#include "kernels_misc.cuh"

#include <type_traits>

namespace xtg {

// R[n-1-i, c] = conj(G[i, c]) for i < k_c (0 elsewhere): the right-hand sides of the
// transposed solves in reversed orientation.  Real storage conjugates the Im column of a
// pair; complex storage conjugates every entry.
template <class E>
__global__ void adj_rhs_kernel(const E *G, int ldg, E *R, int ldr, int n, int m, const int *colk,
                               const uint8_t *kind)
{
    const int c = blockIdx.y;
    if (c >= m) return;
    const int k = colk[c];
    const bool neg = kind && kind[c] == kPairIm;
    for (int row = blockIdx.x * blockDim.x + threadIdx.x; row < n; row += gridDim.x * blockDim.x) {
        const int i = n - 1 - row;
        E v = i < k ? maybe_conj(G[(size_t)i + (size_t)c * ldg], 1) : E(0);
        if (neg) v = -v;
        R[(size_t)row + (size_t)c * ldr] = v;
    }
}

// out = in^T (conjugated when cj): 32 x 32 tiles through shared memory.
template <class E>
__global__ void transpose_kernel(const E *in, int ldi, E *out, int ldo, int rows, int cols, int cj)
{
    __shared__ E tile[32][33];
    const int r0 = blockIdx.x * 32, c0 = blockIdx.y * 32;
    const int tx = threadIdx.x, ty = threadIdx.y;  // 32 x 8
    for (int q = ty; q < 32; q += 8) {
        const int r = r0 + tx, c = c0 + q;
        if (r < rows && c < cols) tile[q][tx] = maybe_conj(in[(size_t)r + (size_t)c * ldi], cj);
    }
    __syncthreads();
    for (int q = ty; q < 32; q += 8) {
        const int c = c0 + tx, r = r0 + q;
        if (r < rows && c < cols) out[(size_t)c + (size_t)r * ldo] = tile[tx][q];
    }
}

// Shifted solves of one row block of the transposed problem (reversed orientation).  The
// same operator and block factorisation as diag_solve_real, but: no seed (every active
// column has a right-hand side from G), the column is truncated at its top row
// colk[c] (= n - k): rows of the block above it are left out of the solve and written as
// zero, and there are no overflow guards (a rescaled column would change the gradient).
template <class R>
__global__ void __launch_bounds__(256) diag_adjoint_real(DiagArgs<R> a)
{
    extern __shared__ __align__(16) unsigned char smem_diag[];
    __shared__ uint64_t s_sec;
    R *Ss = reinterpret_cast<R *>(smem_diag);
    R *Ps = Ss + kSmLd * kBlock;
    const int jnb = a.r1 - a.r0;
    load_block(a.S, a.lds, a.P, a.ldp, a.r0, jnb, 1, Ss, Ps);
    __syncthreads();
    pair_mask(Ss, jnb, &s_sec);
    __syncthreads();
    const uint64_t sec = s_sec;
    const int lane = threadIdx.x & 31;
    const int warps = (gridDim.x * blockDim.x) >> 5;
    for (int it = a.it0 + ((blockIdx.x * blockDim.x + threadIdx.x) >> 5); it < a.nitems; it += warps) {
        const int c = a.items[it];
        const uint8_t kd = a.kind[c];
        const int tl = max(a.colk[c] - a.r0, 0);
        const R ac = a.coef[4 * c + 0], br = a.coef[4 * c + 1], bi = a.coef[4 * c + 2], smin = a.coef[4 * c + 3];
        R *colr = a.X + (size_t)c * a.ldx;
        if (kd == kReal) {
            auto W = [&](int i, int j) -> R { return ac * Ss[i + j * kSmLd] - br * Ps[i + j * kSmLd]; };
            R r[2];
#pragma unroll
            for (int s = 0; s < 2; s++) {
                const int i = lane + 32 * s;
                r[s] = (i >= tl && i < jnb) ? colr[a.r0 + i] : R(0);
            }
            Factors<R> F;
            factor_rows(F, sec, jnb, lane, smin, W);
            back_substitute_loop(r, F, sec, jnb, lane, W, tl);
            R ys[2], yp[2];
#pragma unroll
            for (int s = 0; s < 2; s++) {
                const int i = lane + 32 * s;
                const R x = (i >= tl && i < jnb) ? r[s] : R(0);
                if (i < jnb) colr[a.r0 + i] = x;
                ys[s] = -ac * x;
                yp[s] = br * x;
            }
            write_y(a, a.Y + (size_t)c * a.ldy, jnb, false, lane, ys, yp);
        } else {
            using C = cplx<R>;
            R *coli = colr + a.ldx;
            const C b(br, bi);
            auto W = [&](int i, int j) -> C {
                const R s = Ss[i + j * kSmLd], p = Ps[i + j * kSmLd];
                return C(ac * s - br * p, -bi * p);
            };
            C r[2];
#pragma unroll
            for (int s = 0; s < 2; s++) {
                const int i = lane + 32 * s;
                r[s] = (i >= tl && i < jnb) ? C(colr[a.r0 + i], coli[a.r0 + i]) : C(0, 0);
            }
            Factors<C> F;
            factor_rows(F, sec, jnb, lane, smin, W);
            back_substitute_loop(r, F, sec, jnb, lane, W, tl);
            R ysr[2], ysi[2], ypr[2], ypi[2];
#pragma unroll
            for (int s = 0; s < 2; s++) {
                const int i = lane + 32 * s;
                const C x = (i >= tl && i < jnb) ? r[s] : C(0, 0);
                if (i < jnb) {
                    colr[a.r0 + i] = x.x;
                    coli[a.r0 + i] = x.y;
                }
                const C yp = b * x;
                ysr[s] = -ac * x.x;
                ysi[s] = -ac * x.y;
                ypr[s] = yp.x;
                ypi[s] = yp.y;
            }
            R *yre = a.Y + (size_t)c * a.ldy;
            write_y(a, yre, jnb, false, lane, ysr, ypr);
            write_y(a, yre + a.ldy, jnb, false, lane, ysi, ypi);
        }
    }
}

template <class R>
__global__ void __launch_bounds__(256) diag_adjoint_cplx(DiagArgs<R> a)
{
    using C = cplx<R>;
    extern __shared__ __align__(16) unsigned char smem_diag[];
    C *Ss = reinterpret_cast<C *>(smem_diag);
    C *Ps = Ss + kSmLd * kBlock;
    const int jnb = a.r1 - a.r0;
    load_block(reinterpret_cast<const C *>(a.S), a.lds, reinterpret_cast<const C *>(a.P), a.ldp, a.r0, jnb, 0, Ss,
               Ps);
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const int warps = (gridDim.x * blockDim.x) >> 5;
    C *X = reinterpret_cast<C *>(a.X);
    C *Y = reinterpret_cast<C *>(a.Y);
    for (int it = a.it0 + ((blockIdx.x * blockDim.x + threadIdx.x) >> 5); it < a.nitems; it += warps) {
        const int c = a.items[it];
        const int tl = max(a.colk[c] - a.r0, 0);
        const C ac(a.coef[6 * c + 0], a.coef[6 * c + 1]);
        const C bc(a.coef[6 * c + 2], a.coef[6 * c + 3]);
        const R smin = a.coef[6 * c + 4];
        C *col = X + (size_t)c * a.ldx;
        auto W = [&](int i, int j) -> C { return ac * Ss[i + j * kSmLd] - bc * Ps[i + j * kSmLd]; };
        C r[2];
#pragma unroll
        for (int s = 0; s < 2; s++) {
            const int i = lane + 32 * s;
            r[s] = (i >= tl && i < jnb) ? col[a.r0 + i] : C(0, 0);
        }
        Factors<C> F;
        factor_rows(F, 0ull, jnb, lane, smin, W);
        back_substitute(r, F, 0ull, jnb, lane, W, tl);
        C ys[2], yp[2];
#pragma unroll
        for (int s = 0; s < 2; s++) {
            const int i = lane + 32 * s;
            const C x = (i >= tl && i < jnb) ? r[s] : C(0, 0);
            if (i < jnb) col[a.r0 + i] = x;
            ys[s] = -(ac * x);
            yp[s] = bc * x;
        }
        write_y(a, Y + (size_t)c * a.ldy, jnb, false, lane, ys, yp);
    }
}

// Operands of the gradient GEMMs (original orientation):  lambda_c[i] = Rsol[n-1-i, c]
// for i < k_c, and  AS = -ac lambda, AP = b lambda  per column (real pairs combine the Re
// and Im columns as Re(. x^T) needs; complex storage is conjugated so that the GEMM with
// conj(X)^T gives the conjugate gradient dL/dRe + i dL/dIm).
template <class R>
__global__ void adj_operands_real(const R *Rs, int ldr, int n, int m, const int *colk, const uint8_t *kind,
                                  const R *coef, R *AS, R *AP, int lda)
{
    const int c = blockIdx.y;
    if (c >= m) return;
    const int k = colk[c];
    const uint8_t kd = kind[c];
    const R ac = coef[4 * c + 0], br = coef[4 * c + 1], bi = coef[4 * c + 2];
    const int cre = kd == kPairIm ? c - 1 : c;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        R s = R(0), p = R(0);
        if (i < k) {
            const size_t row = (size_t)(n - 1 - i);
            if (kd == kReal) {
                const R l = Rs[row + (size_t)c * ldr];
                s = -ac * l;
                p = br * l;
            } else {
                const R lr = Rs[row + (size_t)cre * ldr], li = Rs[row + (size_t)(cre + 1) * ldr];
                if (kd == kPairRe) {
                    s = -ac * lr;
                    p = br * lr - bi * li;
                } else {
                    s = ac * li;
                    p = -(br * li + bi * lr);
                }
            }
        }
        AS[(size_t)i + (size_t)c * lda] = s;
        AP[(size_t)i + (size_t)c * lda] = p;
    }
}

template <class R>
__global__ void adj_operands_cplx(const cplx<R> *Rs, int ldr, int n, int m, const int *colk, const R *coef,
                                  cplx<R> *AS, cplx<R> *AP, int lda)
{
    using C = cplx<R>;
    const int c = blockIdx.y;
    if (c >= m) return;
    const int k = colk[c];
    const C ac(coef[6 * c + 0], coef[6 * c + 1]), bc(coef[6 * c + 2], coef[6 * c + 3]);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        C s(0, 0), p(0, 0);
        if (i < k) {
            const C l = Rs[(size_t)(n - 1 - i) + (size_t)c * ldr];
            s = conjg(-(ac * l));
            p = conjg(bc * l);
        }
        AS[(size_t)i + (size_t)c * lda] = s;
        AP[(size_t)i + (size_t)c * lda] = p;
    }
}

// Seed and column-scale terms of the complex pairs (real arithmetic), one warp per pair.
// items: the pairs' Re columns.  eig: alphar, alphai, beta (device).  dnorm[0/1] collect
// dL/d anorm and dL/d bnorm.
template <class R>
__global__ void adj_pair_terms(const R *S, int lds, const R *P, int ldp, const R *X, int ldx, const R *G, int ldg,
                               const R *Rs, int ldr, int n, const int *pairs, int npairs, const R *coef,
                               const R *eig, const R *norms, R *dS, int ldds, R *dP, int lddp, R *dnorm)
{
    using C = cplx<R>;
    const int lane = threadIdx.x & 31;
    const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (w >= npairs) return;
    const int c = pairs[w];  // Re column; Im column c + 1; eigenvalue index k = c
    const int k = c;
    const R ac = coef[4 * c + 0], br = coef[4 * c + 1], bi = coef[4 * c + 2];
    const C b(br, bi);
    auto Wc = [&](int i, int j) -> C {
        const R s = S[(size_t)i + (size_t)j * lds], p = P[(size_t)i + (size_t)j * ldp];
        return C(ac * s - br * p, -bi * p);
    };
    // W[0:k, k+q]^T lambda and the pair's share of L
    C t0(0, 0), t1(0, 0);
    R lc = R(0);
    for (int i = lane; i < n; i += 32) {
        if (i < k) {
            const size_t row = (size_t)(n - 1 - i);
            const C l(Rs[row + (size_t)c * ldr], Rs[row + (size_t)(c + 1) * ldr]);
            t0 = t0 + Wc(i, k) * l;
            t1 = t1 + Wc(i, k + 1) * l;
        }
        lc += G[(size_t)i + (size_t)c * ldg] * X[(size_t)i + (size_t)c * ldx] +
              G[(size_t)i + (size_t)(c + 1) * ldg] * X[(size_t)i + (size_t)(c + 1) * ldx];
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        t0.x += __shfl_xor_sync(0xffffffffu, t0.x, o);
        t0.y += __shfl_xor_sync(0xffffffffu, t0.y, o);
        t1.x += __shfl_xor_sync(0xffffffffu, t1.x, o);
        t1.y += __shfl_xor_sync(0xffffffffu, t1.y, o);
        lc += __shfl_xor_sync(0xffffffffu, lc, o);
    }
    if (lane != 0) return;
    // nu = conj(g[k:k+2]) - W[0:k, k:k+2]^T lambda
    const C nu0 = C(G[(size_t)k + (size_t)c * ldg], -G[(size_t)k + (size_t)(c + 1) * ldg]) - t0;
    const C nu1 = C(G[(size_t)(k + 1) + (size_t)c * ldg], -G[(size_t)(k + 1) + (size_t)(c + 1) * ldg]) - t1;
    // sigma: |x[k:k+2]| / |unscaled seed (-W[k,k+1], W[k,k])|
    const C s0 = -Wc(k, k + 1), s1 = Wc(k, k);
    const R xk = X[(size_t)k + (size_t)c * ldx], yk = X[(size_t)k + (size_t)(c + 1) * ldx];
    const R xk1 = X[(size_t)(k + 1) + (size_t)c * ldx], yk1 = X[(size_t)(k + 1) + (size_t)(c + 1) * ldx];
    const R sn = sqrt(s0.x * s0.x + s0.y * s0.y + s1.x * s1.x + s1.y * s1.y);
    const R sigma = sn > R(0) ? sqrt(xk * xk + yk * yk + xk1 * xk1 + yk1 * yk1) / sn : R(1);
    // ds = (-dW[k, k+1], dW[k, k]),  dW = ac dS - b dP
    dS[(size_t)k + (size_t)(k + 1) * ldds] += -sigma * ac * nu0.x;
    dP[(size_t)k + (size_t)(k + 1) * lddp] += sigma * (nu0 * b).x;
    dS[(size_t)k + (size_t)k * ldds] += sigma * ac * nu1.x;
    dP[(size_t)k + (size_t)k * lddp] += -sigma * (nu1 * b).x;
    // column scale of the pair: kappa = 1 / ((|ar| + |ai|) bnorm) or 1 / (|beta| anorm)
    const R safemin = limits<R>::safemin;
    const R anorm = norms[0], bnorm = norms[1];
    const R ar = eig[k], ai = eig[n + k], be = eig[2 * n + k];
    if (fabs(be) <= safemin && (fabs(ar) + fabs(ai)) > safemin) return;  // infinite: fixed (0, 1)
    const R ascale = R(1) / fmax(anorm, safemin), bscale = R(1) / fmax(bnorm, safemin);
    const R a1 = (fabs(ar) + fabs(ai)) * ascale, b1 = fabs(be) * bscale;
    if (a1 >= b1 && a1 > safemin && bnorm > safemin) atomicAdd(dnorm + 1, -lc / bnorm);
    else if (b1 > a1 && b1 > safemin && anorm > safemin) atomicAdd(dnorm + 0, -lc / anorm);
}

// norms[0/1] = max column sum of |S| / |P| (rows <= col + extra), jmax[0/1] = the first
// column attaining it.  One block.
template <class R>
__global__ void colargmax_kernel(const R *sums, int n, R *norms, int *jmax)
{
    __shared__ R sv[2][32];
    __shared__ int si[2][32];
    R v[2] = {R(-1), R(-1)};
    int ix[2] = {0, 0};
    for (int i = threadIdx.x; i < n; i += blockDim.x)
        for (int q = 0; q < 2; q++)
            if (sums[q * n + i] > v[q]) {
                v[q] = sums[q * n + i];
                ix[q] = i;
            }
    for (int q = 0; q < 2; q++) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const R ov = __shfl_xor_sync(0xffffffffu, v[q], o);
            const int oi = __shfl_xor_sync(0xffffffffu, ix[q], o);
            if (ov > v[q] || (ov == v[q] && oi < ix[q])) {
                v[q] = ov;
                ix[q] = oi;
            }
        }
        if ((threadIdx.x & 31) == 0) {
            sv[q][threadIdx.x >> 5] = v[q];
            si[q][threadIdx.x >> 5] = ix[q];
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int q = 0; q < 2; q++) {
            R bv = sv[q][0];
            int bix = si[q][0];
            for (int w = 1; w < (int)(blockDim.x >> 5); w++)
                if (sv[q][w] > bv || (sv[q][w] == bv && si[q][w] < bix)) {
                    bv = sv[q][w];
                    bix = si[q][w];
                }
            norms[q] = fmax(bv, R(0));
            jmax[q] = bix;
        }
    }
}

template <class R> __device__ __forceinline__ R sgn(R v) { return v > R(0) ? R(1) : (v < R(0) ? R(-1) : R(0)); }

// Mask the gradients to the entries the forward reads (real S: i <= j + 1; P and complex
// pencils: i <= j)
// and add the norm terms (real only: d anorm / dS[i, jS] = sign(S[i, jS]) for
// i <= jS + 1, likewise for P).
template <class E, class R>
__global__ void adj_finalize_kernel(E *dS, int ldds, E *dP, int lddp, const E *S, int lds, const E *P, int ldp,
                                    int n, const R *dnorm, const int *jmax)
{
    const int j = blockIdx.y;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        E &gs = dS[(size_t)i + (size_t)j * ldds];
        E &gp = dP[(size_t)i + (size_t)j * lddp];
        if constexpr (std::is_same<E, R>::value) {
            if (i > j) gp = R(0);
            if (i > j + 1) {
                gs = R(0);
                continue;
            }
            if (j == jmax[0] && i <= j + 1) gs = gs + dnorm[0] * sgn(S[(size_t)i + (size_t)j * lds]);
            if (j == jmax[1] && i <= j + 1) gp = gp + dnorm[1] * sgn(P[(size_t)i + (size_t)j * ldp]);
        } else {
            if (i > j) {
                gs = E(0);
                gp = E(0);
            }
        }
    }
}

}  // namespace xtg
