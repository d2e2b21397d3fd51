// Diagonal-block shifted solves of the right-looking substitution.
//
// For one row block I = [r0, r1) (r1 - r0 <= kBlock) and every active eigenvector
// column c (eigenvalue index k_c >= r0), solve
//        (ac_c * S[I,I] - b_c * P[I,I]) x = rhs_c
// where rhs_c is the accumulated right-hand side held in X[I, c] (k_c >= r1), or, when
// the eigenvalue lies inside the block (r0 <= k_c < r1, the "diagonal" case), the seed
// x_k = 1 (real) / the 2x2 closed-form null vector (complex pair) with
// rhs = -W[0:kl, seed rows] * seed.  This is the per-eigenvalue local solve of the
// upstream driver (dlalsr, src/dtgevc3.cpp:616-822; zlalsr, src/ztgevc3.cpp:116-211),
// done for all columns of the matrix at once instead of one 32-column panel at a time.
//
// Layout: one warp owns one eigenvector (a real column, a (Re, Im) column pair, or a
// complex column); lane l holds rows l and l + 32 of the block.  S[I,I], P[I,I] live in
// shared memory.  The solve is column-oriented block back substitution: after x_j is
// known it is broadcast by shuffle and every lane updates its rows.  2x2 diagonal blocks
// of S (S[j, j-1] != 0) are solved as 2x2 systems with partial pivoting.
//
// Overflow guards, per column (the upstream code rescales a whole 32-column panel):
//   * before the solve: if max|rhs| > bignum/10, scale the column by (bignum/10)/max
//     (src/dtgevc3.cpp:682-698);
//   * before the update: if max(|ac x|, |b x|) > bignum/jnb, scale the column
//     (src/dtgevc3.cpp:1404-1426, with the panel width replaced by the block height).
// Scaling a column means scaling every stored row of it: the accumulated rows above the
// block, the rows solved in earlier blocks and the current block.
//
// Output: X[I, c] (solution), and the stacked update operand
//   Y[0:bpad, c] = -ac * x,  Y[bpad:2*bpad, c] = b * x   (zero padded)
// consumed by the update GEMM  X[0:r0, c] += S[0:r0, I] Y[0:bpad] + P[0:r0, I] Y[bpad:].
#pragma once
#include "common.cuh"

namespace xtg {

constexpr int kSmLd = kBlock + 1;  // shared-memory leading dimension of the S/P block

template <class T>
__device__ __forceinline__ T shfl(T v, int src) { return __shfl_sync(0xffffffffu, v, src); }

template <class R>
__device__ __forceinline__ R warp_max(R v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// Row `row` of the block lives in slot row >> 5 of lane row & 31.  Selects instead of
// r[row >> 5] keep the two slots in registers.
template <class T>
__device__ __forceinline__ T row_of(const T (&r)[2], int row) { return (row >> 5) ? r[1] : r[0]; }
template <class T>
__device__ __forceinline__ void set_row(T (&r)[2], int row, int lane, T v)
{
    if (lane == (row & 31)) {
        if (row >> 5) r[1] = v;
        else r[0] = v;
    }
}

template <class R>
__device__ __forceinline__ R floor_pivot(R w, R smin)
{
    return fabs(w) < smin ? (w < R(0) ? -smin : smin) : w;
}

template <class R>
__device__ __forceinline__ cplx<R> floor_pivot(cplx<R> w, R smin)
{
    return l1abs(w) < smin ? cplx<R>(smin, R(0)) : w;
}

template <class R>
struct DiagArgs {
    const R *S, *P;  // pencil in the orientation being solved (right problem)
    int lds, ldp, n;
    int r0, r1, bpad;
    int c0, m;
    const int *colk;         // eigenvalue index (first member of a pair) per column
    const uint8_t *kind;     // kReal / kPairRe / kPairIm (real arithmetic only)
    const R *coef;           // 4 per column: ac, b_re, b_im, smin  (complex: 6: ac, b, smin, 0)
    R *X;                    // n x m computed eigenvectors (complex: interleaved)
    int ldx;
    R *Y;                    // 2*bpad x m update operand
    int ldy;
    R thr_rhs, thr_upd;
    int left_seed;           // 2x2 seed of the left problem (see seed_pair)
};

// Multiply rows [a, b) of one column by s (warp-cooperative).  Used on the rows of a
// column outside the current block when an overflow guard fires.
template <class R>
__device__ __forceinline__ void scale_rows(R *col, int a, int b, R s, int lane)
{
    for (int i = a + lane; i < b; i += 32) col[i] *= s;
}

// ------------------------------------------------------------------------------------
// Real arithmetic (s/d): real columns and (Re, Im) column pairs
// ------------------------------------------------------------------------------------
template <class R>
__global__ void __launch_bounds__(256) diag_solve_real(DiagArgs<R> a)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    R *Ss = reinterpret_cast<R *>(smem_raw);
    R *Ps = Ss + kSmLd * kBlock;
    const int jnb = a.r1 - a.r0;
    for (int t = threadIdx.x; t < jnb * jnb; t += blockDim.x) {
        int i = t % jnb, j = t / jnb;
        bool keep = i <= j + 1;  // upper triangle plus the subdiagonal
        size_t gs = (size_t)(a.r0 + i) + (size_t)(a.r0 + j) * a.lds;
        size_t gp = (size_t)(a.r0 + i) + (size_t)(a.r0 + j) * a.ldp;
        Ss[i + j * kSmLd] = keep ? a.S[gs] : R(0);
        Ps[i + j * kSmLd] = keep ? a.P[gp] : R(0);
    }
    __syncthreads();

    const int lane = threadIdx.x & 31;
    const int warps = (gridDim.x * blockDim.x) >> 5;
    for (int c = a.c0 + ((blockIdx.x * blockDim.x + threadIdx.x) >> 5); c < a.m; c += warps) {
        const uint8_t kd = a.kind[c];
        if (kd == kPairIm) continue;
        const int k = a.colk[c];
        const int kl = k - a.r0;
        const bool diag = k < a.r1;
        const R ac = a.coef[4 * c + 0], br = a.coef[4 * c + 1], bi = a.coef[4 * c + 2], smin = a.coef[4 * c + 3];
        R *colr = a.X + (size_t)c * a.ldx;
        const int nrows = diag ? kl : jnb;
        if (kd == kReal) {
            const int top = k;
            R r[2];
            R seed = diag ? R(1) : R(0);
#pragma unroll
            for (int s = 0; s < 2; s++) {
                int i = lane + 32 * s;
                R v = R(0);
                if (i < nrows)
                    v = diag ? -(ac * Ss[i + kl * kSmLd] - br * Ps[i + kl * kSmLd]) : colr[a.r0 + i];
                r[s] = v;
            }
            if (nrows > 0) {
                R mx = warp_max(fmax(fabs(r[0]), fabs(r[1])));
                if (mx > a.thr_rhs) {
                    R sc = a.thr_rhs / mx;
                    r[0] *= sc; r[1] *= sc; seed *= sc;
                    if (!diag) { scale_rows(colr, 0, a.r0, sc, lane); scale_rows(colr, a.r1, top + 1, sc, lane); }
                }
            }
            // block back substitution
            int j = nrows - 1;
            while (j >= 0) {
                const bool two = j >= 1 && Ss[j + (j - 1) * kSmLd] != R(0);
                if (!two) {
                    R w = floor_pivot(ac * Ss[j + j * kSmLd] - br * Ps[j + j * kSmLd], smin);
                    R rj = shfl(row_of(r, j), j & 31);
                    R xj = rj / w;
                    set_row(r, j, lane, xj);
#pragma unroll
                    for (int s = 0; s < 2; s++) {
                        int i = lane + 32 * s;
                        if (i < j) r[s] -= (ac * Ss[i + j * kSmLd] - br * Ps[i + j * kSmLd]) * xj;
                    }
                    j -= 1;
                } else {
                    const int p = j - 1, q = j;
                    R w11 = ac * Ss[p + p * kSmLd] - br * Ps[p + p * kSmLd];
                    R w12 = ac * Ss[p + q * kSmLd] - br * Ps[p + q * kSmLd];
                    R w21 = ac * Ss[q + p * kSmLd] - br * Ps[q + p * kSmLd];
                    R w22 = ac * Ss[q + q * kSmLd] - br * Ps[q + q * kSmLd];
                    R rp = shfl(row_of(r, p), p & 31), rq = shfl(row_of(r, q), q & 31);
                    if (fabs(w21) > fabs(w11)) {  // row interchange (partial pivoting on column p)
                        R t;
                        t = w11; w11 = w21; w21 = t;
                        t = w12; w12 = w22; w22 = t;
                        t = rp; rp = rq; rq = t;
                    }
                    w11 = floor_pivot(w11, smin);
                    R mult = w21 / w11;
                    R u22 = floor_pivot(w22 - mult * w12, smin);
                    R xq = (rq - mult * rp) / u22;
                    R xp = (rp - w12 * xq) / w11;
                    set_row(r, p, lane, xp);
                    set_row(r, q, lane, xq);
#pragma unroll
                    for (int s = 0; s < 2; s++) {
                        int i = lane + 32 * s;
                        if (i < p)
                            r[s] -= (ac * Ss[i + p * kSmLd] - br * Ps[i + p * kSmLd]) * xp +
                                    (ac * Ss[i + q * kSmLd] - br * Ps[i + q * kSmLd]) * xq;
                    }
                    j -= 2;
                }
            }
            // assemble the block column (solution rows, seed, zeros below the seed)
            R x[2];
#pragma unroll
            for (int s = 0; s < 2; s++) {
                int i = lane + 32 * s;
                x[s] = i < nrows ? r[s] : (diag && i == kl ? seed : R(0));
            }
            R mx = warp_max(fmax(fmax(fabs(ac * x[0]), fabs(br * x[0])), fmax(fabs(ac * x[1]), fabs(br * x[1]))));
            if (mx > a.thr_upd) {
                R sc = a.thr_upd / mx;
                x[0] *= sc; x[1] *= sc;
                if (!diag) { scale_rows(colr, 0, a.r0, sc, lane); scale_rows(colr, a.r1, top + 1, sc, lane); }
            }
            R *ycol = a.Y + (size_t)c * a.ldy;
#pragma unroll
            for (int s = 0; s < 2; s++) {
                int i = lane + 32 * s;
                if (i < jnb) colr[a.r0 + i] = x[s];
                if (i < a.bpad) {
                    bool in = i < jnb;
                    ycol[i] = in ? -ac * x[s] : R(0);
                    ycol[a.bpad + i] = in ? br * x[s] : R(0);
                }
            }
        } else {
            // complex pair stored as (Re, Im) in columns (c, c+1); shift b = br + i*bi
            using C = cplx<R>;
            R *coli = colr + a.ldx;
            const int top = k + 1;
            const C b(br, bi);
            auto W = [&](int i, int j) -> C {
                R s = Ss[i + j * kSmLd], p = Ps[i + j * kSmLd];
                return C(ac * s - br * p, -bi * p);
            };
            C seed0(0, 0), seed1(0, 0);
            if (diag) {
                if (!a.left_seed) {  // (x_k, x_k+1) = (-w12, w11), src/dtgevc3.cpp:727-740
                    seed0 = -W(kl, kl + 1);
                    seed1 = W(kl, kl);
                } else {             // (x_k, x_k+1) = (w22, -w21): the left-problem seed, mirrored
                    seed0 = W(kl + 1, kl + 1);
                    seed1 = -W(kl + 1, kl);
                }
            }
            C r[2];
#pragma unroll
            for (int s = 0; s < 2; s++) {
                int i = lane + 32 * s;
                C v(0, 0);
                if (i < nrows) {
                    if (diag) v = -(W(i, kl) * seed0 + W(i, kl + 1) * seed1);
                    else v = C(colr[a.r0 + i], coli[a.r0 + i]);
                }
                r[s] = v;
            }
            if (nrows > 0) {
                R mx = warp_max(fmax(fmax(fabs(r[0].x), fabs(r[0].y)), fmax(fabs(r[1].x), fabs(r[1].y))));
                if (mx > a.thr_rhs) {
                    R sc = a.thr_rhs / mx;
                    r[0] = sc * r[0]; r[1] = sc * r[1]; seed0 = sc * seed0; seed1 = sc * seed1;
                    if (!diag) {
                        scale_rows(colr, 0, a.r0, sc, lane); scale_rows(colr, a.r1, top + 1, sc, lane);
                        scale_rows(coli, 0, a.r0, sc, lane); scale_rows(coli, a.r1, top + 1, sc, lane);
                    }
                }
            }
            int j = nrows - 1;
            while (j >= 0) {
                const bool two = j >= 1 && Ss[j + (j - 1) * kSmLd] != R(0);
                if (!two) {
                    C w = floor_pivot(W(j, j), smin);
                    C rs = row_of(r, j);
                    C rj(shfl(rs.x, j & 31), shfl(rs.y, j & 31));
                    C xj = cdiv(rj, w);
                    set_row(r, j, lane, xj);
#pragma unroll
                    for (int s = 0; s < 2; s++) {
                        int i = lane + 32 * s;
                        if (i < j) r[s] = r[s] - W(i, j) * xj;
                    }
                    j -= 1;
                } else {
                    const int p = j - 1, q = j;
                    C w11 = W(p, p), w12 = W(p, q), w21 = W(q, p), w22 = W(q, q);
                    C sp_ = row_of(r, p), sq_ = row_of(r, q);
                    C rp(shfl(sp_.x, p & 31), shfl(sp_.y, p & 31));
                    C rq(shfl(sq_.x, q & 31), shfl(sq_.y, q & 31));
                    if (l1abs(w21) > l1abs(w11)) {
                        C t;
                        t = w11; w11 = w21; w21 = t;
                        t = w12; w12 = w22; w22 = t;
                        t = rp; rp = rq; rq = t;
                    }
                    w11 = floor_pivot(w11, smin);
                    C mult = cdiv(w21, w11);
                    C u22 = floor_pivot(w22 - mult * w12, smin);
                    C xq = cdiv(rq - mult * rp, u22);
                    C xp = cdiv(rp - w12 * xq, w11);
                    set_row(r, p, lane, xp);
                    set_row(r, q, lane, xq);
#pragma unroll
                    for (int s = 0; s < 2; s++) {
                        int i = lane + 32 * s;
                        if (i < p) r[s] = r[s] - (W(i, p) * xp + W(i, q) * xq);
                    }
                    j -= 2;
                }
            }
            C x[2];
#pragma unroll
            for (int s = 0; s < 2; s++) {
                int i = lane + 32 * s;
                x[s] = i < nrows ? r[s] : (diag && i == kl ? seed0 : (diag && i == kl + 1 ? seed1 : C(0, 0)));
            }
            R mx = R(0);
#pragma unroll
            for (int s = 0; s < 2; s++) {
                C ys = ac * x[s], yp = b * x[s];
                mx = fmax(mx, fmax(fmax(fabs(ys.x), fabs(ys.y)), fmax(fabs(yp.x), fabs(yp.y))));
            }
            mx = warp_max(mx);
            if (mx > a.thr_upd) {
                R sc = a.thr_upd / mx;
                x[0] = sc * x[0]; x[1] = sc * x[1];
                if (!diag) {
                    scale_rows(colr, 0, a.r0, sc, lane); scale_rows(colr, a.r1, top + 1, sc, lane);
                    scale_rows(coli, 0, a.r0, sc, lane); scale_rows(coli, a.r1, top + 1, sc, lane);
                }
            }
            R *yre = a.Y + (size_t)c * a.ldy, *yim = yre + a.ldy;
#pragma unroll
            for (int s = 0; s < 2; s++) {
                int i = lane + 32 * s;
                if (i < jnb) { colr[a.r0 + i] = x[s].x; coli[a.r0 + i] = x[s].y; }
                if (i < a.bpad) {
                    bool in = i < jnb;
                    C yp = b * x[s];
                    yre[i] = in ? -ac * x[s].x : R(0);
                    yim[i] = in ? -ac * x[s].y : R(0);
                    yre[a.bpad + i] = in ? yp.x : R(0);
                    yim[a.bpad + i] = in ? yp.y : R(0);
                }
            }
        }
    }
}

// ------------------------------------------------------------------------------------
// Complex arithmetic (c/z): S triangular, one complex column per eigenvalue
// ------------------------------------------------------------------------------------
template <class R>
__global__ void __launch_bounds__(256) diag_solve_cplx(DiagArgs<R> a)
{
    using C = cplx<R>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C *Ss = reinterpret_cast<C *>(smem_raw);
    C *Ps = Ss + kSmLd * kBlock;
    const C *S = reinterpret_cast<const C *>(a.S);
    const C *P = reinterpret_cast<const C *>(a.P);
    const int jnb = a.r1 - a.r0;
    for (int t = threadIdx.x; t < jnb * jnb; t += blockDim.x) {
        int i = t % jnb, j = t / jnb;
        bool keep = i <= j;
        size_t gs = (size_t)(a.r0 + i) + (size_t)(a.r0 + j) * a.lds;
        size_t gp = (size_t)(a.r0 + i) + (size_t)(a.r0 + j) * a.ldp;
        Ss[i + j * kSmLd] = keep ? S[gs] : C(0, 0);
        Ps[i + j * kSmLd] = keep ? P[gp] : C(0, 0);
    }
    __syncthreads();

    const int lane = threadIdx.x & 31;
    const int warps = (gridDim.x * blockDim.x) >> 5;
    C *X = reinterpret_cast<C *>(a.X);
    C *Y = reinterpret_cast<C *>(a.Y);
    for (int c = a.c0 + ((blockIdx.x * blockDim.x + threadIdx.x) >> 5); c < a.m; c += warps) {
        const int k = a.colk[c];
        const int kl = k - a.r0;
        const bool diag = k < a.r1;
        const C ac(a.coef[6 * c + 0], a.coef[6 * c + 1]);
        const C bc(a.coef[6 * c + 2], a.coef[6 * c + 3]);
        const R smin = a.coef[6 * c + 4];
        C *col = X + (size_t)c * a.ldx;
        const int nrows = diag ? kl : jnb;
        const int top = k;
        auto W = [&](int i, int j) -> C { return ac * Ss[i + j * kSmLd] - bc * Ps[i + j * kSmLd]; };
        C seed = diag ? C(1, 0) : C(0, 0);
        C r[2];
#pragma unroll
        for (int s = 0; s < 2; s++) {
            int i = lane + 32 * s;
            C v(0, 0);
            if (i < nrows) v = diag ? -W(i, kl) : col[a.r0 + i];
            r[s] = v;
        }
        if (nrows > 0) {
            R mx = warp_max(fmax(l1abs(r[0]), l1abs(r[1])));
            if (mx > a.thr_rhs) {
                R sc = a.thr_rhs / mx;
                r[0] = sc * r[0]; r[1] = sc * r[1]; seed = sc * seed;
                if (!diag) {
                    for (int i = lane; i < a.r0; i += 32) col[i] = sc * col[i];
                    for (int i = a.r1 + lane; i <= top; i += 32) col[i] = sc * col[i];
                }
            }
        }
        for (int j = nrows - 1; j >= 0; j--) {
            C w = floor_pivot(W(j, j), smin);
            C rs = row_of(r, j);
            C rj(shfl(rs.x, j & 31), shfl(rs.y, j & 31));
            C xj = cdiv(rj, w);
            set_row(r, j, lane, xj);
#pragma unroll
            for (int s = 0; s < 2; s++) {
                int i = lane + 32 * s;
                if (i < j) r[s] = r[s] - W(i, j) * xj;
            }
        }
        C x[2];
#pragma unroll
        for (int s = 0; s < 2; s++) {
            int i = lane + 32 * s;
            x[s] = i < nrows ? r[s] : (diag && i == kl ? seed : C(0, 0));
        }
        R mx = R(0);
#pragma unroll
        for (int s = 0; s < 2; s++) mx = fmax(mx, fmax(l1abs(ac * x[s]), l1abs(bc * x[s])));
        mx = warp_max(mx);
        if (mx > a.thr_upd) {
            R sc = a.thr_upd / mx;
            x[0] = sc * x[0]; x[1] = sc * x[1];
            if (!diag) {
                for (int i = lane; i < a.r0; i += 32) col[i] = sc * col[i];
                for (int i = a.r1 + lane; i <= top; i += 32) col[i] = sc * col[i];
            }
        }
        C *ycol = Y + (size_t)c * a.ldy;
#pragma unroll
        for (int s = 0; s < 2; s++) {
            int i = lane + 32 * s;
            if (i < jnb) col[a.r0 + i] = x[s];
            if (i < a.bpad) {
                bool in = i < jnb;
                ycol[i] = in ? -(ac * x[s]) : C(0, 0);
                ycol[a.bpad + i] = in ? bc * x[s] : C(0, 0);
            }
        }
    }
}

}  // namespace xtg
