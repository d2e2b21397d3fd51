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
// shared memory.  Per eigenvector the lanes first factor, in parallel, every diagonal
// block of W = ac S - b P: the reciprocal of each 1x1 pivot and the partially pivoted LU
// of each 2x2 block (S[j, j-1] != 0; rows paired greedily from the bottom of the block).
// The solve is then column-oriented block back substitution: the lane owning a block's
// rows computes its solution, broadcasts it by shuffle, and every lane updates its rows.
// An exactly zero (or subnormal) pivot is replaced by the column's smin =
// max(eps (|ac| anorm + |b| bnorm), safemin), LAPACK xTGEVC's perturbation, so repeated
// infinite eigenvalues give finite vectors; the upstream code divides by zero there.
//
// Overflow guards, per column (the upstream code rescales a whole 32-column panel):
//   * before the solve: if max|rhs| > bignum/10, scale the column by (bignum/10)/max
//     (src/dtgevc3.cpp:682-698);
//   * before the update: if max(|ac x|, |b x|) > bignum/jnb, scale the column
//     (src/dtgevc3.cpp:1404-1426, with the panel width replaced by the block height).
// Scaling a column means scaling every stored row of it: the accumulated rows above the
// block, the rows solved in earlier blocks and the current block, and the update-operand
// rows of the lower blocks of the same group (or pair), which the group's trailing GEMM has
// not consumed yet.  A third
// check, inside the block once its rows at and above kMidRow are solved, keeps at most 32
// rows between checks, as upstream's 32-row local solves do.
//
// Output: X[I, c] (solution), and this block's rows of the stacked update operand
//   Y[ys_off + i, c] = -ac * x_i,  Y[ys_off + yhalf + i, c] = b * x_i   (zero padded)
// consumed by the update GEMMs  X[rows above, c] += S[rows above, I] (-ac x) + P[..] (b x).
#pragma once
#include <type_traits>
#include "common.cuh"

namespace xtg {

constexpr int kSmLd = kBlock + 1;  // shared-memory leading dimension of the S/P block

template <class T>
__device__ __forceinline__ T shfl(T v, int src) { return __shfl_sync(0xffffffffu, v, src); }
template <class R>
__device__ __forceinline__ cplx<R> shfl(cplx<R> v, int src)
{
    return cplx<R>(__shfl_sync(0xffffffffu, v.x, src), __shfl_sync(0xffffffffu, v.y, src));
}

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

__device__ __forceinline__ double rcp(double v) { return __drcp_rn(v); }
__device__ __forceinline__ float rcp(float v) { return __frcp_rn(v); }
// 1 / v by Smith's method (R. L. Smith, Comm. ACM 5(8), 1962), its two real divisions done
// as reciprocals: with |a| >= |b| the larger and smaller part of v, r = b / a and
// d = a + r b, 1 / (a + i b) = (1 - i r) / d and 1 / (b + i a) = (r - i) / d.  v != 0.
template <class R>
__device__ __forceinline__ cplx<R> rcp(cplx<R> v)
{
    const bool re_big = fabs(v.x) >= fabs(v.y);
    const R a = re_big ? v.x : v.y, b = re_big ? v.y : v.x;
    const R r = b * rcp(a);
    const R id = rcp(a + r * b);
    return re_big ? cplx<R>(id, -r * id) : cplx<R>(r * id, -id);
}

template <class R>
__device__ __forceinline__ R mag(R v) { return fabs(v); }
template <class R>
__device__ __forceinline__ R mag(cplx<R> v) { return l1abs(v); }

// A pivot that is zero (or subnormal) is replaced by smin; every other pivot is used as
// is, like the upstream solves, which divide by whatever pivot they meet.  Graded pencils
// legitimately have pivots far below eps * ||W||, so only exact singularity is perturbed.
template <class R>
__device__ __forceinline__ R floor_pivot(R w, R smin)
{
    return fabs(w) < limits<R>::safemin ? (w < R(0) ? -smin : smin) : w;
}

template <class R>
__device__ __forceinline__ cplx<R> floor_pivot(cplx<R> w, R smin)
{
    return l1abs(w) < limits<R>::safemin ? cplx<R>(smin, R(0)) : w;
}

template <class R>
struct DiagArgs {
    const R *S, *P;  // pencil in the orientation being solved (right problem)
    int lds, ldp, n;
    int r0, r1;
    // update operand layout: this block's -ac x rows start at Y row ys_off, its b x rows at
    // ys_off + yhalf; ypad (>= r1 - r0) rows are written, zeros past the block.  For a
    // column whose eigenvalue lies in this block, rows [zl_off, zl_off + zl_len) of both
    // halves (a lower block of the same update, where such a column is zero) are zeroed;
    // for the other columns a guard rescales them with the column (scale_lower_y).
    int ys_off, yhalf, ypad, zl_off, zl_len;
    const int *items;        // columns that start an eigenvector (a pair's Re column), ascending
    int it0, nitems;         // items [it0, nitems) are active in this block
    const int *colk;         // eigenvalue index (first member of a pair) per column
    const uint8_t *kind;     // kReal / kPairRe / kPairIm (real arithmetic only)
    const R *coef;           // 4 per column: ac, b_re, b_im, smin  (complex: 6: ac, b, smin, 0)
    R *X;                    // n x m computed eigenvectors (complex: interleaved)
    int ldx;
    R *Y;                    // 2 yhalf x m update operand (-ac x rows, then b x rows)
    int ldy;
    R thr_rhs, thr_upd;
    int left_seed;           // 2x2 seed of the left problem (see the pair branch)
    // Deferred guard scaling (nullable).  When set, a guard rescales the rows of a column
    // above the block only down to row safe_lo and multiplies pending[c] by the factor; the
    // caller applies pending to rows [0, safe_lo) once no other kernel writes them.
    R *pending;
    int safe_lo;
};

// Multiply rows [a, b) of one column by s (warp-cooperative).  Used on the rows of a
// column outside the current block when an overflow guard fires.
template <class E, class R>
__device__ __forceinline__ void scale_rows(E *col, int a, int b, R s, int lane)
{
    for (int i = a + lane; i < b; i += 32) col[i] = s * col[i];
}

// Guard rescaling of the rows above the block [0, r0) of column c: all of them at once,
// or (deferred mode) rows [safe_lo, r0) now and the rest through pending[c].
template <class E, class R>
__device__ __forceinline__ void scale_above(const DiagArgs<R> &a, E *col, int c, R s, int lane)
{
    if (!a.pending) {
        scale_rows(col, 0, a.r0, s, lane);
        return;
    }
    scale_rows(col, a.safe_lo < a.r0 ? a.safe_lo : a.r0, a.r0, s, lane);
    if (lane == 0) a.pending[c] *= s;
}

// A block above others in a group (or pair): the lower blocks' rows of the update operand
// (rows [zl_off, zl_off + zl_len) of both halves, written by their solves) are consumed by
// the group's trailing update together with this block's rows.  A guard that rescales a
// column here rescales those rows too, so that all the blocks' operands carry the same scale
// (upstream applies each block's update before the next solve and has no such operand).
template <class E, class R>
__device__ __forceinline__ void scale_lower_y(const DiagArgs<R> &a, E *ycol, R s, int lane)
{
    for (int i = lane; i < a.zl_len; i += 32) {
        ycol[a.zl_off + i] = s * ycol[a.zl_off + i];
        ycol[a.zl_off + a.yhalf + i] = s * ycol[a.zl_off + a.yhalf + i];
    }
}

// Write this block's rows of one update-operand column: ys = -ac x, yp = b x for rows
// i < jnb, zeros up to ypad, and the lower-block zeros of a diagonal-case column.
template <class E, class R>
__device__ __forceinline__ void write_y(const DiagArgs<R> &a, E *ycol, int jnb, bool diag, int lane, const E (&ys)[2],
                                       const E (&yp)[2])
{
#pragma unroll
    for (int s = 0; s < 2; s++) {
        const int i = lane + 32 * s;
        if (i < a.ypad) {
            const bool in = i < jnb;
            ycol[a.ys_off + i] = in ? ys[s] : E(0);
            ycol[a.ys_off + a.yhalf + i] = in ? yp[s] : E(0);
        }
    }
    for (int i = 64 + lane; i < a.ypad; i += 32) {  // padding past a full block (jnb <= 64)
        ycol[a.ys_off + i] = E(0);
        ycol[a.ys_off + a.yhalf + i] = E(0);
    }
    if (diag)
        for (int i = lane; i < a.zl_len; i += 32) {
            ycol[a.zl_off + i] = E(0);
            ycol[a.zl_off + a.yhalf + i] = E(0);
        }
}

template <class E, int kBatch = 8>
__device__ __forceinline__ void load_block(const E *S, int lds, const E *P, int ldp, int r0, int jnb, int sub,
                                           E *Ss, E *Ps)
{
    // kBatch elements of each matrix per thread are loaded before any is stored, so that the
    // block's loads are in flight together instead of one memory round trip per element
    // (kBatch x blockDim = 4096 covers a full block in one pass).  The whole square is read
    // (it lies inside the matrix); the part below the upper triangle (plus the subdiagonal
    // for real S) is stored as zeros.
    const int tot = jnb * jnb;
    for (int t0 = threadIdx.x; t0 < tot; t0 += kBatch * blockDim.x) {
        E vs[kBatch], vp[kBatch];
#pragma unroll
        for (int u = 0; u < kBatch; u++) {
            const int t = t0 + u * blockDim.x;
            if (t < tot) {
                const int i = t % jnb, j = t / jnb;
                vs[u] = S[(size_t)(r0 + i) + (size_t)(r0 + j) * lds];
                vp[u] = P[(size_t)(r0 + i) + (size_t)(r0 + j) * ldp];
            }
        }
#pragma unroll
        for (int u = 0; u < kBatch; u++) {
            const int t = t0 + u * blockDim.x;
            if (t < tot) {
                const int i = t % jnb, j = t / jnb;
                const bool keep = i <= j + sub;
                Ss[i + j * kSmLd] = keep ? vs[u] : E(0);
                Ps[i + j * kSmLd] = keep ? vp[u] : E(0);
            }
        }
    }
}

// Factors of the diagonal blocks of W for the rows a lane owns: inv1 = 1 / w_ii for every
// 1x1 row (rows of a 2x2 block keep 0); for the second row i of a 2x2 block (i-1, i): the LU with partial pivoting on
// column i-1:  swap rows if |w_i,i-1| > |w_i-1,i-1|, then (a b; c d) -> a^-1, b, m = c/a,
// (d - m b)^-1.
template <class E>
struct Factors {
    E inv1[2], fa[2], fb[2], fm[2], fu[2];
    bool sw[2];
};

template <class E, class R, class WF>
__device__ __forceinline__ void factor_rows(Factors<E> &F, uint64_t sec, int nrows, int lane, R smin, WF W)
{
#pragma unroll
    for (int s = 0; s < 2; s++) {
        const int i = lane + 32 * s;
        F.inv1[s] = E(0);
        F.fa[s] = F.fb[s] = F.fm[s] = F.fu[s] = E(0);
        F.sw[s] = false;
        if (i < nrows) {
            // rows of a 2x2 block are solved with its LU; inv1 serves 1x1 rows only
            const bool in2 = ((sec >> i) & 1ull) || (i + 1 < nrows && ((sec >> (i + 1)) & 1ull));
            if (!in2) F.inv1[s] = rcp(floor_pivot(W(i, i), smin));
            if (i >= 1 && ((sec >> i) & 1ull)) {
                E w11 = W(i - 1, i - 1), w12 = W(i - 1, i), w21 = W(i, i - 1), w22 = W(i, i);
                const bool sw = mag(w21) > mag(w11);
                E pa = sw ? w21 : w11, pb = sw ? w22 : w12, pc = sw ? w11 : w21, pd = sw ? w12 : w22;
                E ia = rcp(floor_pivot(pa, smin));
                E m = pc * ia;
                F.fa[s] = ia;
                F.fb[s] = pb;
                F.fm[s] = m;
                F.fu[s] = rcp(floor_pivot(pd - m * pb, smin));
                F.sw[s] = sw;
            }
        }
    }
}

// Growth checks inside a block.  Upstream checks the right-hand side before every local
// solve of at most 32 rows (`max |rhs| > bignum/10`, src/ztgevc3.cpp:183-199, bsize = 32 at
// :454; src/dtgevc3.cpp:688-698); a block here has up to 64 rows, so the substitution calls
// g.mid(r, jtop) once every row at or above kMidRow is solved, where rows [0, jtop] hold the
// partially updated right-hand side of the block's upper rows.  Without it, a column that
// enters the block near bignum/10 can overflow within the block where upstream's solves stay
// finite.
//
// With the per-row cap (Guard<true, ...>), a solved component above g.cap (the largest
// finite value / 4096: room for the updates of a block's rows, |w_ij| <= 2) makes the
// substitution rescale the column, g.rescale(r, s), by the factor that brings that
// component to g.target (bignum/10, the level the block checks rescale to), computed from the
// row's right-hand side and pivot without forming the overflowing product; a 2x2 block does
// this for its second and then its first component.
// Upstream rescales whole 32-column panels, so a column whose own growth passes the range of
// the format inside 32 rows (rows of a graded pencil differing by 1e16) can still come back
// finite there, scaled down by the guards of other columns of its panel; the cap gives the
// per-column guards the same reach for one compare per row.  NoGuard is the unguarded form.
constexpr int kMidRow = 32;
struct NoGuard {
    static constexpr bool on = false;
    template <class E>
    __device__ __forceinline__ void mid(E (&)[2], int) const {}
    template <class E, class T>
    __device__ __forceinline__ void rescale(E (&)[2], T) const {}
    static constexpr double cap = 0, target = 0;
};
// ON: mid-block check and per-row cap; off: the mid-block check only
template <bool ON, class R, class MF, class RF>
struct Guard {
    static constexpr bool on = ON;
    MF mid_f;
    RF rescale_f;
    R cap, target;
    template <class E>
    __device__ __forceinline__ void mid(E (&r)[2], int jtop) const { mid_f(r, jtop); }
    template <class E>
    __device__ __forceinline__ void rescale(E (&r)[2], R s) const { rescale_f(r, s); }
};
template <bool ON, class R, class MF, class RF>
__device__ __forceinline__ Guard<ON, R, MF, RF> make_guard(R cap, R target, MF mid, RF rescale)
{
    return Guard<ON, R, MF, RF>{mid, rescale, cap, target};
}

// Per-row cap: x = r_j / w_jj (x0 = r_j, iv = 1 / w_jj, uniform across the warp) passed
// g.cap: rescale the column so that |x| becomes g.target, and return the recomputed x.
template <class E, class G>
__device__ __forceinline__ E cap_row(E (&r)[2], const G &g, E x0, E iv)
{
    const auto s = (g.target / mag(iv)) / mag(x0);
    g.rescale(r, s);
    return (s * x0) * iv;
}

// The same for a 2x2 block: xq = (r2 - m r1) iu, xp = (r1 - b xq) ia (uniform inputs).
template <class E, class G>
__device__ __forceinline__ void cap_pair(E (&r)[2], const G &g, E r1, E r2, E m, E iu, E b, E ia, E &xp, E &xq)
{
    auto s = (g.target / mag(iu)) / (mag(r2) + mag(m) * mag(r1));
    if (s < decltype(s)(1)) {
        g.rescale(r, s);
        r1 = s * r1;
        r2 = s * r2;
    }
    xq = (r2 - m * r1) * iu;
    s = (g.target / mag(ia)) / (mag(r1) + mag(b) * mag(xq));
    if (s < decltype(s)(1)) {
        g.rescale(r, s);
        r1 = s * r1;
        xq = s * xq;
    }
    xp = (r1 - b * xq) * ia;
}

// Block back substitution of one eigenvector held in r (rows [jlo, nrows)); on return r
// holds the solution in those rows (rows below jlo receive updates that mean nothing).
// W(i, j) gives the shifted operator entry.  jlo must not split a 2x2 block.  The row loop
// is unrolled over the block's 64 rows, so every row index, register slot and lane test is
// a constant; rows at or past nrows (uniform across the warp) are skipped.
template <class E, class WF, class G = NoGuard>
__device__ __forceinline__ void back_substitute(E (&r)[2], const Factors<E> &F, uint64_t sec, int nrows, int lane,
                                                WF W, int jlo = 0, G g = G())
{
    bool skip = false;  // the row was consumed by the 2x2 block above it
    bool checked = nrows <= kMidRow;
#pragma unroll
    for (int j = kBlock - 1; j >= 0; j--) {
        if (j >= nrows || j < jlo) continue;
        if (skip) {
            skip = false;
            continue;
        }
        // the first unsolved row below kMidRow is kMidRow - 1, or kMidRow - 2 when a 2x2
        // block took rows (kMidRow - 1, kMidRow): two call sites, not one per row
        if ((j == kMidRow - 1 || j == kMidRow - 2) && !checked) {
            checked = true;
            g.mid(r, j);
        }
        if (j >= 1 && ((sec >> j) & 1ull)) {
            const int p = j - 1, q = j;
            const E rp = shfl(r[p >> 5], p & 31);
            const E rq = r[q >> 5];  // valid on the owner of q, which does the solve
            const bool sw = F.sw[q >> 5];
            const E ia = F.fa[q >> 5], b = F.fb[q >> 5], m = F.fm[q >> 5], iu = F.fu[q >> 5];
            const E r1 = sw ? rq : rp, r2 = sw ? rp : rq;
            E xq = (r2 - m * r1) * iu;
            E xp = (r1 - b * xq) * ia;
            xq = shfl(xq, q & 31);
            xp = shfl(xp, q & 31);
            if constexpr (G::on) {
                if (!(mag(xq) <= g.cap && mag(xp) <= g.cap)) {
                    const int o = q & 31;
                    cap_pair(r, g, shfl(r1, o), shfl(r2, o), shfl(m, o), shfl(iu, o), shfl(b, o), shfl(ia, o), xp, xq);
                }
            }
            if (lane == (p & 31)) r[p >> 5] = xp;
            if (lane == (q & 31)) r[q >> 5] = xq;
            if (p > 0) {
                if (p >= 32 || lane < p) r[0] = r[0] - (W(lane, p) * xp + W(lane, q) * xq);
                if (p > 32 && lane + 32 < p) r[1] = r[1] - (W(lane + 32, p) * xp + W(lane + 32, q) * xq);
            }
            skip = true;
        } else {
            E x = shfl(r[j >> 5] * F.inv1[j >> 5], j & 31);
            if constexpr (G::on) {
                if (!(mag(x) <= g.cap)) x = cap_row(r, g, shfl(r[j >> 5], j & 31), shfl(F.inv1[j >> 5], j & 31));
            }
            if (lane == (j & 31)) r[j >> 5] = x;
            if (j > 0) {
                if (j >= 32 || lane < j) r[0] = r[0] - W(lane, j) * x;
                if (j > 32 && lane + 32 < j) r[1] = r[1] - W(lane + 32, j) * x;
            }
        }
    }
}

// The same substitution as a runtime row loop (fewer registers: one code path per row
// instead of 64): used where register pressure matters more than instructions per row.
template <class E, class WF, class G = NoGuard>
__device__ __forceinline__ void back_substitute_loop(E (&r)[2], const Factors<E> &F, uint64_t sec, int nrows,
                                                     int lane, WF W, int jlo = 0, G g = G())
{
    // one row, or the 2x2 block ending at row j; returns the next unsolved row
    auto step = [&](int j) -> int {
        if (j >= 1 && ((sec >> j) & 1ull)) {
            const int p = j - 1, q = j;
            const int sq = q >> 5;
            const E rp = shfl(row_of(r, p), p & 31);
            const E rq = row_of(r, q);
            const bool sw = sq ? F.sw[1] : F.sw[0];
            const E ia = sq ? F.fa[1] : F.fa[0], b = sq ? F.fb[1] : F.fb[0];
            const E m = sq ? F.fm[1] : F.fm[0], iu = sq ? F.fu[1] : F.fu[0];
            const E r1 = sw ? rq : rp, r2 = sw ? rp : rq;
            E xq = (r2 - m * r1) * iu;
            E xp = (r1 - b * xq) * ia;
            xq = shfl(xq, q & 31);
            xp = shfl(xp, q & 31);
            if constexpr (G::on) {
                if (!(mag(xq) <= g.cap && mag(xp) <= g.cap)) {
                    const int o = q & 31;
                    cap_pair(r, g, shfl(r1, o), shfl(r2, o), shfl(m, o), shfl(iu, o), shfl(b, o), shfl(ia, o), xp, xq);
                }
            }
            set_row(r, p, lane, xp);
            set_row(r, q, lane, xq);
            if (lane < p) r[0] = r[0] - (W(lane, p) * xp + W(lane, q) * xq);
            if (p > 32 && lane + 32 < p) r[1] = r[1] - (W(lane + 32, p) * xp + W(lane + 32, q) * xq);
            return j - 2;
        }
        E x = shfl((j >> 5) ? r[1] * F.inv1[1] : r[0] * F.inv1[0], j & 31);
        if constexpr (G::on) {
            if (!(mag(x) <= g.cap))
                x = cap_row(r, g, shfl(row_of(r, j), j & 31), shfl((j >> 5) ? F.inv1[1] : F.inv1[0], j & 31));
        }
        set_row(r, j, lane, x);
        if (lane < j) r[0] = r[0] - W(lane, j) * x;
        if (j > 32 && lane + 32 < j) r[1] = r[1] - W(lane + 32, j) * x;
        return j - 1;
    };
    // rows at and above kMidRow, the mid-block check, then the rest (no per-row test)
    int j = nrows - 1;
    const int jsplit = jlo > kMidRow ? jlo : kMidRow;
    while (j >= jsplit) j = step(j);
    if (nrows > kMidRow && j >= jlo) g.mid(r, j);
    while (j >= jlo) j = step(j);
}

// The substitution of back_substitute_loop for the shifted operator W = ac S - b P of the
// diagonal solves (S, P: the block in shared memory, leading dimension kSmLd; b real for a
// real column, complex for a (Re, Im) pair), with two differences in form:
//  * the update of the rows above a solved row j is r -= S(:, j) (ac x) - P(:, j) (b x):
//    two FMAs per row slot against ac x and b x formed once per step, instead of forming
//    W(i, j) for every row;
//  * rows 32..63 (slot 1) and rows 0..31 (slot 0) are solved by separate loops, so every
//    step reads and writes a slot fixed at compile time; the 2x2 block (31, 32), whose rows
//    lie in different slots, is a case of its own.
// Pivots, 2x2 LU steps, the per-row cap and the mid-block check are those of
// back_substitute_loop (jlo = 0).
template <class E, class B, class R, class G>
__device__ __forceinline__ void back_substitute_sp(E (&r)[2], const Factors<E> &F, uint64_t sec, int nrows, int lane,
                                                   const R *Ss, const R *Ps, R ac, B b, G g)
{
    // rows i < j of both slots: r_i -= S(i, j) u - P(i, j) v
    auto upd1 = [&](int j, E x) {
        const E u = ac * x, v = b * x;
        const R *sc = Ss + j * kSmLd, *pc = Ps + j * kSmLd;
        if (lane < j) r[0] = (r[0] - sc[lane] * u) + pc[lane] * v;
        if (lane + 32 < j) r[1] = (r[1] - sc[lane + 32] * u) + pc[lane + 32] * v;
    };
    auto upd2 = [&](int p, int q, E xp, E xq) {
        const E up = ac * xp, vp = b * xp, uq = ac * xq, vq = b * xq;
        const R *sp = Ss + p * kSmLd, *pp = Ps + p * kSmLd, *sq = Ss + q * kSmLd, *pq = Ps + q * kSmLd;
        if (lane < p) r[0] = ((r[0] - sp[lane] * up) - sq[lane] * uq) + (pp[lane] * vp + pq[lane] * vq);
        if (lane + 32 < p)
            r[1] = ((r[1] - sp[lane + 32] * up) - sq[lane + 32] * uq) + (pp[lane + 32] * vp + pq[lane + 32] * vq);
    };
    // one 1x1 row j held in slot SL
    auto step1 = [&](auto slot, int j) {
        constexpr int SL = decltype(slot)::value;
        E x = shfl(r[SL] * F.inv1[SL], j & 31);
        if constexpr (G::on) {
            if (!(mag(x) <= g.cap)) x = cap_row(r, g, shfl(r[SL], j & 31), shfl(F.inv1[SL], j & 31));
        }
        if (lane == (j & 31)) r[SL] = x;
        upd1(j, x);
    };
    // the 2x2 block (p, q = p + 1), rows in slots SP, SQ; the owner of q solves it
    auto step2 = [&](auto sp_, auto sq_, int p) {
        constexpr int SP = decltype(sp_)::value, SQ = decltype(sq_)::value;
        const int q = p + 1;
        const E rp = shfl(r[SP], p & 31);
        const E rq = r[SQ];
        const bool sw = F.sw[SQ];
        const E ia = F.fa[SQ], bb = F.fb[SQ], m = F.fm[SQ], iu = F.fu[SQ];
        const E r1 = sw ? rq : rp, r2 = sw ? rp : rq;
        E xq = (r2 - m * r1) * iu;
        E xp = (r1 - bb * xq) * ia;
        xq = shfl(xq, q & 31);
        xp = shfl(xp, q & 31);
        if constexpr (G::on) {
            if (!(mag(xq) <= g.cap && mag(xp) <= g.cap)) {
                const int o = q & 31;
                cap_pair(r, g, shfl(r1, o), shfl(r2, o), shfl(m, o), shfl(iu, o), shfl(bb, o), shfl(ia, o), xp, xq);
            }
        }
        if (lane == (p & 31)) r[SP] = xp;
        if (lane == (q & 31)) r[SQ] = xq;
        if (p > 0) upd2(p, q, xp, xq);
    };
    using S0 = std::integral_constant<int, 0>;
    using S1 = std::integral_constant<int, 1>;
    int j = nrows - 1;
    while (j >= kMidRow) {
        if ((sec >> j) & 1ull) {
            if (j == kMidRow) step2(S0(), S1(), j - 1);
            else step2(S1(), S1(), j - 1);
            j -= 2;
        } else {
            step1(S1(), j);
            j -= 1;
        }
    }
    if (nrows > kMidRow && j >= 0) g.mid(r, j);
    while (j >= 0) {
        if (j >= 1 && ((sec >> j) & 1ull)) {
            step2(S0(), S0(), j - 1);
            j -= 2;
        } else {
            step1(S0(), j);
            j -= 1;
        }
    }
}

// bit j set: rows (j-1, j) of the block form a 2x2 block, pairing greedily from the bottom
template <class R>
__device__ __forceinline__ void pair_mask(const R *Ss, int jnb, uint64_t *out)
{
    if (threadIdx.x < 32) {
        const int l = threadIdx.x;
        const bool b0 = l >= 1 && l < jnb && Ss[l + (l - 1) * kSmLd] != R(0);
        const bool b1 = l + 32 < jnb && Ss[(l + 32) + (l + 31) * kSmLd] != R(0);
        const uint64_t sub = (uint64_t)__ballot_sync(0xffffffffu, b0) | ((uint64_t)__ballot_sync(0xffffffffu, b1) << 32);
        // Greedy pairing from the bottom takes, in every run of set bits, the top bit and
        // every second one below it: bit j is taken when the run of set bits directly above
        // it has even length.  Each lane decides its two bits.
        uint64_t sec = 0;
#pragma unroll
        for (int s = 0; s < 2; s++) {
            const int j = l + 32 * s;
            bool take = false;
            if ((sub >> j) & 1ull) {
                int k = j + 1;
                while (k < 64 && ((sub >> k) & 1ull)) k++;
                take = ((k - j - 1) & 1) == 0;
            }
            sec |= (uint64_t)__ballot_sync(0xffffffffu, take) << (32 * s);
        }
        if (l == 0) *out = sec;
    }
}

// ------------------------------------------------------------------------------------
// Real arithmetic (s/d): real columns and (Re, Im) column pairs
// ------------------------------------------------------------------------------------
template <class R>
__global__ void __launch_bounds__(256) diag_solve_real(DiagArgs<R> a)
{
    extern __shared__ __align__(16) unsigned char smem_diag[];
    __shared__ uint64_t s_sec;
    R *Ss = reinterpret_cast<R *>(smem_diag);
    R *Ps = Ss + kSmLd * kBlock;
    const int jnb = a.r1 - a.r0;
    load_block<R, 16>(a.S, a.lds, a.P, a.ldp, a.r0, jnb, 1, Ss, Ps);
    __syncthreads();
    pair_mask(Ss, jnb, &s_sec);
    __syncthreads();
    const uint64_t sec = s_sec;

    const int lane = threadIdx.x & 31;
    const int warps = (gridDim.x * blockDim.x) >> 5;
    for (int it = a.it0 + ((blockIdx.x * blockDim.x + threadIdx.x) >> 5); it < a.nitems; it += warps) {
        const int c = a.items[it];
        const uint8_t kd = a.kind[c];
        const int k = a.colk[c];
        const int kl = k - a.r0;
        const bool diag = k < a.r1;
        const R ac = a.coef[4 * c + 0], br = a.coef[4 * c + 1], bi = a.coef[4 * c + 2], smin = a.coef[4 * c + 3];
        R *colr = a.X + (size_t)c * a.ldx;
        const int nrows = diag ? kl : jnb;
        if (kd == kReal) {
            const int top = k;
            auto W = [&](int i, int j) -> R { return ac * Ss[i + j * kSmLd] - br * Ps[i + j * kSmLd]; };
            R r[2];
            R seed = diag ? R(1) : R(0);
#pragma unroll
            for (int s = 0; s < 2; s++) {
                int i = lane + 32 * s;
                R v = R(0);
                if (i < nrows) v = diag ? -W(i, kl) : colr[a.r0 + i];
                r[s] = v;
            }
            if (nrows > 0) {
                R mx = warp_max(fmax(fabs(r[0]), fabs(r[1])));
                if (mx > a.thr_rhs) {
                    R sc = a.thr_rhs / mx;
                    r[0] *= sc; r[1] *= sc; seed *= sc;
                    if (!diag) {
                        scale_above(a, colr, c, sc, lane); scale_rows(colr, a.r1, top + 1, sc, lane);
                        scale_lower_y(a, a.Y + (size_t)c * a.ldy, sc, lane);
                    }
                }
            }
            Factors<R> F;
            factor_rows(F, sec, nrows, lane, smin, W);
            auto rescale = [&](R (&rr)[2], R sc) {  // the whole column, by sc
                rr[0] *= sc; rr[1] *= sc; seed *= sc;
                if (!diag) {
                    scale_above(a, colr, c, sc, lane); scale_rows(colr, a.r1, top + 1, sc, lane);
                    scale_lower_y(a, a.Y + (size_t)c * a.ldy, sc, lane);
                }
            };
            auto mid = [&](R (&rr)[2], int jtop) {
                const R mx = warp_max(lane <= jtop ? fabs(rr[0]) : R(0));
                if (mx > a.thr_rhs) rescale(rr, a.thr_rhs / mx);
            };
            back_substitute_sp(r, F, sec, nrows, lane, Ss, Ps, ac, br,
                               make_guard<true>(limits<R>::big / R(4096), a.thr_rhs, mid, rescale));
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
                if (!diag) {
                    scale_above(a, colr, c, sc, lane); scale_rows(colr, a.r1, top + 1, sc, lane);
                    scale_lower_y(a, a.Y + (size_t)c * a.ldy, sc, lane);
                }
            }
            R ys[2], yp[2];
#pragma unroll
            for (int s = 0; s < 2; s++) {
                int i = lane + 32 * s;
                if (i < jnb) colr[a.r0 + i] = x[s];
                ys[s] = -ac * x[s];
                yp[s] = br * x[s];
            }
            write_y(a, a.Y + (size_t)c * a.ldy, jnb, diag, lane, ys, yp);
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
                        scale_above(a, colr, c, sc, lane); scale_rows(colr, a.r1, top + 1, sc, lane);
                        scale_above(a, coli, c + 1, sc, lane); scale_rows(coli, a.r1, top + 1, sc, lane);
                        scale_lower_y(a, a.Y + (size_t)c * a.ldy, sc, lane);
                        scale_lower_y(a, a.Y + (size_t)(c + 1) * a.ldy, sc, lane);
                    }
                }
            }
            Factors<C> F;
            factor_rows(F, sec, nrows, lane, smin, W);
            auto rescale = [&](C (&rr)[2], R sc) {  // the whole column pair, by sc
                rr[0] = sc * rr[0]; rr[1] = sc * rr[1]; seed0 = sc * seed0; seed1 = sc * seed1;
                if (!diag) {
                    scale_above(a, colr, c, sc, lane); scale_rows(colr, a.r1, top + 1, sc, lane);
                    scale_above(a, coli, c + 1, sc, lane); scale_rows(coli, a.r1, top + 1, sc, lane);
                    scale_lower_y(a, a.Y + (size_t)c * a.ldy, sc, lane);
                    scale_lower_y(a, a.Y + (size_t)(c + 1) * a.ldy, sc, lane);
                }
            };
            auto mid = [&](C (&rr)[2], int jtop) {
                const R mx = warp_max(lane <= jtop ? fmax(fabs(rr[0].x), fabs(rr[0].y)) : R(0));
                if (mx > a.thr_rhs) rescale(rr, a.thr_rhs / mx);
            };
            back_substitute_sp(r, F, sec, nrows, lane, Ss, Ps, ac, b,
                               make_guard<true>(limits<R>::big / R(4096), a.thr_rhs, mid, rescale));
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
                    scale_above(a, colr, c, sc, lane); scale_rows(colr, a.r1, top + 1, sc, lane);
                    scale_above(a, coli, c + 1, sc, lane); scale_rows(coli, a.r1, top + 1, sc, lane);
                    scale_lower_y(a, a.Y + (size_t)c * a.ldy, sc, lane);
                    scale_lower_y(a, a.Y + (size_t)(c + 1) * a.ldy, sc, lane);
                }
            }
            R ysr[2], ysi[2], ypr[2], ypi[2];
#pragma unroll
            for (int s = 0; s < 2; s++) {
                int i = lane + 32 * s;
                if (i < jnb) { colr[a.r0 + i] = x[s].x; coli[a.r0 + i] = x[s].y; }
                C yp = b * x[s];
                ysr[s] = -ac * x[s].x;
                ysi[s] = -ac * x[s].y;
                ypr[s] = yp.x;
                ypi[s] = yp.y;
            }
            R *yre = a.Y + (size_t)c * a.ldy;
            write_y(a, yre, jnb, diag, lane, ysr, ypr);
            write_y(a, yre + a.ldy, jnb, diag, lane, ysi, ypi);
        }
    }
}

// ------------------------------------------------------------------------------------
// Complex arithmetic (c/z): S triangular, one complex column per eigenvalue
// ------------------------------------------------------------------------------------
// 16 warps per CTA: in double complex the S/P block (133 KB) allows one CTA per SM, so a
// larger CTA is how more eigenvectors share the block and hide the solves' latency
constexpr int kDiagThreadsCplx = 512;
template <class R>
__global__ void __launch_bounds__(kDiagThreadsCplx, 1) diag_solve_cplx(DiagArgs<R> a)
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
                    scale_above(a, col, c, sc, lane); scale_rows(col, a.r1, top + 1, sc, lane);
                    scale_lower_y(a, Y + (size_t)c * a.ldy, sc, lane);
                }
            }
        }
        Factors<C> F;
        factor_rows(F, 0ull, nrows, lane, smin, W);
        // The unrolled substitution runs without the per-row cap (its compare on every row
        // costs a quarter of this kernel); a block in which a component passed the cap, or
        // overflowed, is solved again from its right-hand side with the cap, in loop form.
        // Factors applied to the stored rows during the first pass (acc) carry over.
        const C r_in[2] = {r[0], r[1]};
        R acc = R(1);
        auto rescale = [&](C (&rr)[2], R sc) {  // the whole column, by sc
            rr[0] = sc * rr[0]; rr[1] = sc * rr[1]; seed = sc * seed; acc *= sc;
            if (!diag) {
                scale_above(a, col, c, sc, lane); scale_rows(col, a.r1, top + 1, sc, lane);
                scale_lower_y(a, Y + (size_t)c * a.ldy, sc, lane);
            }
        };
        auto mid = [&](C (&rr)[2], int jtop) {  // a non-finite maximum (first pass) is left to the second
            const R mx = warp_max(lane <= jtop ? l1abs(rr[0]) : R(0));
            if (mx > a.thr_rhs && mx <= limits<R>::big) rescale(rr, a.thr_rhs / mx);
        };
        const R cap = limits<R>::big / R(4096);
        back_substitute(r, F, 0ull, nrows, lane, W, 0, make_guard<false>(cap, a.thr_rhs, mid, rescale));
        if (__any_sync(0xffffffffu, !(l1abs(r[0]) <= cap) || !(l1abs(r[1]) <= cap))) {
            r[0] = acc * r_in[0];
            r[1] = acc * r_in[1];
            back_substitute_loop(r, F, 0ull, nrows, lane, W, 0, make_guard<true>(cap, a.thr_rhs, mid, rescale));
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
                scale_above(a, col, c, sc, lane); scale_rows(col, a.r1, top + 1, sc, lane);
                scale_lower_y(a, Y + (size_t)c * a.ldy, sc, lane);
            }
        }
        C ys[2], yp[2];
#pragma unroll
        for (int s = 0; s < 2; s++) {
            int i = lane + 32 * s;
            if (i < jnb) col[a.r0 + i] = x[s];
            ys[s] = -(ac * x[s]);
            yp[s] = bc * x[s];
        }
        write_y(a, Y + (size_t)c * a.ldy, jnb, diag, lane, ys, yp);
    }
}

}  // namespace xtg
