// Eigenvalue reordering of a complex generalized Schur pencil (LAPACK xTGEXC for complex
// pencils, ZTGEXC / CTGEXC with their single swaps ZTGEX2 / CTGEX2): the eigenvalue at row
// IFST moves to row ILST by swaps of adjacent 1x1 diagonal blocks.  One swap of rows and
// columns (j, j+1) is the equivalence transformation of the direct swapping method
// (B. Kagstrom, "A direct method for reordering eigenvalues in the generalized real Schur form
// of a regular matrix pair (A, B)", 1993; B. Kagstrom and P. Poromaa, 1996), here for 1x1
// blocks, where it reduces to two Givens rotations computed from the 2x2 blocks
//     S = A[j:j+2, j:j+2], T = B[j:j+2, j:j+2]:
//   * right rotation (columns) from f = s11 t00 - t11 s00, g = s11 t01 - t11 s01: the
//     rotation (cz, sz) with [cz sz; -conj(sz) cz] [g; f] = [r; 0], sz negated, applied to the
//     column pairs as (x, y) <- (cz x + conj(sz) y, cz y - sz x);
//   * left rotation (rows) that zeroes the new (1, 0) entry of S (when |s11 t00| >= |s00 t11|)
//     or of T, applied to the row pairs as (x, y) <- (cq x + sq y, cq y - conj(sq) x);
//   * the swap is accepted when both new (1, 0) entries are at most 20 eps ||block||_F (the
//     weak test) and undoing both rotations on the swapped blocks gives back the original
//     blocks within the same bound (the strong test); otherwise the pencil is left as it is
//     and INFO = 1.
// Every rotation has a real cosine >= 0 (LAPACK's ZLARTG convention), so the results match
// LAPACK's to rounding.  Q (rows of the left rotations, conjugated) and Z (right rotations)
// are updated when asked.
//
// B200 form: one CTA walks the swaps in order (each depends on the previous one); thread 0
// computes a swap's rotations and tests from the 2x2 blocks, then the CTA applies them to the
// two columns of A, B, Z and the two rows of A, B and columns of Q, O(n) work per swap.
//
// Real pencils (D/STGEXC, with their swaps D/STGEX2): moves whose rows hold only 1x1
// diagonal blocks, by the same method in real arithmetic, following the real routine's own
// conventions: with (cs, sn) the rotation [cs sn; -sn cs] [F; G] = [r; 0] (cs >= 0, r of
// F's sign; F = s11 t00 - t11 s00, G = s11 t01 - t11 s01), the columns take (c, s) =
// (sn, -cs), the rows the rotation that zeroes the new (1, 0) entry of S or T, both applied
// as (x, y) <- (c x + s y, c y - s x); Z takes the column rotation, Q the row rotation.
// Moves across or of 2x2 blocks (complex pairs) run the general walk and swaps of
// tgexc_real_blocks.cuh (a small generalized Sylvester equation per swap, LAPACK's block
// walk with its 2x2 splits); IFST is in and out there, as in D/STGEXC.
#include "../../include/xtgevc3.h"
#include "common.cuh"
#include "engine.cuh"
#include "tgexc_real_blocks.cuh"

#include <algorithm>
#include <string>

namespace xtg {
namespace {

constexpr int kReorderThreads = 512;

template <class R>
__device__ __forceinline__ R cabs_(cplx<R> v) { return hypot(v.x, v.y); }

// Givens rotation with real cosine c >= 0: [c s; -conj(s) c] [f; g] = [r; 0].
template <class R>
__device__ void givens(cplx<R> f, cplx<R> g, R &c, cplx<R> &s)
{
    if (g.x == R(0) && g.y == R(0)) {
        c = R(1);
        s = cplx<R>(R(0), R(0));
        return;
    }
    if (f.x == R(0) && f.y == R(0)) {
        const R ga = cabs_(g);
        c = R(0);
        s = cplx<R>(g.x / ga, -g.y / ga);
        return;
    }
    const R fa = cabs_(f), ga = cabs_(g), h = hypot(fa, ga);
    c = fa / h;
    const cplx<R> u(f.x / fa, f.y / fa);  // f / |f|
    s = (R(1) / h) * (conjg(g) * u);
}

// (x, y) <- (c x + s y, c y - conj(s) x)
template <class R>
__device__ __forceinline__ void rot(cplx<R> &x, cplx<R> &y, R c, cplx<R> s)
{
    const cplx<R> xn = c * x + s * y, yn = c * y - conjg(s) * x;
    x = xn;
    y = yn;
}

// Complex product with every multiply and add rounded on its own (no fused multiply-add):
// the swap's f and g are formed this way, as LAPACK forms them, so that a product at the
// edge of the range overflows (and the swap is rejected) exactly when LAPACK's does.
__device__ __forceinline__ cplx<double> cmul_sep(cplx<double> a, cplx<double> b)
{
    return {__dsub_rn(__dmul_rn(a.x, b.x), __dmul_rn(a.y, b.y)), __dadd_rn(__dmul_rn(a.x, b.y), __dmul_rn(a.y, b.x))};
}
__device__ __forceinline__ cplx<float> cmul_sep(cplx<float> a, cplx<float> b)
{
    return {__fsub_rn(__fmul_rn(a.x, b.x), __fmul_rn(a.y, b.y)), __fadd_rn(__fmul_rn(a.x, b.y), __fmul_rn(a.y, b.x))};
}
__device__ __forceinline__ cplx<double> csub_sep(cplx<double> a, cplx<double> b)
{
    return {__dsub_rn(a.x, b.x), __dsub_rn(a.y, b.y)};
}
__device__ __forceinline__ cplx<float> csub_sep(cplx<float> a, cplx<float> b)
{
    return {__fsub_rn(a.x, b.x), __fsub_rn(a.y, b.y)};
}
template <class R>
__device__ __forceinline__ bool cfinite(cplx<R> v) { return isfinite(v.x) && isfinite(v.y); }

// Frobenius norm of a 2x2 block (scaled: no overflow or underflow of the squares)
template <class R>
__device__ __forceinline__ R fnorm2(cplx<R> a, cplx<R> b, cplx<R> c, cplx<R> d)
{
    return hypot(hypot(cabs_(a), cabs_(b)), hypot(cabs_(c), cabs_(d)));
}

// Rotation passes of a swap, with every thread's pairs loaded before any is stored (one
// memory round trip per batch instead of one per element): element i of the pass is the
// pair (x(i), y(i)) of matrix M (one matrix) or of M and N (two, with the same rotation).
// pairs per thread and batch (double complex: 1, its kernel has no registers to spare)
template <class E>
constexpr int kBatchOf = sizeof(E) >= 16 ? 1 : 4;

template <int KB, class E, class AX, class AY, class ROT>
__device__ __forceinline__ void rot_pass(int cnt, AX ax, AY ay, ROT rot)
{
    for (int base = threadIdx.x; base < cnt; base += KB * blockDim.x) {
        E x[KB], y[KB];
#pragma unroll
        for (int u = 0; u < KB; u++) {
            const int i = base + u * blockDim.x;
            if (i < cnt) {
                x[u] = ax(i);
                y[u] = ay(i);
            }
        }
#pragma unroll
        for (int u = 0; u < KB; u++) {
            const int i = base + u * blockDim.x;
            if (i < cnt) {
                rot(x[u], y[u]);
                ax(i) = x[u];
                ay(i) = y[u];
            }
        }
    }
}

template <class R>
struct ReorderArgs {
    int n, ifst, ilst, wantq, wantz;  // ifst, ilst 0-based
    cplx<R> *A, *B, *Q, *Z;
    int lda, ldb, ldq, ldz;
    int *status;  // {position reached, or first row of the rejected swap; 0 / 1}
};

template <class R>
__global__ void __launch_bounds__(kReorderThreads, 1) tgexc_cplx_kernel(ReorderArgs<R> a)
{
    using C = cplx<R>;
    __shared__ R s_cz, s_cq;
    __shared__ C s_szc, s_sq;
    __shared__ int s_ok;
    const R eps = limits<R>::eps, smlnum = limits<R>::safemin / eps;
    const int step = a.ifst < a.ilst ? 1 : -1;
    int here = a.ifst, bad = -1;
    auto at = [](C *M, int ld, int i, int j) -> C & { return M[(size_t)i + (size_t)j * ld]; };
    while (here != a.ilst) {
        const int j = step > 0 ? here : here - 1;  // swap rows / columns j and j + 1
        if (threadIdx.x == 0) {
            const C a00 = at(a.A, a.lda, j, j), a01 = at(a.A, a.lda, j, j + 1);
            const C a10 = at(a.A, a.lda, j + 1, j), a11 = at(a.A, a.lda, j + 1, j + 1);
            const C b00 = at(a.B, a.ldb, j, j), b01 = at(a.B, a.ldb, j, j + 1);
            const C b10 = at(a.B, a.ldb, j + 1, j), b11 = at(a.B, a.ldb, j + 1, j + 1);
            const R tha = fmax(R(20) * eps * fnorm2(a00, a10, a01, a11), smlnum);
            const R thb = fmax(R(20) * eps * fnorm2(b00, b10, b01, b11), smlnum);
            const C f = csub_sep(cmul_sep(a11, b00), cmul_sep(b11, a00));
            const C g = csub_sep(cmul_sep(a11, b01), cmul_sep(b11, a01));
            const R sa = cabs_(a11) * cabs_(b00), sb = cabs_(a00) * cabs_(b11);
            R cz;
            C sz;
            givens(g, f, cz, sz);
            const C szc = conjg(-sz);  // the column pairs take (cz, conj(sz)) with sz negated
            C s00 = a00, s01 = a01, s10 = a10, s11 = a11, t00 = b00, t01 = b01, t10 = b10, t11 = b11;
            rot(s00, s01, cz, szc);
            rot(s10, s11, cz, szc);
            rot(t00, t01, cz, szc);
            rot(t10, t11, cz, szc);
            R cq;
            C sq;
            if (sa >= sb) givens(s00, s10, cq, sq);
            else givens(t00, t10, cq, sq);
            rot(s00, s10, cq, sq);
            rot(s01, s11, cq, sq);
            rot(t00, t10, cq, sq);
            rot(t01, t11, cq, sq);
            // a swap whose rotations or blocks are not finite is rejected (LAPACK's tests
            // compare NaN and fail the same way)
            bool ok = cabs_(s10) <= tha && cabs_(t10) <= thb && isfinite(cz) && isfinite(cq) && cfinite(szc) &&
                      cfinite(sq) && cfinite(s00) && cfinite(s01) && cfinite(s11) && cfinite(t00) && cfinite(t01) &&
                      cfinite(t11);
            if (ok) {
                // undo both rotations on the swapped blocks; the originals must come back
                const C szu = -szc, squ = -sq;
                C w00 = s00, w01 = s01, w10 = s10, w11 = s11, v00 = t00, v01 = t01, v10 = t10, v11 = t11;
                rot(w00, w01, cz, szu);
                rot(w10, w11, cz, szu);
                rot(v00, v01, cz, szu);
                rot(v10, v11, cz, szu);
                rot(w00, w10, cq, squ);
                rot(w01, w11, cq, squ);
                rot(v00, v10, cq, squ);
                rot(v01, v11, cq, squ);
                ok = fnorm2(w00 - a00, w10 - a10, w01 - a01, w11 - a11) <= tha &&
                     fnorm2(v00 - b00, v10 - b10, v01 - b01, v11 - b11) <= thb;
            }
            s_ok = ok ? 1 : 0;
            s_cz = cz;
            s_szc = szc;
            s_cq = cq;
            s_sq = sq;
        }
        __syncthreads();
        if (!s_ok) {
            bad = j;
            break;
        }
        const R cz = s_cz, cq = s_cq;
        const C szc = s_szc, sq = s_sq;
        // columns j, j+1: rows [0, j + 2) of A and B, all rows of Z (A's and B's pairs as one
        // pass of 2 (j + 2) elements)
        {
            const int m2 = j + 2;
            auto rc = [&](C &x, C &y) { rot(x, y, cz, szc); };
            rot_pass<kBatchOf<C>, C>(2 * m2,
                           [&](int i) -> C & { return i < m2 ? at(a.A, a.lda, i, j) : at(a.B, a.ldb, i - m2, j); },
                           [&](int i) -> C & {
                               return i < m2 ? at(a.A, a.lda, i, j + 1) : at(a.B, a.ldb, i - m2, j + 1);
                           },
                           rc);
            if (a.wantz)
                rot_pass<kBatchOf<C>, C>(a.n, [&](int i) -> C & { return at(a.Z, a.ldz, i, j); },
                               [&](int i) -> C & { return at(a.Z, a.ldz, i, j + 1); }, rc);
        }
        __syncthreads();  // the 2x2 block takes the column rotation before the row rotation
        // rows j, j+1: columns [j, n) of A and B; Q's columns j, j+1 take the conjugate rotation
        {
            const int m2 = a.n - j;
            rot_pass<kBatchOf<C>, C>(2 * m2,
                           [&](int i) -> C & { return i < m2 ? at(a.A, a.lda, j, j + i) : at(a.B, a.ldb, j, j + i - m2); },
                           [&](int i) -> C & {
                               return i < m2 ? at(a.A, a.lda, j + 1, j + i) : at(a.B, a.ldb, j + 1, j + i - m2);
                           },
                           [&](C &x, C &y) { rot(x, y, cq, sq); });
            if (a.wantq) {
                const C sqc = conjg(sq);
                rot_pass<kBatchOf<C>, C>(a.n, [&](int i) -> C & { return at(a.Q, a.ldq, i, j); },
                               [&](int i) -> C & { return at(a.Q, a.ldq, i, j + 1); },
                               [&](C &x, C &y) { rot(x, y, cq, sqc); });
            }
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            at(a.A, a.lda, j + 1, j) = C(R(0), R(0));
            at(a.B, a.ldb, j + 1, j) = C(R(0), R(0));
        }
        __syncthreads();
        here += step;
    }
    if (threadIdx.x == 0) {
        a.status[0] = bad >= 0 ? bad : here;
        a.status[1] = bad >= 0 ? 1 : 0;
    }
}

// Real plane rotation [c s; -s c] [f; g] = [r; 0] with c >= 0 and r of f's sign, computed in
// range (the scaled form near underflow and overflow).
template <class R>
__device__ void lartg_real(R f, R g, R &c, R &s)
{
    const R safmin = limits<R>::safemin, safmax = R(1) / safmin;
    const R rtmin = sqrt(safmin), rtmax = sqrt(safmax / R(2));
    if (g == R(0)) {
        c = R(1);
        s = R(0);
        return;
    }
    if (f == R(0)) {
        c = R(0);
        s = copysign(R(1), g);
        return;
    }
    const R f1 = fabs(f), g1 = fabs(g);
    if (f1 > rtmin && f1 < rtmax && g1 > rtmin && g1 < rtmax) {
        const R d = sqrt(f * f + g * g);
        c = f1 / d;
        s = g / copysign(d, f);
    } else {
        const R u = fmin(safmax, fmax(safmin, fmax(f1, g1)));
        const R fs = f / u, gs = g / u, d = sqrt(fs * fs + gs * gs);
        c = fabs(fs) / d;
        s = gs / copysign(d, f);
    }
}

// (x, y) <- (c x + s y, c y - s x)
template <class R>
__device__ __forceinline__ void rot_real(R &x, R &y, R c, R s)
{
    const R xn = c * x + s * y, yn = c * y - s * x;
    x = xn;
    y = yn;
}

__device__ __forceinline__ double mul_sep(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float mul_sep(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double sub_sep(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ float sub_sep(float a, float b) { return __fsub_rn(a, b); }

template <class R>
struct ReorderArgsReal {
    int n, ifst, ilst, wantq, wantz;  // ifst, ilst 0-based
    R *A, *B, *Q, *Z;
    int lda, ldb, ldq, ldz;
    int *status;  // {position reached, or first row of the rejected swap; 0 / 1 / 2}
};

template <class R>
__global__ void __launch_bounds__(kReorderThreads, 1) tgexc_real_kernel(ReorderArgsReal<R> a)
{
    __shared__ R s_cz, s_sz, s_cq, s_sq;
    __shared__ int s_ok;
    const R eps = limits<R>::eps, smlnum = limits<R>::safemin / eps;
    const int step = a.ifst < a.ilst ? 1 : -1;
    auto at = [](R *M, int ld, int i, int j) -> R & { return M[(size_t)i + (size_t)j * ld]; };
    // a 2x2 block in rows [lo - 1, hi + 1] (subdiagonal entries A(k + 1, k)) stops the move
    if (threadIdx.x == 0) {
        const int lo = min(a.ifst, a.ilst), hi = max(a.ifst, a.ilst);
        int pair = 0;
        for (int k = max(lo - 1, 0); k <= min(hi, a.n - 2); k++)
            if (at(a.A, a.lda, k + 1, k) != R(0)) pair = 1;
        s_ok = pair ? 0 : 1;
    }
    __syncthreads();
    if (!s_ok) {
        if (threadIdx.x == 0) {
            a.status[0] = a.ifst;
            a.status[1] = 2;
        }
        return;
    }
    int here = a.ifst, bad = -1;
    while (here != a.ilst) {
        const int j = step > 0 ? here : here - 1;  // swap rows / columns j and j + 1
        if (threadIdx.x == 0) {
            const R a00 = at(a.A, a.lda, j, j), a01 = at(a.A, a.lda, j, j + 1);
            const R a10 = at(a.A, a.lda, j + 1, j), a11 = at(a.A, a.lda, j + 1, j + 1);
            const R b00 = at(a.B, a.ldb, j, j), b01 = at(a.B, a.ldb, j, j + 1);
            const R b10 = at(a.B, a.ldb, j + 1, j), b11 = at(a.B, a.ldb, j + 1, j + 1);
            const R tha = fmax(R(20) * eps * hypot(hypot(a00, a10), hypot(a01, a11)), smlnum);
            const R thb = fmax(R(20) * eps * hypot(hypot(b00, b10), hypot(b01, b11)), smlnum);
            const R f = sub_sep(mul_sep(a11, b00), mul_sep(b11, a00));
            const R g = sub_sep(mul_sep(a11, b01), mul_sep(b11, a01));
            const R sa = fabs(a11) * fabs(b00), sb = fabs(a00) * fabs(b11);
            R cs, sn;
            lartg_real(f, g, cs, sn);
            const R cz = sn, sz = -cs;  // the column rotation
            R s00 = a00, s01 = a01, s10 = a10, s11 = a11, t00 = b00, t01 = b01, t10 = b10, t11 = b11;
            rot_real(s00, s01, cz, sz);
            rot_real(s10, s11, cz, sz);
            rot_real(t00, t01, cz, sz);
            rot_real(t10, t11, cz, sz);
            R cq, sq;
            if (sa >= sb) lartg_real(s00, s10, cq, sq);
            else lartg_real(t00, t10, cq, sq);
            rot_real(s00, s10, cq, sq);
            rot_real(s01, s11, cq, sq);
            rot_real(t00, t10, cq, sq);
            rot_real(t01, t11, cq, sq);
            bool ok = fabs(s10) <= tha && fabs(t10) <= thb && isfinite(cz) && isfinite(sz) && isfinite(cq) &&
                      isfinite(sq) && isfinite(s00) && isfinite(s01) && isfinite(s11) && isfinite(t00) &&
                      isfinite(t01) && isfinite(t11);
            if (ok) {  // undo both rotations on the swapped blocks: the originals must come back
                R w00 = s00, w01 = s01, w10 = s10, w11 = s11, v00 = t00, v01 = t01, v10 = t10, v11 = t11;
                rot_real(w00, w10, cq, -sq);
                rot_real(w01, w11, cq, -sq);
                rot_real(v00, v10, cq, -sq);
                rot_real(v01, v11, cq, -sq);
                rot_real(w00, w01, cz, -sz);
                rot_real(w10, w11, cz, -sz);
                rot_real(v00, v01, cz, -sz);
                rot_real(v10, v11, cz, -sz);
                ok = hypot(hypot(w00 - a00, w10 - a10), hypot(w01 - a01, w11 - a11)) <= tha &&
                     hypot(hypot(v00 - b00, v10 - b10), hypot(v01 - b01, v11 - b11)) <= thb;
            }
            s_ok = ok ? 1 : 0;
            s_cz = cz;
            s_sz = sz;
            s_cq = cq;
            s_sq = sq;
        }
        __syncthreads();
        if (!s_ok) {
            bad = j;
            break;
        }
        const R cz = s_cz, sz = s_sz, cq = s_cq, sq = s_sq;
        // columns j, j+1: rows [0, j + 2) of A and B, all rows of Z
        {
            const int m2 = j + 2;
            auto rc = [&](R &x, R &y) { rot_real(x, y, cz, sz); };
            rot_pass<kBatchOf<R>, R>(2 * m2,
                           [&](int i) -> R & { return i < m2 ? at(a.A, a.lda, i, j) : at(a.B, a.ldb, i - m2, j); },
                           [&](int i) -> R & {
                               return i < m2 ? at(a.A, a.lda, i, j + 1) : at(a.B, a.ldb, i - m2, j + 1);
                           },
                           rc);
            if (a.wantz)
                rot_pass<kBatchOf<R>, R>(a.n, [&](int i) -> R & { return at(a.Z, a.ldz, i, j); },
                               [&](int i) -> R & { return at(a.Z, a.ldz, i, j + 1); }, rc);
        }
        __syncthreads();  // the 2x2 block takes the column rotation before the row rotation
        // rows j, j+1: columns [j, n) of A and B; Q's columns j, j+1
        {
            const int m2 = a.n - j;
            auto rr = [&](R &x, R &y) { rot_real(x, y, cq, sq); };
            rot_pass<kBatchOf<R>, R>(2 * m2,
                           [&](int i) -> R & { return i < m2 ? at(a.A, a.lda, j, j + i) : at(a.B, a.ldb, j, j + i - m2); },
                           [&](int i) -> R & {
                               return i < m2 ? at(a.A, a.lda, j + 1, j + i) : at(a.B, a.ldb, j + 1, j + i - m2);
                           },
                           rr);
            if (a.wantq)
                rot_pass<kBatchOf<R>, R>(a.n, [&](int i) -> R & { return at(a.Q, a.ldq, i, j); },
                               [&](int i) -> R & { return at(a.Q, a.ldq, i, j + 1); }, rr);
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            at(a.A, a.lda, j + 1, j) = R(0);
            at(a.B, a.ldb, j + 1, j) = R(0);
        }
        __syncthreads();
        here += step;
    }
    if (threadIdx.x == 0) {
        a.status[0] = bad >= 0 ? bad : here;
        a.status[1] = bad >= 0 ? 1 : 0;
    }
}

// Real pencils with 2x2 blocks in the rows of the move (the general D/STGEXC walk and D/STGEX2
// swaps of tgexc_real_blocks.cuh, rb::walk_cta: thread 0 walks and computes each swap's
// small-block arithmetic, the CTA applies the swap between barriers; bounded by 4 n + 16 swaps,
// status 3 if that were ever reached).
// status: {ILST on exit (1-based), INFO (0 / 1 / 3), IFST on exit (1-based)}
template <class R>
__global__ void __launch_bounds__(kReorderThreads, 1)
    tgexc_real_blocks_kernel(rb::Pencil<R> p, int ifst, int ilst, int *status)
{
    __shared__ rb::WalkShared<R> sh;
    rb::walk_cta(rb::CtaDev{}, sh, p, ifst, ilst);
    if (threadIdx.x == 0) {
        status[0] = sh.ilst;
        status[1] = sh.info;
        status[2] = sh.ifst;
    }
}

// LAPACK xTGEXC's argument checks, in its order.
int tgexc_check(int wantq, int wantz, int n, int lda, int ldb, int ldq, int ldz, int ifst, int ilst)
{
    if (n < 0) return -3;
    if (lda < std::max(1, n)) return -5;
    if (ldb < std::max(1, n)) return -7;
    if (ldq < 1 || (wantq && ldq < std::max(1, n))) return -9;
    if (ldz < 1 || (wantz && ldz < std::max(1, n))) return -11;
    if (ifst < 1 || ifst > n) return -12;
    if (ilst < 1 || ilst > n) return -13;
    return 0;
}

// Device pointers.  On return *ilst is where the eigenvalue is (LAPACK: with INFO = 1, the
// first row of the swap that was rejected).  Returns 0, or 1 when a CUDA call failed.
template <class R>
int tgexc_device(cudaStream_t st, int wantq, int wantz, int n, cplx<R> *A, int lda, cplx<R> *B, int ldb, cplx<R> *Q,
                 int ldq, cplx<R> *Z, int ldz, int ifst, int *ilst, int *info)
{
    set_last_error("");
    *info = tgexc_check(wantq, wantz, n, lda, ldb, ldq, ldz, ifst, *ilst);
    if (*info) {
        set_last_error("xTGEXC: argument " + std::to_string(-*info) + " has an illegal value");
        return 0;
    }
    if (n <= 1 || ifst == *ilst) return 0;
    int *d_status = nullptr;
    int h_status[2] = {0, 0};
    cudaError_t e = cudaMallocAsync(&d_status, 2 * sizeof(int), st);
    if (e == cudaSuccess) {
        ReorderArgs<R> ra{n, ifst - 1, *ilst - 1, wantq ? 1 : 0, wantz ? 1 : 0, A, B, Q, Z, lda, ldb, ldq, ldz, d_status};
        tgexc_cplx_kernel<R><<<1, kReorderThreads, 0, st>>>(ra);
        count_launches(1);
        e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaMemcpyAsync(h_status, d_status, sizeof(h_status), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        cudaFreeAsync(d_status, st);
    }
    if (e != cudaSuccess) {
        set_last_error(std::string("xTGEXC: ") + cudaGetErrorString(e));
        *info = 1;
        return 1;
    }
    *ilst = h_status[0] + 1;
    *info = h_status[1];
    return 0;
}

// Host pointers: A, B (and Q, Z when wanted) go to the device, come back reordered.
template <class R>
void tgexc_host(int wantq, int wantz, int n, cplx<R> *A, int lda, cplx<R> *B, int ldb, cplx<R> *Q, int ldq,
                cplx<R> *Z, int ldz, int ifst, int *ilst, int *info)
{
    set_last_error("");
    *info = tgexc_check(wantq, wantz, n, lda, ldb, ldq, ldz, ifst, *ilst);
    if (*info) {
        set_last_error("xTGEXC: argument " + std::to_string(-*info) + " has an illegal value");
        return;
    }
    if (n <= 1 || ifst == *ilst) return;
    using C = cplx<R>;
    cudaStream_t st = nullptr;
    C *dm[4] = {nullptr, nullptr, nullptr, nullptr};
    C *hm[4] = {A, B, wantq ? Q : nullptr, wantz ? Z : nullptr};
    const int hl[4] = {lda, ldb, ldq, ldz};
    const size_t bytes = (size_t)n * n * sizeof(C);
    cudaError_t e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
    for (int k = 0; k < 4 && e == cudaSuccess; k++) {
        if (!hm[k]) continue;
        e = cudaMallocAsync(&dm[k], bytes, st);
        if (e == cudaSuccess)
            e = cudaMemcpy2DAsync(dm[k], (size_t)n * sizeof(C), hm[k], (size_t)hl[k] * sizeof(C), (size_t)n * sizeof(C),
                                  n, cudaMemcpyHostToDevice, st);
    }
    int rc = 0;
    if (e == cudaSuccess) {
        // Q and Z are not referenced when not wanted: the kernel gets valid but unused pointers
        rc = tgexc_device<R>(st, wantq, wantz, n, dm[0], n, dm[1], n, dm[2] ? dm[2] : dm[0], n, dm[3] ? dm[3] : dm[0],
                             n, ifst, ilst, info);
        for (int k = 0; k < 4 && rc == 0 && e == cudaSuccess; k++)
            if (hm[k])
                e = cudaMemcpy2DAsync(hm[k], (size_t)hl[k] * sizeof(C), dm[k], (size_t)n * sizeof(C),
                                      (size_t)n * sizeof(C), n, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    }
    for (C *p : dm)
        if (p) cudaFreeAsync(p, st);
    if (st) {
        cudaStreamSynchronize(st);
        cudaStreamDestroy(st);
    }
    if (e != cudaSuccess) {
        set_last_error(std::string("xTGEXC staging: ") + cudaGetErrorString(e));
        *info = 1;
    }
}

// Real pencils, device pointers: as tgexc_device, with IFST in and out as in D/STGEXC (moved to
// the first row of its 2x2 block).  A move whose rows hold only 1x1 blocks runs the rotation
// kernel; when that kernel finds a 2x2 block in the way (status 2, nothing changed) the block
// kernel does the move.
template <class R>
int tgexc_device_real(cudaStream_t st, int wantq, int wantz, int n, R *A, int lda, R *B, int ldb, R *Q, int ldq, R *Z,
                      int ldz, int *ifst, int *ilst, int *info)
{
    set_last_error("");
    *info = tgexc_check(wantq, wantz, n, lda, ldb, ldq, ldz, *ifst, *ilst);
    if (*info) {
        set_last_error("xTGEXC: argument " + std::to_string(-*info) + " has an illegal value");
        return 0;
    }
    if (n <= 1) return 0;  // IFST = ILST still runs: LAPACK moves both to their blocks' first rows
    int *d_status = nullptr;
    int h_status[3] = {0, 0, 0};
    cudaError_t e = cudaMallocAsync(&d_status, 3 * sizeof(int), st);
    bool blocks = false;
    if (e == cudaSuccess) {
        ReorderArgsReal<R> ra{n, *ifst - 1, *ilst - 1, wantq ? 1 : 0, wantz ? 1 : 0, A, B, Q, Z, lda, ldb, ldq, ldz,
                              d_status};
        tgexc_real_kernel<R><<<1, kReorderThreads, 0, st>>>(ra);
        count_launches(1);
        e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaMemcpyAsync(h_status, d_status, 2 * sizeof(int), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e == cudaSuccess && h_status[1] == 2) {
            blocks = true;
            rb::Pencil<R> p{n, wantq ? 1 : 0, wantz ? 1 : 0, A, B, Q, Z, lda, ldb, ldq, ldz};
            tgexc_real_blocks_kernel<R><<<1, kReorderThreads, 0, st>>>(p, *ifst, *ilst, d_status);
            count_launches(1);
            e = cudaGetLastError();
            if (e == cudaSuccess) e = cudaMemcpyAsync(h_status, d_status, sizeof(h_status), cudaMemcpyDeviceToHost, st);
            if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        }
        cudaFreeAsync(d_status, st);
    }
    if (e != cudaSuccess) {
        set_last_error(std::string("xTGEXC: ") + cudaGetErrorString(e));
        *info = 1;
        return 1;
    }
    if (!blocks) {
        *info = h_status[1];
        *ilst = h_status[0] + 1;
        return 0;
    }
    if (h_status[1] == 3) {
        set_last_error("xTGEXC (real): the block walk did not end within its swap bound");
        *info = 1;
        return 1;
    }
    *info = h_status[1];
    *ilst = h_status[0];
    *ifst = h_status[2];
    return 0;
}

// Real pencils, host pointers: as tgexc_host.
template <class R>
void tgexc_host_real(int wantq, int wantz, int n, R *A, int lda, R *B, int ldb, R *Q, int ldq, R *Z, int ldz, int *ifst,
                     int *ilst, int *info)
{
    set_last_error("");
    *info = tgexc_check(wantq, wantz, n, lda, ldb, ldq, ldz, *ifst, *ilst);
    if (*info) {
        set_last_error("xTGEXC: argument " + std::to_string(-*info) + " has an illegal value");
        return;
    }
    if (n <= 1) return;
    cudaStream_t st = nullptr;
    R *dm[4] = {nullptr, nullptr, nullptr, nullptr};
    R *hm[4] = {A, B, wantq ? Q : nullptr, wantz ? Z : nullptr};
    const int hl[4] = {lda, ldb, ldq, ldz};
    const size_t bytes = (size_t)n * n * sizeof(R);
    cudaError_t e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
    for (int k = 0; k < 4 && e == cudaSuccess; k++) {
        if (!hm[k]) continue;
        e = cudaMallocAsync(&dm[k], bytes, st);
        if (e == cudaSuccess)
            e = cudaMemcpy2DAsync(dm[k], (size_t)n * sizeof(R), hm[k], (size_t)hl[k] * sizeof(R), (size_t)n * sizeof(R),
                                  n, cudaMemcpyHostToDevice, st);
    }
    int rc = 0;
    if (e == cudaSuccess) {
        rc = tgexc_device_real<R>(st, wantq, wantz, n, dm[0], n, dm[1], n, dm[2] ? dm[2] : dm[0], n,
                                  dm[3] ? dm[3] : dm[0], n, ifst, ilst, info);
        for (int k = 0; k < 4 && rc == 0 && e == cudaSuccess; k++)
            if (hm[k])
                e = cudaMemcpy2DAsync(hm[k], (size_t)hl[k] * sizeof(R), dm[k], (size_t)n * sizeof(R),
                                      (size_t)n * sizeof(R), n, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    }
    for (R *p : dm)
        if (p) cudaFreeAsync(p, st);
    if (st) {
        cudaStreamSynchronize(st);
        cudaStreamDestroy(st);
    }
    if (e != cudaSuccess) {
        set_last_error(std::string("xTGEXC staging: ") + cudaGetErrorString(e));
        *info = 1;
    }
}

}  // namespace
}  // namespace xtg

using xtg::cplx;

extern "C" {

void xtgevc3_ztgexc(int wantq, int wantz, int n, double *A, int lda, double *B, int ldb, double *Q, int ldq, double *Z,
                    int ldz, int ifst, int *ilst, int *info)
{
    xtg::tgexc_host<double>(wantq, wantz, n, reinterpret_cast<cplx<double> *>(A), lda, reinterpret_cast<cplx<double> *>(B),
                            ldb, reinterpret_cast<cplx<double> *>(Q), ldq, reinterpret_cast<cplx<double> *>(Z), ldz, ifst,
                            ilst, info);
}

void xtgevc3_ctgexc(int wantq, int wantz, int n, float *A, int lda, float *B, int ldb, float *Q, int ldq, float *Z,
                    int ldz, int ifst, int *ilst, int *info)
{
    xtg::tgexc_host<float>(wantq, wantz, n, reinterpret_cast<cplx<float> *>(A), lda, reinterpret_cast<cplx<float> *>(B),
                           ldb, reinterpret_cast<cplx<float> *>(Q), ldq, reinterpret_cast<cplx<float> *>(Z), ldz, ifst,
                           ilst, info);
}

int xtgevc3_ztgexc_dev(void *stream, int wantq, int wantz, int n, double *A, int lda, double *B, int ldb, double *Q,
                       int ldq, double *Z, int ldz, int ifst, int *ilst, int *info)
{
    return xtg::tgexc_device<double>(static_cast<cudaStream_t>(stream), wantq, wantz, n,
                                     reinterpret_cast<cplx<double> *>(A), lda, reinterpret_cast<cplx<double> *>(B), ldb,
                                     reinterpret_cast<cplx<double> *>(Q), ldq, reinterpret_cast<cplx<double> *>(Z), ldz,
                                     ifst, ilst, info);
}

int xtgevc3_ctgexc_dev(void *stream, int wantq, int wantz, int n, float *A, int lda, float *B, int ldb, float *Q,
                       int ldq, float *Z, int ldz, int ifst, int *ilst, int *info)
{
    return xtg::tgexc_device<float>(static_cast<cudaStream_t>(stream), wantq, wantz, n,
                                    reinterpret_cast<cplx<float> *>(A), lda, reinterpret_cast<cplx<float> *>(B), ldb,
                                    reinterpret_cast<cplx<float> *>(Q), ldq, reinterpret_cast<cplx<float> *>(Z), ldz, ifst,
                                    ilst, info);
}

void xtgevc3_dtgexc(int wantq, int wantz, int n, double *A, int lda, double *B, int ldb, double *Q, int ldq, double *Z,
                    int ldz, int *ifst, int *ilst, int *info)
{
    xtg::tgexc_host_real<double>(wantq, wantz, n, A, lda, B, ldb, Q, ldq, Z, ldz, ifst, ilst, info);
}

void xtgevc3_stgexc(int wantq, int wantz, int n, float *A, int lda, float *B, int ldb, float *Q, int ldq, float *Z,
                    int ldz, int *ifst, int *ilst, int *info)
{
    xtg::tgexc_host_real<float>(wantq, wantz, n, A, lda, B, ldb, Q, ldq, Z, ldz, ifst, ilst, info);
}

int xtgevc3_dtgexc_dev(void *stream, int wantq, int wantz, int n, double *A, int lda, double *B, int ldb, double *Q,
                       int ldq, double *Z, int ldz, int *ifst, int *ilst, int *info)
{
    return xtg::tgexc_device_real<double>(static_cast<cudaStream_t>(stream), wantq, wantz, n, A, lda, B, ldb, Q, ldq, Z,
                                          ldz, ifst, ilst, info);
}

int xtgevc3_stgexc_dev(void *stream, int wantq, int wantz, int n, float *A, int lda, float *B, int ldb, float *Q,
                       int ldq, float *Z, int ldz, int *ifst, int *ilst, int *info)
{
    return xtg::tgexc_device_real<float>(static_cast<cudaStream_t>(stream), wantq, wantz, n, A, lda, B, ldb, Q, ldq, Z,
                                         ldz, ifst, ilst, info);
}

}  // extern "C"
