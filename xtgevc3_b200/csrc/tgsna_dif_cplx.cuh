// DIF of LAPACK Z/CTGSNA (JOB = 'V' / 'B'): the complex counterpart of tgsna_dif.cuh.  For a
// complex generalized Schur pencil (A, B) (both upper triangular) and a selected eigenvalue k:
//   1. a copy of (A, B) with eigenvalue k moved to the top by swaps of adjacent diagonal
//      entries (ZTGEXC / ZTGEX2: two rotations with real cosines per swap, weak and strong
//      tests; a rejected swap gives DIF = 0);
//   2. ZTGSYL's Frobenius-norm estimate (IJOB = 3) for the Sylvester operator
//      (R, L) -> (A22 R - L a11, B22 R - L b11) of the rest of the pencil: ZTGSYL's blocks of
//      A22 (ILAENV's 2 rows, the last block to the end), inside each ZTGSY2's substitution over
//      the diagonal entries, bottom to top, each a 2 x 2 complex system (ZGETC2) solved by
//      ZLATDF for the current residual plus +-1 entries chosen by look-ahead, then the rows
//      above take the solution; DIF = sqrt(2 n2) / ||all solutions||_F;
//   3. n = 1: DIF = |(|a11|, |b11|)|.
// The swaps' rotations are LAPACK's (no sign freedom), so DIF agrees with LAPACK's to rounding
// unless a look-ahead choice is a near tie.
//
// Host and device code: the GPU kernel (tgsna_dif.cu) runs one CTA per eigenvalue, the tests
// compile this header for the CPU and compare with LAPACK.
#pragma once

#include "tgsna_dif.cuh"

namespace xtg {
namespace rb {

// complex number as two reals (re, im), laid out as LAPACK's COMPLEX / COMPLEX*16
template <class R>
struct zc {
    R re, im;
};
template <class R>
XTG_HD inline zc<R> mk(R a, R b) { return zc<R>{a, b}; }
template <class R>
XTG_HD inline zc<R> operator+(zc<R> a, zc<R> b) { return {a.re + b.re, a.im + b.im}; }
template <class R>
XTG_HD inline zc<R> operator-(zc<R> a, zc<R> b) { return {a.re - b.re, a.im - b.im}; }
template <class R>
XTG_HD inline zc<R> operator-(zc<R> a) { return {-a.re, -a.im}; }
template <class R>
XTG_HD inline zc<R> operator*(zc<R> a, zc<R> b) { return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; }
template <class R>
XTG_HD inline zc<R> operator*(R s, zc<R> a) { return {s * a.re, s * a.im}; }
template <class R>
XTG_HD inline zc<R> conj(zc<R> a) { return {a.re, -a.im}; }
template <class R>
XTG_HD inline R cabs(zc<R> a) { return xhypot(a.re, a.im); }
template <class R>
XTG_HD inline bool zero(zc<R> a) { return a.re == R(0) && a.im == R(0); }
template <class R>
XTG_HD inline bool finite(zc<R> a) { return xfinite(a.re) && xfinite(a.im); }
// a / b by Smith's method (scaled by the larger component of b)
template <class R>
XTG_HD inline zc<R> cdiv(zc<R> a, zc<R> b)
{
    if (xabs(b.re) >= xabs(b.im)) {
        const R r = b.im / b.re, d = b.re + b.im * r;
        return {(a.re + a.im * r) / d, (a.im - a.re * r) / d};
    }
    const R r = b.re / b.im, d = b.im + b.re * r;
    return {(a.re * r + a.im) / d, (a.im * r - a.re) / d};
}
// product and difference rounded term by term (no fused multiply-add), as LAPACK forms the
// swap's f and g
template <class R>
XTG_HD inline zc<R> mul_sep(zc<R> a, zc<R> b)
{
    return {sub_rn(mul_rn(a.re, b.re), mul_rn(a.im, b.im)), mul_rn(a.re, b.im) + mul_rn(a.im, b.re)};
}

// Rotation with real cosine c >= 0: [c s; -conj(s) c] [f; g] = [r; 0] (ZLARTG's convention)
template <class R>
XTG_HD void zgivens(zc<R> f, zc<R> g, R &c, zc<R> &s)
{
    if (zero(g)) {
        c = R(1);
        s = mk(R(0), R(0));
        return;
    }
    if (zero(f)) {
        const R ga = cabs(g);
        c = R(0);
        s = mk(g.re / ga, -g.im / ga);
        return;
    }
    const R fa = cabs(f), ga = cabs(g), h = xhypot(fa, ga);
    c = fa / h;
    const zc<R> u = mk(f.re / fa, f.im / fa);
    s = (R(1) / h) * (conj(g) * u);
}

// (x, y) <- (c x + s y, c y - conj(s) x)
template <class R>
XTG_HD inline void zrot(zc<R> &x, zc<R> &y, R c, zc<R> s)
{
    const zc<R> xn = c * x + s * y, yn = c * y - conj(s) * x;
    x = xn;
    y = yn;
}

template <class R>
XTG_HD inline R zfnorm2(zc<R> a, zc<R> b, zc<R> c, zc<R> d)
{
    return xhypot(xhypot(cabs(a), cabs(b)), xhypot(cabs(c), cabs(d)));
}

// One complex swap of rows / columns (j, j + 1) from the 2x2 blocks (ZTGEX2): the column
// rotation (cz, szc) and the row rotation (cq, sq), applied as zrot; false when the swap
// fails the weak or the strong test.
template <class R>
XTG_HD bool zswap11(zc<R> a00, zc<R> a10, zc<R> a01, zc<R> a11, zc<R> b00, zc<R> b10, zc<R> b01, zc<R> b11, R &cz,
                    zc<R> &szc, R &cq, zc<R> &sq)
{
    const R eps = Mach<R>::prec, smlnum = Mach<R>::sfmin / eps;
    const R tha = xmax(R(20) * eps * zfnorm2(a00, a10, a01, a11), smlnum);
    const R thb = xmax(R(20) * eps * zfnorm2(b00, b10, b01, b11), smlnum);
    const zc<R> f = mul_sep(a11, b00) - mul_sep(b11, a00);
    const zc<R> g = mul_sep(a11, b01) - mul_sep(b11, a01);
    const R sa = cabs(a11) * cabs(b00), sb = cabs(a00) * cabs(b11);
    zc<R> sz;
    zgivens(g, f, cz, sz);
    szc = conj(-sz);
    zc<R> s00 = a00, s01 = a01, s10 = a10, s11 = a11, t00 = b00, t01 = b01, t10 = b10, t11 = b11;
    zrot(s00, s01, cz, szc);
    zrot(s10, s11, cz, szc);
    zrot(t00, t01, cz, szc);
    zrot(t10, t11, cz, szc);
    if (sa >= sb) zgivens(s00, s10, cq, sq);
    else zgivens(t00, t10, cq, sq);
    zrot(s00, s10, cq, sq);
    zrot(s01, s11, cq, sq);
    zrot(t00, t10, cq, sq);
    zrot(t01, t11, cq, sq);
    bool ok = cabs(s10) <= tha && cabs(t10) <= thb && xfinite(cz) && xfinite(cq) && finite(szc) && finite(sq) &&
              finite(s00) && finite(s01) && finite(s11) && finite(t00) && finite(t01) && finite(t11);
    if (ok) {  // undo both rotations on the swapped blocks: the originals must come back
        const zc<R> szu = -szc, squ = -sq;
        zc<R> w00 = s00, w01 = s01, w10 = s10, w11 = s11, v00 = t00, v01 = t01, v10 = t10, v11 = t11;
        zrot(w00, w01, cz, szu);
        zrot(w10, w11, cz, szu);
        zrot(v00, v01, cz, szu);
        zrot(v10, v11, cz, szu);
        zrot(w00, w10, cq, squ);
        zrot(w01, w11, cq, squ);
        zrot(v00, v10, cq, squ);
        zrot(v01, v11, cq, squ);
        ok = zfnorm2(w00 - a00, w10 - a10, w01 - a01, w11 - a11) <= tha &&
             zfnorm2(v00 - b00, v10 - b10, v01 - b01, v11 - b11) <= thb;
    }
    return ok;
}

// One complex swap, the state a CTA shares: where (j, 0-based), whether done, the rotations
template <class R>
struct ZSwap {
    int j, ok;
    R cz, cq;
    zc<R> szc, sq;
};

// The swap's arithmetic (one thread); A, B with leading dimension ld
template <class R>
XTG_HD void zswap_prepare(const zc<R> *A, const zc<R> *B, int ld, ZSwap<R> &s)
{
    const int j = s.j;
    auto a = [&](int i, int k) { return A[(size_t)(j + i) + (size_t)(j + k) * ld]; };
    auto b = [&](int i, int k) { return B[(size_t)(j + i) + (size_t)(j + k) * ld]; };
    s.ok = zswap11(a(0, 0), a(1, 0), a(0, 1), a(1, 1), b(0, 0), b(1, 0), b(0, 1), b(1, 1), s.cz, s.szc, s.cq, s.sq) ? 1
                                                                                                                    : 0;
}

// Applying a done swap to A and B (n x n, leading dimension ld) by thread tid of nth:
// phase 0 rotates columns j, j+1 (rows [0, j + 2)), phase 1 (after a barrier) rows j, j+1
// (columns [j, n)), phase 2 (after a barrier, one thread) zeroes the subdiagonal entries.
template <class R>
XTG_HD void zswap_apply(zc<R> *A, zc<R> *B, int n, int ld, const ZSwap<R> &s, int phase, int tid, int nth)
{
    const int j = s.j;
    auto at = [&](zc<R> *M, int i, int k) -> zc<R> & { return M[(size_t)i + (size_t)k * ld]; };
    if (phase == 0) {
        const int r = j + 2;
        for (int i = tid; i < 2 * r; i += nth) {
            zc<R> *M = i < r ? A : B;
            const int row = i < r ? i : i - r;
            zrot(at(M, row, j), at(M, row, j + 1), s.cz, s.szc);
        }
    } else if (phase == 1) {
        const int c = n - j;
        for (int i = tid; i < 2 * c; i += nth) {
            zc<R> *M = i < c ? A : B;
            const int col = j + (i < c ? i : i - c);
            zrot(at(M, j, col), at(M, j + 1, col), s.cq, s.sq);
        }
    } else if (tid == 0) {
        at(A, j + 1, j) = mk(R(0), R(0));
        at(B, j + 1, j) = mk(R(0), R(0));
    }
}

// Sum of squares of the real and imaginary parts (ZLASSQ)
template <class R>
XTG_HD void zlassq(int n, const zc<R> *x, R &scale, R &sumsq)
{
    for (int i = 0; i < n; i++) {
        const R parts[2] = {x[i].re, x[i].im};
        lassq(2, parts, scale, sumsq);
    }
}

// LU with complete pivoting of the 2 x 2 complex matrix Z (column-major), pivots raised to
// smin (ZGETC2).  Returns 0 or the first raised pivot (1-based).
template <class R>
XTG_HD int zgetc2(zc<R> *Z, int *ipiv, int *jpiv)
{
    const int n = 2;
    const R eps = Mach<R>::prec, smlnum = Mach<R>::sfmin / eps;
    int info = 0;
    R smin = R(0);
    for (int i = 0; i < n - 1; i++) {
        R xmx = R(0);
        int ipv = i, jpv = i;
        for (int ip = i; ip < n; ip++)
            for (int jp = i; jp < n; jp++)
                if (cabs(Z[ip + 2 * jp]) >= xmx) {
                    xmx = cabs(Z[ip + 2 * jp]);
                    ipv = ip;
                    jpv = jp;
                }
        if (i == 0) smin = xmax(eps * xmx, smlnum);
        if (ipv != i)
            for (int j = 0; j < n; j++) {
                const zc<R> t = Z[ipv + 2 * j];
                Z[ipv + 2 * j] = Z[i + 2 * j];
                Z[i + 2 * j] = t;
            }
        ipiv[i] = ipv;
        if (jpv != i)
            for (int j = 0; j < n; j++) {
                const zc<R> t = Z[j + 2 * jpv];
                Z[j + 2 * jpv] = Z[j + 2 * i];
                Z[j + 2 * i] = t;
            }
        jpiv[i] = jpv;
        if (cabs(Z[i + 2 * i]) < smin) {
            info = i + 1;
            Z[i + 2 * i] = mk(smin, R(0));
        }
        for (int j = i + 1; j < n; j++) Z[j + 2 * i] = cdiv(Z[j + 2 * i], Z[i + 2 * i]);
        for (int jj = i + 1; jj < n; jj++)
            for (int ii = i + 1; ii < n; ii++) Z[ii + 2 * jj] = Z[ii + 2 * jj] - Z[ii + 2 * i] * Z[i + 2 * jj];
    }
    if (cabs(Z[(n - 1) + 2 * (n - 1)]) < smin) {
        info = n;
        Z[(n - 1) + 2 * (n - 1)] = mk(smin, R(0));
    }
    ipiv[n - 1] = n - 1;
    jpiv[n - 1] = n - 1;
    return info;
}

// ZLATDF with the look-ahead strategy on the 2 x 2 factors of zgetc2: rhs <- the solution for
// rhs + (+-1 entries), its sum of squares added to (rdscal, rdsum)
template <class R>
XTG_HD void zlatdf(const zc<R> *Z, zc<R> *rhs, R &rdsum, R &rdscal, const int *ipiv, const int *jpiv)
{
    const int n = 2;
    const zc<R> one = mk(R(1), R(0));
    for (int i = 0; i < n - 1; i++)
        if (ipiv[i] != i) {
            const zc<R> t = rhs[i];
            rhs[i] = rhs[ipiv[i]];
            rhs[ipiv[i]] = t;
        }
    zc<R> pmone = mk(R(-1), R(0));
    for (int j = 0; j < n - 1; j++) {
        const zc<R> bp = rhs[j] + one, bm = rhs[j] - one;
        R splus = R(1), sminu = R(0);
        for (int k = j + 1; k < n; k++) splus += (conj(Z[k + 2 * j]) * Z[k + 2 * j]).re;
        for (int k = j + 1; k < n; k++) sminu += (conj(Z[k + 2 * j]) * rhs[k]).re;
        splus *= rhs[j].re;
        if (splus > sminu) {
            rhs[j] = bp;
        } else if (sminu > splus) {
            rhs[j] = bm;
        } else {
            rhs[j] = rhs[j] + pmone;
            pmone = one;
        }
        const zc<R> t = -rhs[j];
        for (int k = j + 1; k < n; k++) rhs[k] = rhs[k] + t * Z[k + 2 * j];
    }
    zc<R> xp[2];
    for (int i = 0; i < n - 1; i++) xp[i] = rhs[i];
    xp[n - 1] = rhs[n - 1] + one;
    rhs[n - 1] = rhs[n - 1] - one;
    R splus = R(0), sminu = R(0);
    for (int i = n - 1; i >= 0; i--) {
        const zc<R> t = cdiv(one, Z[i + 2 * i]);
        xp[i] = xp[i] * t;
        rhs[i] = rhs[i] * t;
        for (int k = i + 1; k < n; k++) {
            xp[i] = xp[i] - xp[k] * (Z[i + 2 * k] * t);
            rhs[i] = rhs[i] - rhs[k] * (Z[i + 2 * k] * t);
        }
        splus += cabs(xp[i]);
        sminu += cabs(rhs[i]);
    }
    if (splus > sminu)
        for (int i = 0; i < n; i++) rhs[i] = xp[i];
    for (int i = n - 2; i >= 0; i--)
        if (jpiv[i] != i) {
            const zc<R> t = rhs[i];
            rhs[i] = rhs[jpiv[i]];
            rhs[jpiv[i]] = t;
        }
    zlassq(n, rhs, rdscal, rdsum);
}

// ZTGSYL's operands for the estimate: A22, B22 (n2 x n2, leading dimension ld), a11, b11, the
// right-hand sides C, F (n2 entries each) and the running sum of squares
template <class R>
struct ZSylv {
    int n2, ld;
    const zc<R> *A22, *B22;
    zc<R> a11, b11;
    zc<R> *C, *F;
    R dsum, dscale;
};

// One ZTGSYL block, rows [is, ie] of A22: ZTGSY2 with IJOB = 1 over its diagonal entries,
// bottom to top, the block's own rows above each entry updated.  Returns ZGETC2's INFO.
template <class R>
XTG_HD int ztgsyl_block(ZSylv<R> &y, int is, int ie)
{
    const int ld = y.ld;
    int info = 0;
    for (int i = ie; i >= is; i--) {
        zc<R> Z[4], rhs[2];
        Z[0] = y.A22[(size_t)i + (size_t)i * ld];
        Z[1] = y.B22[(size_t)i + (size_t)i * ld];
        Z[2] = -y.a11;
        Z[3] = -y.b11;
        rhs[0] = y.C[i];
        rhs[1] = y.F[i];
        int ipiv[2], jpiv[2];
        const int ierr = zgetc2(Z, ipiv, jpiv);
        if (ierr > 0) info = ierr;
        zlatdf(Z, rhs, y.dsum, y.dscale, ipiv, jpiv);
        y.C[i] = rhs[0];
        y.F[i] = rhs[1];
        const zc<R> alpha = -rhs[0];
        for (int r = is; r < i; r++) {
            y.C[r] = y.C[r] + alpha * y.A22[(size_t)r + (size_t)i * ld];
            y.F[r] = y.F[r] + alpha * y.B22[(size_t)r + (size_t)i * ld];
        }
    }
    return info;
}

// Rows [0, is) after the block [is, ie]: C -= A22[:, is:ie] R, F -= B22[:, is:ie] R
template <class R>
XTG_HD void ztgsyl_update_above(ZSylv<R> &y, int is, int ie, int tid, int nth)
{
    const int ld = y.ld;
    for (int r = tid; r < is; r += nth) {
        zc<R> c = y.C[r], f = y.F[r];
        for (int p = is; p <= ie; p++) {
            c = c - y.A22[(size_t)r + (size_t)p * ld] * y.C[p];
            f = f - y.B22[(size_t)r + (size_t)p * ld] * y.C[p];
        }
        y.C[r] = c;
        y.F[r] = f;
    }
}

// ZTGSYL's block starts of A22 (2 rows each, the last one to the end); starts[count] = n2
XTG_HD inline int ztgsyl_blocks(int m, int *starts)
{
    if (m <= 2) {
        starts[0] = 0;
        starts[1] = m;
        return 1;
    }
    int p = 0, i = 1;
    while (i <= m) {
        starts[p++] = i - 1;
        i += 2;
        if (i >= m) break;
    }
    starts[p] = m;
    if (starts[p - 1] == starts[p]) p--;
    return p;
}

// DIF from the reordered copy (eigenvalue first; A, B n x n, leading dimension ld) on one
// thread (the tests' CPU build); C, F: n entries each, starts: n / 2 + 2 ints
template <class R>
XTG_HD R zdif_reordered_serial(int n, const zc<R> *A, const zc<R> *B, int ld, zc<R> *C, zc<R> *F, int *starts)
{
    ZSylv<R> y;
    y.n2 = n - 1;
    y.ld = ld;
    y.A22 = A + 1 + (size_t)ld;
    y.B22 = B + 1 + (size_t)ld;
    y.a11 = A[0];
    y.b11 = B[0];
    y.C = C;
    y.F = F;
    for (int i = 0; i < y.n2; i++) C[i] = F[i] = mk(R(0), R(0));
    y.dsum = R(1);
    y.dscale = R(0);
    const int nbk = ztgsyl_blocks(y.n2, starts);
    for (int b = nbk - 1; b >= 0; b--) {
        ztgsyl_block(y, starts[b], starts[b + 1] - 1);
        ztgsyl_update_above(y, starts[b], starts[b + 1] - 1, 0, 1);
    }
    return xsqrt(R(2 * y.n2)) / (y.dscale * xsqrt(y.dsum));
}

// The whole DIF of eigenvalue k (0-based) on one thread: reorder a copy (Aw, Bw: n x n
// scratch, leading dimension n), then the estimate; 0 when a swap is rejected
template <class R>
XTG_HD R zdif_serial(int n, const zc<R> *A, int lda, const zc<R> *B, int ldb, int k, zc<R> *Aw, zc<R> *Bw, zc<R> *C,
                     zc<R> *F, int *starts)
{
    if (n == 1) return lapy2(cabs(A[0]), cabs(B[0]));
    for (int j = 0; j < n; j++)
        for (int i = 0; i < n; i++) {
            Aw[i + (size_t)j * n] = A[i + (size_t)j * lda];
            Bw[i + (size_t)j * n] = B[i + (size_t)j * ldb];
        }
    for (int here = k; here > 0; here--) {
        ZSwap<R> s;
        s.j = here - 1;
        zswap_prepare(Aw, Bw, n, s);
        if (!s.ok) return R(0);
        for (int ph = 0; ph < 3; ph++) zswap_apply(Aw, Bw, n, n, s, ph, 0, 1);
    }
    return zdif_reordered_serial(n, Aw, Bw, n, C, F, starts);
}

// ---- the GPU kernel's body, one CTA (CTA context as for dif_cta in tgsna_dif.cuh) ---------

// workspace of one CTA in complex elements: the copy (2 n^2), C and F (n each), ZTGSYL's block
// starts (n / 2 + 4 ints in n + 8 elements of room)
XTG_HD inline size_t zdif_work_elems(int n) { return 2 * (size_t)n * n + 3 * (size_t)n + 8; }

template <class R>
struct ZDifShared {
    ZSwap<R> s;
    ZSylv<R> y;
    int rej, nbk;
};

// DIF of the items it = c.cta(), c.cta() + c.ncta(), ... of a complex pencil: copy, move the
// eigenvalue up one row per swap (thread 0 computes the rotations, the CTA applies them; at
// most k swaps), ZTGSYL's estimate (thread 0 per block, the CTA updates the rows above).
template <class R, class Cta>
XTG_HD void zdif_cta(const Cta &c, ZDifShared<R> &sh, int n, const zc<R> *A, int lda, const zc<R> *B, int ldb,
                     const DifItem *items, int count, R *dif, zc<R> *work, size_t per_cta)
{
    const int tid = c.tid(), nth = c.nth();
    zc<R> *Aw = work + (size_t)c.cta() * per_cta;
    zc<R> *Bw = Aw + (size_t)n * n;
    zc<R> *Cw = Bw + (size_t)n * n;
    zc<R> *Fw = Cw + n;
    int *starts = reinterpret_cast<int *>(Fw + n);
    for (int it = c.cta(); it < count; it += c.ncta()) {
        const DifItem item = items[it];
        if (n == 1) {
            if (tid == 0) dif[item.ks] = lapy2(cabs(A[0]), cabs(B[0]));
            continue;
        }
        for (size_t e = tid; e < (size_t)n * n; e += nth) {
            const size_t i = e % n, j = e / n;
            Aw[e] = A[i + j * lda];
            Bw[e] = B[i + j * ldb];
        }
        for (int e = tid; e < n; e += nth) {
            Cw[e] = mk(R(0), R(0));
            Fw[e] = mk(R(0), R(0));
        }
        if (tid == 0) sh.rej = 0;
        c.sync();  // the copy is complete before thread 0 reads it
        for (int here = item.k; here > 0; here--) {
            if (tid == 0) {
                sh.s.j = here - 1;
                zswap_prepare(Aw, Bw, n, sh.s);
                sh.rej = sh.s.ok ? 0 : 1;
            }
            c.sync();  // thread 0 writes rej / s again only after this iteration's last barrier
            if (sh.rej) break;
            zswap_apply(Aw, Bw, n, n, sh.s, 0, tid, nth);
            c.sync();  // the 2x2 block takes the column rotation before the row rotation
            zswap_apply(Aw, Bw, n, n, sh.s, 1, tid, nth);
            c.sync();
            zswap_apply(Aw, Bw, n, n, sh.s, 2, tid, nth);
            c.sync();
        }
        c.sync();  // every thread has left the walk
        if (tid == 0) {
            sh.nbk = 0;
            if (!sh.rej) {
                ZSylv<R> &y = sh.y;
                y.n2 = n - 1;
                y.ld = n;
                y.A22 = Aw + 1 + (size_t)n;
                y.B22 = Bw + 1 + (size_t)n;
                y.a11 = Aw[0];
                y.b11 = Bw[0];
                y.C = Cw;
                y.F = Fw;
                y.dsum = R(1);
                y.dscale = R(0);
                sh.nbk = ztgsyl_blocks(n - 1, starts);
            }
        }
        c.sync();
        const int nbk = sh.nbk;
        for (int b = nbk - 1; b >= 0; b--) {
            if (tid == 0) ztgsyl_block(sh.y, starts[b], starts[b + 1] - 1);
            c.sync();
            ztgsyl_update_above(sh.y, starts[b], starts[b + 1] - 1, tid, nth);
            c.sync();
        }
        if (tid == 0)  // a rejected swap: DIF = 0
            dif[item.ks] = nbk > 0 ? xsqrt(R(2 * sh.y.n2)) / (sh.y.dscale * xsqrt(sh.y.dsum)) : R(0);
        c.sync();  // the workspace is reused by the next item
    }
}

}  // namespace rb
}  // namespace xtg
