// The generalized Schur form of a complex pencil (LAPACK ZGGES / CGGES without ordering):
// unitary Q, Z with A = Q S Z^H, B = Q T Z^H, S and T upper triangular, T's diagonal real and
// non-negative, alpha = diag(S), beta = diag(T).  Three stages, each a chain of plane
// rotations (ZLARTG's convention: real cosine c >= 0, [c s; -conj(s) c] [f; g] = [r; 0]):
//   1. B upper triangular: rotations of adjacent rows, column by column from the bottom;
//   2. A upper Hessenberg with B kept triangular (ZGGHRD): a row rotation zeroes A(i, j), a
//      column rotation then zeroes the entry it made below B's diagonal;
//   3. single-shift QZ iterations (ZHGEQZ's steps for the full Schur form): deflation where a
//      subdiagonal entry of the Hessenberg matrix is negligible against its diagonal
//      neighbours, infinite eigenvalues (a negligible diagonal entry of T) split off at the top
//      or chased to the bottom, the Wilkinson shift from the trailing 2 x 2 pencil (an
//      exceptional shift every tenth iteration), the bulge chased by row and column
//      rotations; each deflated eigenvalue's T entry made real and non-negative.  At most
//      30 n iterations; INFO = (index of the last undeflated eigenvalue) + 1 past that.
//
// One CTA: every thread evaluates the same decisions and rotations from memory between
// barriers (the values are identical on all threads), the CTA applies each rotation to its
// O(n) rows or columns, thread 0 writes the single entries a rotation sets.  Written against
// a CTA context (tgexc_real_blocks.cuh's CtaDev on the GPU, host threads with a barrier in the
// tests).  Host and device code.
#pragma once

#include "tgsna_dif_cplx.cuh"

namespace xtg {
namespace rb {

template <class R>
XTG_HD inline R abs1(zc<R> a) { return xabs(a.re) + xabs(a.im); }

// principal square root
template <class R>
XTG_HD inline zc<R> csqrt_(zc<R> z)
{
    const R r = cabs(z);
    if (r == R(0)) return mk(R(0), R(0));
    const R t = xsqrt((r + xabs(z.re)) / R(2));
    if (z.re >= R(0)) return mk(t, z.im / (R(2) * t));
    return mk(xabs(z.im) / (R(2) * t), xsign(t, z.im));
}

// ZLARTG: [c s; -conj(s) c] [f; g] = [r; 0], c real >= 0
template <class R>
XTG_HD void zlartg(zc<R> f, zc<R> g, R &c, zc<R> &s, zc<R> &r)
{
    if (zero(g)) {
        c = R(1);
        s = mk(R(0), R(0));
        r = f;
        return;
    }
    if (zero(f)) {
        const R ga = cabs(g);
        c = R(0);
        s = mk(g.re / ga, -g.im / ga);
        r = mk(ga, R(0));
        return;
    }
    const R fa = cabs(f), ga = cabs(g), h = xhypot(fa, ga);
    c = fa / h;
    const zc<R> u = mk(f.re / fa, f.im / fa);  // f / |f|
    s = (R(1) / h) * (conj(g) * u);
    r = h * u;
}

template <class R>
struct QzPencil {
    int n, wantq, wantz;
    zc<R> *A, *B, *Q, *Z;
    int lda, ldb, ldq, ldz;
};

// Rotation of rows (i, i + 1), (x, y) <- (c x + s y, c y - conj(s) x), over columns [a0, n)
// of A and [b0, n) of B; Q's columns (i, i + 1) take (c, conj(s)) (A = Q S Z^H kept).
template <class R>
XTG_HD void qz_rows(const QzPencil<R> &p, int i, int a0, int b0, R c, zc<R> s, int tid, int nth)
{
    const int n = p.n, na = n - a0, nb = n - b0, nq = p.wantq ? n : 0;
    for (int e = tid; e < na + nb + nq; e += nth) {
        if (e < na) {
            zc<R> &x = p.A[i + (size_t)(a0 + e) * p.lda];
            zc<R> &y = p.A[i + 1 + (size_t)(a0 + e) * p.lda];
            zrot(x, y, c, s);
        } else if (e < na + nb) {
            const int col = b0 + e - na;
            zrot(p.B[i + (size_t)col * p.ldb], p.B[i + 1 + (size_t)col * p.ldb], c, s);
        } else {
            const int r = e - na - nb;
            zrot(p.Q[r + (size_t)i * p.ldq], p.Q[r + (size_t)(i + 1) * p.ldq], c, conj(s));
        }
    }
}

// Rotation of columns (j, j - 1) as (x, y) = (column j, column j - 1) <- (c x + s y, c y -
// conj(s) x), over rows [0, ra) of A and [0, rb) of B, and Z's columns (j, j - 1).
template <class R>
XTG_HD void qz_cols(const QzPencil<R> &p, int j, int ra, int rb, R c, zc<R> s, int tid, int nth)
{
    const int n = p.n, nz = p.wantz ? n : 0;
    for (int e = tid; e < ra + rb + nz; e += nth) {
        if (e < ra) {
            zrot(p.A[e + (size_t)j * p.lda], p.A[e + (size_t)(j - 1) * p.lda], c, s);
        } else if (e < ra + rb) {
            const int r = e - ra;
            zrot(p.B[r + (size_t)j * p.ldb], p.B[r + (size_t)(j - 1) * p.ldb], c, s);
        } else {
            const int r = e - ra - rb;
            zrot(p.Z[r + (size_t)j * p.ldz], p.Z[r + (size_t)(j - 1) * p.ldz], c, s);
        }
    }
}

// The Wilkinson shift of the trailing 2 x 2 pencil at ilast (ZHGEQZ's formula)
template <class R>
XTG_HD zc<R> qz_shift(const QzPencil<R> &p, int il, R ascale, R bscale)
{
    auto A = [&](int i, int j) { return p.A[i + (size_t)j * p.lda]; };
    auto B = [&](int i, int j) { return p.B[i + (size_t)j * p.ldb]; };
    const zc<R> u12 = cdiv(bscale * B(il - 1, il), bscale * B(il, il));
    const zc<R> ad11 = cdiv(ascale * A(il - 1, il - 1), bscale * B(il - 1, il - 1));
    const zc<R> ad21 = cdiv(ascale * A(il, il - 1), bscale * B(il - 1, il - 1));
    const zc<R> ad12 = cdiv(ascale * A(il - 1, il), bscale * B(il, il));
    const zc<R> ad22 = cdiv(ascale * A(il, il), bscale * B(il, il));
    const zc<R> abi22 = ad22 - u12 * ad21, abi12 = ad12 - u12 * ad11;
    zc<R> shift = abi22;
    const zc<R> ctemp = csqrt_(abi12) * csqrt_(ad21);
    if (!zero(ctemp)) {
        const zc<R> x = R(0.5) * (ad11 - shift);
        const R temp2 = abs1(x), temp = xmax(abs1(ctemp), temp2);
        const zc<R> xt = mk(x.re / temp, x.im / temp), ct = mk(ctemp.re / temp, ctemp.im / temp);
        zc<R> y = temp * csqrt_(xt * xt + ct * ct);
        if (temp2 > R(0)) {
            const zc<R> xs = mk(x.re / temp2, x.im / temp2);
            if (xs.re * y.re + xs.im * y.im < R(0)) y = -y;
        }
        shift = shift - ctemp * cdiv(ctemp, x + y);
    }
    return shift;
}

// The generalized Schur form of the complex pencil (p.A, p.B) in place on one CTA, Q and Z
// accumulated from the identity when wanted.  Returns INFO (0, or the index + 1 of the last
// eigenvalue not deflated within 30 n QZ iterations).
template <class R, class Cta>
XTG_HD int zgges_cta(const Cta &c, const QzPencil<R> &p)
{
    const int n = p.n, tid = c.tid(), nth = c.nth();
    auto A = [&](int i, int j) -> zc<R> & { return p.A[i + (size_t)j * p.lda]; };
    auto B = [&](int i, int j) -> zc<R> & { return p.B[i + (size_t)j * p.ldb]; };
    const zc<R> zero_ = mk(R(0), R(0)), one = mk(R(1), R(0));
    for (int e = tid; e < n * n; e += nth) {
        const int i = e % n, j = e / n;
        if (p.wantq) p.Q[i + (size_t)j * p.ldq] = i == j ? one : zero_;
        if (p.wantz) p.Z[i + (size_t)j * p.ldz] = i == j ? one : zero_;
    }
    R cs;
    zc<R> sn, r;
    // 1. B upper triangular
    for (int j = 0; j + 1 < n; j++)
        for (int i = n - 1; i > j; i--) {
            c.sync();
            if (zero(B(i, j))) continue;  // the same decision on every thread
            zlartg(B(i - 1, j), B(i, j), cs, sn, r);
            c.sync();
            qz_rows(p, i - 1, 0, j + 1, cs, sn, tid, nth);
            if (tid == 0) {
                B(i - 1, j) = r;
                B(i, j) = zero_;
            }
        }
    // 2. A upper Hessenberg, B upper triangular (ZGGHRD)
    for (int jcol = 0; jcol + 2 < n; jcol++)
        for (int jrow = n - 1; jrow >= jcol + 2; jrow--) {
            c.sync();
            zlartg(A(jrow - 1, jcol), A(jrow, jcol), cs, sn, r);
            c.sync();
            qz_rows(p, jrow - 1, jcol + 1, jrow - 1, cs, sn, tid, nth);
            if (tid == 0) {
                A(jrow - 1, jcol) = r;
                A(jrow, jcol) = zero_;
            }
            c.sync();
            zlartg(B(jrow, jrow), B(jrow, jrow - 1), cs, sn, r);
            c.sync();
            qz_cols(p, jrow, n, jrow, cs, sn, tid, nth);
            if (tid == 0) {
                B(jrow, jrow) = r;
                B(jrow, jrow - 1) = zero_;
            }
        }
    // 3. QZ iterations (ZHGEQZ, full Schur form)
    c.sync();
    R as = R(0), aq = R(1), bs = R(0), bq = R(1);
    for (int j = 0; j < n; j++) {
        for (int i = 0; i <= j + 1 && i < n; i++) {
            const R v[2] = {A(i, j).re, A(i, j).im};
            lassq(2, v, as, aq);
        }
        for (int i = 0; i <= j; i++) {
            const R v[2] = {B(i, j).re, B(i, j).im};
            lassq(2, v, bs, bq);
        }
    }
    const R anorm = as * xsqrt(aq), bnorm = bs * xsqrt(bq);
    const R safmin = Mach<R>::sfmin, ulp = Mach<R>::prec;
    const R atol = xmax(safmin, ulp * anorm), btol = xmax(safmin, ulp * bnorm);
    const R ascale = R(1) / xmax(safmin, anorm), bscale = R(1) / xmax(safmin, bnorm);
    auto small_sub = [&](int j) {  // A(j, j - 1) negligible
        return abs1(A(j, j - 1)) <= xmax(safmin, ulp * (abs1(A(j, j)) + abs1(A(j - 1, j - 1))));
    };
    int ilast = n - 1, iiter = 0, info = 0;
    zc<R> eshift = zero_;
    const int maxit = 30 * n;
    for (int jiter = 0; ilast >= 0; jiter++) {
        if (jiter >= maxit) {
            info = ilast + 1;
            break;
        }
        c.sync();
        // decide: 0 deflate ilast, 1 infinite eigenvalue at the bottom, 2 split a zero of T off
        // at the top (from j), 3 chase a zero of T down (from j), 4 a QZ sweep from ifirst
        int action = 4, j = 0, ifirst = 0;
        bool zero_sub_last = false, zero_b_last = false, zero_sub_j = false, zero_b_j = false, ilazr2 = false;
        if (ilast == 0) {
            action = 0;
        } else if (small_sub(ilast)) {
            action = 0;
            zero_sub_last = true;
        } else if (cabs(B(ilast, ilast)) <= btol) {
            action = 1;
            zero_b_last = true;
        } else {
            for (j = ilast - 1; j >= 0; j--) {
                bool ilazro = j == 0;
                if (!ilazro && small_sub(j)) {
                    ilazro = true;
                    zero_sub_j = true;
                }
                if (cabs(B(j, j)) < btol) {
                    zero_b_j = true;
                    if (!ilazro)
                        ilazr2 = abs1(A(j, j - 1)) * (ascale * abs1(A(j + 1, j))) <= abs1(A(j, j)) * (ascale * atol);
                    action = (ilazro || ilazr2) ? 2 : 3;
                    break;
                }
                if (ilazro) {
                    action = 4;
                    ifirst = j;
                    break;
                }
            }
        }
        c.sync();  // every thread has decided before entries change
        if (tid == 0) {
            if (zero_sub_last) A(ilast, ilast - 1) = zero_;
            if (zero_b_last) B(ilast, ilast) = zero_;
            if (zero_sub_j) A(j, j - 1) = zero_;
            if (zero_b_j) B(j, j) = zero_;
        }
        bool inf_bottom = action == 1, deflate = action == 0;
        if (action == 2) {  // split the zero of T off at the top of the block, row by row
            bool done = false;
            for (int jch = j; jch < ilast && !done; jch++) {
                c.sync();
                zlartg(A(jch, jch), A(jch + 1, jch), cs, sn, r);
                c.sync();
                qz_rows(p, jch, jch + 1, jch + 1, cs, sn, tid, nth);
                if (tid == 0) {
                    A(jch, jch) = r;
                    A(jch + 1, jch) = zero_;
                    if (ilazr2) A(jch, jch - 1) = cs * A(jch, jch - 1);
                }
                ilazr2 = false;
                c.sync();
                const bool nonzero = abs1(B(jch + 1, jch + 1)) >= btol;
                c.sync();
                if (nonzero) {
                    if (jch + 1 >= ilast) deflate = true;
                    else ifirst = jch + 1;
                    done = true;
                    action = jch + 1 >= ilast ? 0 : 4;
                } else if (tid == 0) {
                    B(jch + 1, jch + 1) = zero_;
                }
            }
            if (!done) inf_bottom = true;
        } else if (action == 3) {  // chase the zero of T to the bottom
            for (int jch = j; jch < ilast; jch++) {
                c.sync();
                zlartg(B(jch, jch + 1), B(jch + 1, jch + 1), cs, sn, r);
                c.sync();
                qz_rows(p, jch, jch - 1, jch + 2, cs, sn, tid, nth);
                if (tid == 0) {
                    B(jch, jch + 1) = r;
                    B(jch + 1, jch + 1) = zero_;
                }
                c.sync();
                zlartg(A(jch + 1, jch), A(jch + 1, jch - 1), cs, sn, r);
                c.sync();
                qz_cols(p, jch, jch + 1, jch, cs, sn, tid, nth);
                if (tid == 0) {
                    A(jch + 1, jch) = r;
                    A(jch + 1, jch - 1) = zero_;
                }
            }
            inf_bottom = true;
        }
        if (inf_bottom) {  // T(ilast, ilast) = 0: a column rotation zeroes A(ilast, ilast - 1)
            c.sync();
            zlartg(A(ilast, ilast), A(ilast, ilast - 1), cs, sn, r);
            c.sync();
            qz_cols(p, ilast, ilast, ilast, cs, sn, tid, nth);
            if (tid == 0) {
                A(ilast, ilast) = r;
                A(ilast, ilast - 1) = zero_;
            }
            deflate = true;
        }
        if (deflate) {  // eigenvalue ilast found: T(ilast, ilast) made real and non-negative
            c.sync();
            const zc<R> b = B(ilast, ilast);
            const R absb = cabs(b);
            c.sync();
            if (absb > safmin) {
                const zc<R> sg = conj(mk(b.re / absb, b.im / absb));
                const int nz = p.wantz ? n : 0;
                for (int e = tid; e < (ilast + 1) + ilast + nz; e += nth) {
                    if (e <= ilast) A(e, ilast) = A(e, ilast) * sg;
                    else if (e < 2 * ilast + 1) B(e - ilast - 1, ilast) = B(e - ilast - 1, ilast) * sg;
                    else p.Z[(e - 2 * ilast - 1) + (size_t)ilast * p.ldz] = p.Z[(e - 2 * ilast - 1) + (size_t)ilast * p.ldz] * sg;
                }
                if (tid == 0) B(ilast, ilast) = mk(absb, R(0));
            } else if (tid == 0) {
                B(ilast, ilast) = zero_;
            }
            ilast--;
            iiter = 0;
            eshift = zero_;
            continue;
        }
        if (action != 4) continue;
        // a single-shift QZ sweep over [ifirst, ilast]
        iiter++;
        c.sync();
        zc<R> shift;
        if (iiter % 10 != 0) {
            shift = qz_shift(p, ilast, ascale, bscale);
        } else {  // exceptional shift
            if (iiter % 20 == 0 && bscale * abs1(B(ilast, ilast)) > safmin)
                eshift = eshift + cdiv(ascale * A(ilast, ilast), bscale * B(ilast, ilast));
            else
                eshift = eshift + cdiv(ascale * A(ilast, ilast - 1), bscale * B(ilast - 1, ilast - 1));
            shift = eshift;
        }
        zlartg(ascale * A(ifirst, ifirst) - shift * (bscale * B(ifirst, ifirst)), ascale * A(ifirst + 1, ifirst), cs, sn,
               r);
        for (int jj = ifirst; jj < ilast; jj++) {
            if (jj > ifirst) {
                c.sync();
                zlartg(A(jj, jj - 1), A(jj + 1, jj - 1), cs, sn, r);
            }
            c.sync();
            qz_rows(p, jj, jj, jj, cs, sn, tid, nth);
            if (tid == 0 && jj > ifirst) {
                A(jj, jj - 1) = r;
                A(jj + 1, jj - 1) = zero_;
            }
            c.sync();
            zlartg(B(jj + 1, jj + 1), B(jj + 1, jj), cs, sn, r);
            c.sync();
            qz_cols(p, jj + 1, (jj + 2 < ilast ? jj + 2 : ilast) + 1, jj + 1, cs, sn, tid, nth);
            if (tid == 0) {
                B(jj + 1, jj + 1) = r;
                B(jj + 1, jj) = zero_;
            }
        }
    }
    c.sync();
    return info;
}

}  // namespace rb
}  // namespace xtg
