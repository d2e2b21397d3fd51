// The generalized real Schur form of a real pencil (LAPACK DGGES / SGGES without ordering):
// orthogonal Q, Z with A = Q S Z^T, B = Q T Z^T, S upper quasi-triangular (1x1 blocks and 2x2
// blocks for complex pairs), T upper triangular with non-negative diagonal and each 2x2 block
// of S facing a diagonal block of T with positive entries; alphar, alphai, beta as DHGEQZ
// returns them.  The stages of qz_cplx.cuh in real arithmetic:
//   1. B upper triangular by rotations of adjacent rows;
//   2. the Hessenberg-triangular reduction of DGGHRD;
//   3. QZ iterations with DHGEQZ's steps for the full Schur form: deflation of negligible
//      subdiagonal entries, infinite eigenvalues split off at the top or chased to the bottom,
//      a single real shift when the trailing 2 x 2 pencil has real eigenvalues (xLAG2) and an
//      implicit double shift (3 x 3 reflectors from both sides) when they are complex, an
//      exceptional real shift every tenth iteration; a 2 x 2 block that deflates is
//      standardised by xLAGV2 (two real 1x1 blocks, or a pair with T's block diagonal and
//      positive).  At most 30 n iterations, then INFO = (index of the last undeflated
//      eigenvalue) + 1.
// One CTA, as qz_cplx.cuh: every thread evaluates the same decisions and transforms between
// barriers, the CTA applies them, thread 0 writes single entries.  Host and device code.
#pragma once

#include "qz_cplx.cuh"

namespace xtg {
namespace rb {

template <class R>
struct QzPencilR {
    int n, wantq, wantz;
    R *A, *B, *Q, *Z;
    int lda, ldb, ldq, ldz;
    R *alphar, *alphai, *beta;
};

// sqrt(x^2 + y^2 + z^2) without overflow (xLAPY3)
template <class R>
XTG_HD R lapy3(R x, R y, R z)
{
    const R w = xmax(xmax(xabs(x), xabs(y)), xabs(z));
    if (w == R(0)) return xabs(x) + xabs(y) + xabs(z);
    const R a = x / w, b = y / w, c = z / w;
    return w * xsqrt(a * a + b * b + c * c);
}

// rows (i, i + 1) <- rotation (c, s) as (x, y) <- (c x + s y, c y - s x): A columns [a0, n),
// B columns [b0, n), Q's columns (i, i + 1) with the same rotation
template <class R>
XTG_HD void qzr_rows(const QzPencilR<R> &p, int i, int a0, int b0, R c, R s, int tid, int nth)
{
    const int n = p.n, na = n - a0, nb = n - b0, nq = p.wantq ? n : 0;
    for (int e = tid; e < na + nb + nq; e += nth) {
        if (e < na) rot(p.A[i + (size_t)(a0 + e) * p.lda], p.A[i + 1 + (size_t)(a0 + e) * p.lda], c, s);
        else if (e < na + nb) rot(p.B[i + (size_t)(b0 + e - na) * p.ldb], p.B[i + 1 + (size_t)(b0 + e - na) * p.ldb], c, s);
        else rot(p.Q[(e - na - nb) + (size_t)i * p.ldq], p.Q[(e - na - nb) + (size_t)(i + 1) * p.ldq], c, s);
    }
}

// columns (x, y) = (column j, column j - 1) <- (c x + s y, c y - s x): A rows [0, ra), B rows
// [0, rb), Z's columns (j, j - 1)
template <class R>
XTG_HD void qzr_cols(const QzPencilR<R> &p, int j, int ra, int rb, R c, R s, int tid, int nth)
{
    const int nz = p.wantz ? p.n : 0;
    for (int e = tid; e < ra + rb + nz; e += nth) {
        if (e < ra) rot(p.A[e + (size_t)j * p.lda], p.A[e + (size_t)(j - 1) * p.lda], c, s);
        else if (e < ra + rb) rot(p.B[(e - ra) + (size_t)j * p.ldb], p.B[(e - ra) + (size_t)(j - 1) * p.ldb], c, s);
        else rot(p.Z[(e - ra - rb) + (size_t)j * p.ldz], p.Z[(e - ra - rb) + (size_t)(j - 1) * p.ldz], c, s);
    }
}

// (x0, x1, x2) <- H (x0, x1, x2), H = I - tau v v^T, v = (1, v1, v2)
template <class R>
XTG_HD inline void refl3(R &x0, R &x1, R &x2, R v1, R v2, R tau)
{
    const R t = x0 + v1 * x1 + v2 * x2;
    x0 -= t * tau;
    x1 -= t * (tau * v1);
    x2 -= t * (tau * v2);
}

// rows j .. j+2 <- H rows: A columns [a0, n), B columns [b0, n); Q's columns j .. j+2 <- Q H
template <class R>
XTG_HD void qzr_refl_rows(const QzPencilR<R> &p, int j, int a0, int b0, R v1, R v2, R tau, int tid, int nth)
{
    const int n = p.n, na = n - a0, nb = n - b0, nq = p.wantq ? n : 0;
    for (int e = tid; e < na + nb + nq; e += nth) {
        if (e < na) {
            R *col = p.A + (size_t)(a0 + e) * p.lda;
            refl3(col[j], col[j + 1], col[j + 2], v1, v2, tau);
        } else if (e < na + nb) {
            R *col = p.B + (size_t)(b0 + e - na) * p.ldb;
            refl3(col[j], col[j + 1], col[j + 2], v1, v2, tau);
        } else {
            const int r = e - na - nb;
            refl3(p.Q[r + (size_t)j * p.ldq], p.Q[r + (size_t)(j + 1) * p.ldq], p.Q[r + (size_t)(j + 2) * p.ldq], v1, v2,
                  tau);
        }
    }
}

// columns j .. j+2 <- columns H: A rows [0, ra), B rows [0, rb), Z's columns j .. j+2
template <class R>
XTG_HD void qzr_refl_cols(const QzPencilR<R> &p, int j, int ra, int rb, R v1, R v2, R tau, int tid, int nth)
{
    const int nz = p.wantz ? p.n : 0;
    for (int e = tid; e < ra + rb + nz; e += nth) {
        R *M;
        int ld, r;
        if (e < ra) {
            M = p.A, ld = p.lda, r = e;
        } else if (e < ra + rb) {
            M = p.B, ld = p.ldb, r = e - ra;
        } else {
            M = p.Z, ld = p.ldz, r = e - ra - rb;
        }
        refl3(M[r + (size_t)j * ld], M[r + (size_t)(j + 1) * ld], M[r + (size_t)(j + 2) * ld], v1, v2, tau);
    }
}

// column j negated: A rows [0, ra), B rows [0, rb), Z's column j
template <class R>
XTG_HD void qzr_negate_col(const QzPencilR<R> &p, int j, int ra, int rb, int tid, int nth)
{
    const int nz = p.wantz ? p.n : 0;
    for (int e = tid; e < ra + rb + nz; e += nth) {
        if (e < ra) p.A[e + (size_t)j * p.lda] = -p.A[e + (size_t)j * p.lda];
        else if (e < ra + rb) p.B[(e - ra) + (size_t)j * p.ldb] = -p.B[(e - ra) + (size_t)j * p.ldb];
        else p.Z[(e - ra - rb) + (size_t)j * p.ldz] = -p.Z[(e - ra - rb) + (size_t)j * p.ldz];
    }
}

// alphar, alphai, beta of a standardised 2x2 block (T's block diagonal and positive) with
// complex eigenvalues (DHGEQZ's formulas); false when xLAG2 finds them real after all
template <class R>
XTG_HD bool pair_alphas(const R *a, const R *b, R *ar, R *ai, R *be)
{
    const R safmin = Mach<R>::sfmin;
    R s1, t1_, wr, t2_, wi;
    lag2(a, b, safmin * R(100), s1, t1_, wr, t2_, wi);
    if (wi == R(0)) return false;
    const R s1inv = R(1) / s1;
    const R a11 = a[0], a21 = a[1], a12 = a[LD], a22 = a[1 + LD], b11 = b[0], b22 = b[1 + LD];
    const R c11r = s1 * a11 - wr * b11, c11i = -wi * b11, c12 = s1 * a12, c21 = s1 * a21;
    const R c22r = s1 * a22 - wr * b22, c22i = -wi * b22;
    R cz, szr, szi;
    if (xabs(c11r) + xabs(c11i) + xabs(c12) > xabs(c21) + xabs(c22r) + xabs(c22i)) {
        const R t1 = lapy3(c12, c11r, c11i);
        cz = c12 / t1;
        szr = -c11r / t1;
        szi = -c11i / t1;
    } else {
        cz = lapy2(c22r, c22i);
        if (cz <= safmin) {
            cz = R(0);
            szr = R(1);
            szi = R(0);
        } else {
            const R tr = c22r / cz, ti = c22i / cz, t1 = lapy2(cz, c21);
            cz = cz / t1;
            szr = -c21 * tr / t1;
            szi = c21 * ti / t1;
        }
    }
    const R an = xabs(a11) + xabs(a12) + xabs(a21) + xabs(a22), bn = xabs(b11) + xabs(b22);
    const R wabs = xabs(wr) + xabs(wi);
    R cq, sqr, sqi;
    if (s1 * an > wabs * bn) {
        cq = cz * b11;
        sqr = szr * b22;
        sqi = -szi * b22;
    } else {
        const R a1r = cz * a11 + szr * a12, a1i = szi * a12, a2r = cz * a21 + szr * a22, a2i = szi * a22;
        cq = lapy2(a1r, a1i);
        if (cq <= safmin) {
            cq = R(0);
            sqr = R(1);
            sqi = R(0);
        } else {
            const R tr = a1r / cq, ti = a1i / cq;
            sqr = tr * a2r + ti * a2i;
            sqi = ti * a2r - tr * a2i;
        }
    }
    const R t1 = lapy3(cq, sqr, sqi);
    cq /= t1;
    sqr /= t1;
    sqi /= t1;
    const R tr = sqr * szr - sqi * szi, ti = sqr * szi + sqi * szr;
    const R b1a = lapy2(cq * cz * b11 + tr * b22, ti * b22);
    const R b2a = lapy2(cq * cz * b22 + tr * b11, -ti * b11);
    be[0] = b1a;
    be[1] = b2a;
    ar[0] = (wr * b1a) * s1inv;
    ai[0] = (wi * b1a) * s1inv;
    ar[1] = (wr * b2a) * s1inv;
    ai[1] = -(wi * b2a) * s1inv;
    return true;
}

// The generalized real Schur form of (p.A, p.B) in place on one CTA, Q and Z accumulated from
// the identity when wanted, alphar / alphai / beta written.  Returns INFO.
template <class R, class Cta>
XTG_HD int dgges_cta(const Cta &c, const QzPencilR<R> &p)
{
    const int n = p.n, tid = c.tid(), nth = c.nth();
    auto A = [&](int i, int j) -> R & { return p.A[i + (size_t)j * p.lda]; };
    auto B = [&](int i, int j) -> R & { return p.B[i + (size_t)j * p.ldb]; };
    for (int e = tid; e < n * n; e += nth) {
        const int i = e % n, j = e / n;
        if (p.wantq) p.Q[i + (size_t)j * p.ldq] = i == j ? R(1) : R(0);
        if (p.wantz) p.Z[i + (size_t)j * p.ldz] = i == j ? R(1) : R(0);
    }
    R cs, sn, r;
    // 1. B upper triangular
    for (int j = 0; j + 1 < n; j++)
        for (int i = n - 1; i > j; i--) {
            c.sync();
            if (B(i, j) == R(0)) continue;
            lartg(B(i - 1, j), B(i, j), cs, sn, r);
            c.sync();
            qzr_rows(p, i - 1, 0, j + 1, cs, sn, tid, nth);
            if (tid == 0) {
                B(i - 1, j) = r;
                B(i, j) = R(0);
            }
        }
    // 2. Hessenberg-triangular (DGGHRD)
    for (int jcol = 0; jcol + 2 < n; jcol++)
        for (int jrow = n - 1; jrow >= jcol + 2; jrow--) {
            c.sync();
            lartg(A(jrow - 1, jcol), A(jrow, jcol), cs, sn, r);
            c.sync();
            qzr_rows(p, jrow - 1, jcol + 1, jrow - 1, cs, sn, tid, nth);
            if (tid == 0) {
                A(jrow - 1, jcol) = r;
                A(jrow, jcol) = R(0);
            }
            c.sync();
            lartg(B(jrow, jrow), B(jrow, jrow - 1), cs, sn, r);
            c.sync();
            qzr_cols(p, jrow, n, jrow, cs, sn, tid, nth);
            if (tid == 0) {
                B(jrow, jrow) = r;
                B(jrow, jrow - 1) = R(0);
            }
        }
    // 3. QZ iterations (DHGEQZ, full Schur form)
    c.sync();
    R as = R(0), aq = R(1), bs = R(0), bq = R(1);
    for (int j = 0; j < n; j++) {
        for (int i = 0; i <= j + 1 && i < n; i++) lassq(1, &A(i, j), as, aq);
        for (int i = 0; i <= j; i++) lassq(1, &B(i, j), bs, bq);
    }
    const R anorm = as * xsqrt(aq), bnorm = bs * xsqrt(bq);
    const R safmin = Mach<R>::sfmin, ulp = Mach<R>::prec;
    const R atol = xmax(safmin, ulp * anorm), btol = xmax(safmin, ulp * bnorm);
    const R ascale = R(1) / xmax(safmin, anorm), bscale = R(1) / xmax(safmin, bnorm);
    auto small_sub = [&](int j) {
        return xabs(A(j, j - 1)) <= xmax(safmin, ulp * (xabs(A(j, j)) + xabs(A(j - 1, j - 1))));
    };
    int ilast = n - 1, iiter = 0, info = 0;
    R eshift = R(0);
    const int maxit = 30 * n;
    for (int jiter = 0; ilast >= 0; jiter++) {
        if (jiter >= maxit) {
            info = ilast + 1;
            break;
        }
        c.sync();
        // 0 deflate a 1x1 block, 1 infinite eigenvalue at the bottom, 2 split a zero of T off,
        // 3 chase a zero of T down, 4 iterate on [ifirst, ilast]
        int action = 4, j = 0, ifirst = 0;
        bool zero_sub_last = false, zero_b_last = false, zero_sub_j = false, zero_b_j = false, ilazr2 = false;
        if (ilast == 0) {
            action = 0;
        } else if (small_sub(ilast)) {
            action = 0;
            zero_sub_last = true;
        } else if (xabs(B(ilast, ilast)) <= btol) {
            action = 1;
            zero_b_last = true;
        } else {
            for (j = ilast - 1; j >= 0; j--) {
                bool ilazro = j == 0;
                if (!ilazro && small_sub(j)) {
                    ilazro = true;
                    zero_sub_j = true;
                }
                if (xabs(B(j, j)) < btol) {
                    zero_b_j = true;
                    if (!ilazro)
                        ilazr2 = xabs(A(j, j - 1)) * (ascale * xabs(A(j + 1, j))) <= xabs(A(j, j)) * (ascale * atol);
                    action = (ilazro || ilazr2) ? 2 : 3;
                    break;
                }
                if (ilazro) {
                    ifirst = j;
                    break;
                }
            }
        }
        c.sync();
        if (tid == 0) {
            if (zero_sub_last) A(ilast, ilast - 1) = R(0);
            if (zero_b_last) B(ilast, ilast) = R(0);
            if (zero_sub_j) A(j, j - 1) = R(0);
            if (zero_b_j) B(j, j) = R(0);
        }
        bool inf_bottom = action == 1, deflate = action == 0;
        if (action == 2) {
            bool done = false;
            for (int jch = j; jch < ilast && !done; jch++) {
                c.sync();
                lartg(A(jch, jch), A(jch + 1, jch), cs, sn, r);
                c.sync();
                qzr_rows(p, jch, jch + 1, jch + 1, cs, sn, tid, nth);
                if (tid == 0) {
                    A(jch, jch) = r;
                    A(jch + 1, jch) = R(0);
                    if (ilazr2) A(jch, jch - 1) = cs * A(jch, jch - 1);
                }
                ilazr2 = false;
                c.sync();
                const bool nonzero = xabs(B(jch + 1, jch + 1)) >= btol;
                c.sync();
                if (nonzero) {
                    if (jch + 1 >= ilast) deflate = true;
                    else ifirst = jch + 1;
                    done = true;
                    action = jch + 1 >= ilast ? 0 : 4;
                } else if (tid == 0) {
                    B(jch + 1, jch + 1) = R(0);
                }
            }
            if (!done) inf_bottom = true;
        } else if (action == 3) {
            for (int jch = j; jch < ilast; jch++) {
                c.sync();
                lartg(B(jch, jch + 1), B(jch + 1, jch + 1), cs, sn, r);
                c.sync();
                qzr_rows(p, jch, jch - 1, jch + 2, cs, sn, tid, nth);
                if (tid == 0) {
                    B(jch, jch + 1) = r;
                    B(jch + 1, jch + 1) = R(0);
                }
                c.sync();
                lartg(A(jch + 1, jch), A(jch + 1, jch - 1), cs, sn, r);
                c.sync();
                qzr_cols(p, jch, jch + 1, jch, cs, sn, tid, nth);
                if (tid == 0) {
                    A(jch + 1, jch) = r;
                    A(jch + 1, jch - 1) = R(0);
                }
            }
            inf_bottom = true;
        }
        if (inf_bottom) {
            c.sync();
            lartg(A(ilast, ilast), A(ilast, ilast - 1), cs, sn, r);
            c.sync();
            qzr_cols(p, ilast, ilast, ilast, cs, sn, tid, nth);
            if (tid == 0) {
                A(ilast, ilast) = r;
                A(ilast, ilast - 1) = R(0);
            }
            deflate = true;
        }
        if (deflate) {  // a real eigenvalue: T(ilast, ilast) made non-negative
            c.sync();
            const bool neg = B(ilast, ilast) < R(0);
            c.sync();
            if (neg) qzr_negate_col(p, ilast, ilast + 1, ilast + 1, tid, nth);
            c.sync();
            if (tid == 0) {
                p.alphar[ilast] = A(ilast, ilast);
                p.alphai[ilast] = R(0);
                p.beta[ilast] = B(ilast, ilast);
            }
            ilast--;
            iiter = 0;
            eshift = R(0);
            continue;
        }
        if (action != 4) continue;
        bool single = true;
        R s1 = R(1), wr = R(0);
        if (ifirst + 1 == ilast) {  // a 2x2 block: standardise it (xLAGV2)
            c.sync();
            R a[16], b[16];
            a[0] = A(ilast - 1, ilast - 1), a[1] = A(ilast, ilast - 1), a[LD] = A(ilast - 1, ilast),
            a[1 + LD] = A(ilast, ilast);
            b[0] = B(ilast - 1, ilast - 1), b[1] = R(0), b[LD] = B(ilast - 1, ilast), b[1 + LD] = B(ilast, ilast);
            R csl, snl, csr, snr;
            lagv2(a, b, csl, snl, csr, snr);
            c.sync();
            qzr_rows(p, ilast - 1, ilast + 1, ilast + 1, csl, snl, tid, nth);
            qzr_cols(p, ilast, ilast - 1, ilast - 1, csr, -snr, tid, nth);
            if (tid == 0) {
                A(ilast - 1, ilast - 1) = a[0], A(ilast, ilast - 1) = a[1], A(ilast - 1, ilast) = a[LD],
                                 A(ilast, ilast) = a[1 + LD];
                B(ilast - 1, ilast - 1) = b[0], B(ilast, ilast - 1) = R(0), B(ilast - 1, ilast) = b[LD],
                                 B(ilast, ilast) = b[1 + LD];
            }
            if (a[1] == R(0)) continue;  // real eigenvalues: two 1x1 blocks, deflated next
            // a complex pair: T's block diagonal; make it positive, then deflate both rows
            c.sync();
            const bool n1 = B(ilast - 1, ilast - 1) < R(0), n2 = B(ilast, ilast) < R(0);
            c.sync();
            if (n1) qzr_negate_col(p, ilast - 1, ilast + 1, ilast, tid, nth);
            if (n2) qzr_negate_col(p, ilast, ilast + 1, ilast + 1, tid, nth);
            c.sync();
            R ab[16] = {}, bb[16] = {};
            ab[0] = A(ilast - 1, ilast - 1), ab[1] = A(ilast, ilast - 1), ab[LD] = A(ilast - 1, ilast),
            ab[1 + LD] = A(ilast, ilast);
            bb[0] = B(ilast - 1, ilast - 1), bb[LD] = R(0), bb[1 + LD] = B(ilast, ilast);
            R ar[2], ai[2], be[2];
            if (pair_alphas(ab, bb, ar, ai, be)) {
                c.sync();
                if (tid == 0)
                    for (int k = 0; k < 2; k++) {
                        p.alphar[ilast - 1 + k] = ar[k];
                        p.alphai[ilast - 1 + k] = ai[k];
                        p.beta[ilast - 1 + k] = be[k];
                    }
                ilast -= 2;
                iiter = 0;
                eshift = R(0);
                continue;
            }
            // xLAG2 puts the pair on the real line after all: one real single-shift step
            R t1_, t2_, wi_;
            lag2(ab, bb, safmin * R(100), s1, t1_, wr, t2_, wi_);
        } else {
            iiter++;
            c.sync();
            if (iiter % 10 == 0) {  // exceptional real shift
                if (R(maxit) * safmin * xabs(A(ilast, ilast - 1)) < xabs(B(ilast - 1, ilast - 1)))
                    eshift = A(ilast, ilast - 1) / B(ilast - 1, ilast - 1);
                else
                    eshift = eshift + R(1) / (safmin * R(maxit));
                s1 = R(1);
                wr = eshift;
            } else {  // the trailing 2 x 2 pencil's eigenvalues (xLAG2), the closer one first
                R a[16] = {}, b[16] = {};
                a[0] = A(ilast - 1, ilast - 1), a[1] = A(ilast, ilast - 1), a[LD] = A(ilast - 1, ilast),
                a[1 + LD] = A(ilast, ilast);
                b[0] = B(ilast - 1, ilast - 1), b[LD] = B(ilast - 1, ilast), b[1 + LD] = B(ilast, ilast);
                R s2, wr2, wi;
                lag2(a, b, safmin * R(100), s1, s2, wr, wr2, wi);
                if (xabs((wr / s1) * B(ilast, ilast) - A(ilast, ilast)) >
                    xabs((wr2 / s2) * B(ilast, ilast) - A(ilast, ilast))) {
                    R t = wr;
                    wr = wr2;
                    wr2 = t;
                    t = s1;
                    s1 = s2;
                    s2 = t;
                }
                single = wi == R(0);
            }
        }
        if (single) {  // a single real shift (s1, wr) over [ifirst, ilast]
            lartg(s1 * A(ifirst, ifirst) - wr * B(ifirst, ifirst), s1 * A(ifirst + 1, ifirst), cs, sn, r);
            for (int jj = ifirst; jj < ilast; jj++) {
                if (jj > ifirst) {
                    c.sync();
                    lartg(A(jj, jj - 1), A(jj + 1, jj - 1), cs, sn, r);
                }
                c.sync();
                qzr_rows(p, jj, jj, jj, cs, sn, tid, nth);
                if (tid == 0 && jj > ifirst) {
                    A(jj, jj - 1) = r;
                    A(jj + 1, jj - 1) = R(0);
                }
                c.sync();
                lartg(B(jj + 1, jj + 1), B(jj + 1, jj), cs, sn, r);
                c.sync();
                qzr_cols(p, jj + 1, (jj + 2 < ilast ? jj + 2 : ilast) + 1, jj + 1, cs, sn, tid, nth);
                if (tid == 0) {
                    B(jj + 1, jj + 1) = r;
                    B(jj + 1, jj) = R(0);
                }
            }
            continue;
        }
        // an implicit double shift over [ifirst, ilast] (block of order >= 3)
        R v[3], tau;
        {
            const R ad11 = (ascale * A(ilast - 1, ilast - 1)) / (bscale * B(ilast - 1, ilast - 1));
            const R ad21 = (ascale * A(ilast, ilast - 1)) / (bscale * B(ilast - 1, ilast - 1));
            const R ad12 = (ascale * A(ilast - 1, ilast)) / (bscale * B(ilast, ilast));
            const R ad22 = (ascale * A(ilast, ilast)) / (bscale * B(ilast, ilast));
            const R u12 = B(ilast - 1, ilast) / B(ilast, ilast);
            const R ad11l = (ascale * A(ifirst, ifirst)) / (bscale * B(ifirst, ifirst));
            const R ad21l = (ascale * A(ifirst + 1, ifirst)) / (bscale * B(ifirst, ifirst));
            const R ad12l = (ascale * A(ifirst, ifirst + 1)) / (bscale * B(ifirst + 1, ifirst + 1));
            const R ad22l = (ascale * A(ifirst + 1, ifirst + 1)) / (bscale * B(ifirst + 1, ifirst + 1));
            const R ad32l = (ascale * A(ifirst + 2, ifirst + 1)) / (bscale * B(ifirst + 1, ifirst + 1));
            const R u12l = B(ifirst, ifirst + 1) / B(ifirst + 1, ifirst + 1);
            v[0] = (ad11 - ad11l) * (ad22 - ad11l) - ad12 * ad21 + ad21 * u12 * ad11l + (ad12l - ad11l * u12l) * ad21l;
            v[1] = ((ad22l - ad11l) - ad21l * u12l - (ad11 - ad11l) - (ad22 - ad11l) + ad21 * u12) * ad21l;
            v[2] = ad32l * ad21l;
            larfg(3, v[0], &v[1], 1, tau);
        }
        for (int jj = ifirst; jj + 2 <= ilast; jj++) {
            if (jj > ifirst) {  // the reflector that zeroes A(jj+1, jj-1), A(jj+2, jj-1)
                c.sync();
                R alpha = A(jj, jj - 1);
                v[1] = A(jj + 1, jj - 1);
                v[2] = A(jj + 2, jj - 1);
                larfg(3, alpha, &v[1], 1, tau);
                r = alpha;
            }
            c.sync();
            qzr_refl_rows(p, jj, jj, jj, v[1], v[2], tau, tid, nth);
            if (tid == 0 && jj > ifirst) {
                A(jj, jj - 1) = r;
                A(jj + 1, jj - 1) = R(0);
                A(jj + 2, jj - 1) = R(0);
            }
            // the reflector from the right that zeroes B(jj+1, jj), B(jj+2, jj): a pivoted
            // 2 x 2 solve (DHGEQZ)
            c.sync();
            R w11, w21, w12, w22, u1, u2, scale = R(1);
            bool pivot = false, solved = false;
            const R tmp1 = xmax(xabs(B(jj + 1, jj + 1)), xabs(B(jj + 1, jj + 2)));
            const R tmp2 = xmax(xabs(B(jj + 2, jj + 1)), xabs(B(jj + 2, jj + 2)));
            if (xmax(tmp1, tmp2) < safmin) {
                scale = R(0);
                u1 = R(1);
                u2 = R(0);
                solved = true;
            } else if (tmp1 >= tmp2) {
                w11 = B(jj + 1, jj + 1), w21 = B(jj + 2, jj + 1), w12 = B(jj + 1, jj + 2), w22 = B(jj + 2, jj + 2);
                u1 = B(jj + 1, jj), u2 = B(jj + 2, jj);
            } else {
                w21 = B(jj + 1, jj + 1), w11 = B(jj + 2, jj + 1), w22 = B(jj + 1, jj + 2), w12 = B(jj + 2, jj + 2);
                u2 = B(jj + 1, jj), u1 = B(jj + 2, jj);
            }
            if (!solved) {
                if (xabs(w12) > xabs(w11)) {
                    pivot = true;
                    R t = w12;
                    w12 = w11;
                    w11 = t;
                    t = w22;
                    w22 = w21;
                    w21 = t;
                }
                const R t = w21 / w11;
                u2 -= t * u1;
                w22 -= t * w12;
                if (xabs(w22) < safmin) {
                    scale = R(0);
                    u2 = R(1);
                    u1 = -w12 / w11;
                } else {
                    if (xabs(w22) < xabs(u2)) scale = xabs(w22 / u2);
                    if (xabs(w11) < xabs(u1)) scale = xmin(scale, xabs(w11 / u1));
                    u2 = (scale * u2) / w22;
                    u1 = (scale * u1 - w12 * u2) / w11;
                }
            }
            if (pivot) {
                const R t = u2;
                u2 = u1;
                u1 = t;
            }
            const R t1 = xsqrt(scale * scale + u1 * u1 + u2 * u2);
            const R taur = R(1) + scale / t1, vs = -R(1) / (scale + t1);
            c.sync();
            qzr_refl_cols(p, jj, (jj + 3 < ilast ? jj + 3 : ilast) + 1, jj + 3, vs * u1, vs * u2, taur, tid, nth);
            c.sync();  // the reflector has written B(jj+1, jj), B(jj+2, jj) too: zero them after it
            if (tid == 0) {
                B(jj + 1, jj) = R(0);
                B(jj + 2, jj) = R(0);
            }
        }
        {  // the last step: rotations
            const int jl = ilast - 1;
            c.sync();
            lartg(A(jl, jl - 1), A(jl + 1, jl - 1), cs, sn, r);
            c.sync();
            qzr_rows(p, jl, jl, jl, cs, sn, tid, nth);
            if (tid == 0) {
                A(jl, jl - 1) = r;
                A(jl + 1, jl - 1) = R(0);
            }
            c.sync();
            lartg(B(jl + 1, jl + 1), B(jl + 1, jl), cs, sn, r);
            c.sync();
            qzr_cols(p, jl + 1, ilast + 1, ilast, cs, sn, tid, nth);
            if (tid == 0) {
                B(jl + 1, jl + 1) = r;
                B(jl + 1, jl) = R(0);
            }
        }
    }
    c.sync();
    return info;
}

}  // namespace rb
}  // namespace xtg
