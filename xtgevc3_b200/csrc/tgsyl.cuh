// The generalized Sylvester equation of a pair of real generalized Schur pencils (LAPACK
// D/STGSYL with TRANS = 'N'):
//     A R - L B = scale C,   D R - L E = scale F,
// A, D m x m (A upper quasi-triangular, D upper triangular), B, E n x n (likewise), R and L
// m x n, overwriting C and F.  IJOB 0 solves; IJOB 3 only estimates DIF (C, F start at zero and
// every small system is solved by xLATDF's look-ahead, which accumulates a Frobenius-norm
// estimate of the smallest singular value); IJOB 1 solves, then estimates as IJOB 3 and puts
// the solution back.  Host and device code: the kernels in qz.cu run tgsyl_cta on one CTA; the
// tests run it on host threads and on one thread.
//
// The solve follows xTGSYL's blocked order, because the estimate's accumulators (and the
// rounding of the solution) depend on it: A's rows cut into blocks of ILAENV's 2 rows (one row
// more where a cut would split a 2x2 block), B's columns into 2-column blocks likewise (m <= 2
// and n <= 2: one block, xTGSYL's unblocked case); column blocks left to right, row blocks
// bottom to top; each block solved by xTGSY2 (its 1x1 / 2x2 diagonal blocks, each a Kronecker
// system of order 2, 4 or 8 by xGETC2 with complete pivoting, then xGESC2 with its own scale
// factor or xLATDF), then the rows above it updated (C -= A R, F -= D R) and the columns right
// of it (C += L B, F += L E).  A scale factor below 1 scales all of C and F.
//
// B200 form: thread 0 solves each block (dependent steps on at most 3 x 3 rows and columns);
// between barriers the CTA applies the block's two updates (rows above and columns right are
// disjoint) and any scaling.
//
// Complex pencils (Z/CTGSYL): the same with 1x1 diagonal blocks only (no 2x2 block to keep
// whole), each small system the 2 x 2 complex one of ZTGSY2, ZGESC2 (below) or ZLATDF.
#pragma once

#include "tgsna_dif_cplx.cuh"

namespace xtg {
namespace rb {

template <class R>
struct SylvG {
    int m, n;
    const R *A, *D, *B, *E;
    int lda, ldd, ldb, lde;
    R *C, *F;
    int ldc, ldf;
    R dsum, dscale;  // xLATDF's accumulators (IJOB 1 and 3)
};

// xTGSY2 on the block rows [is0, ie0] x columns [js0, je0] of C, F (0-based): the block's own
// 1x1 / 2x2 diagonal blocks of A (bottom to top) and B (left to right), each solved and
// substituted into the block's rows above and columns right.  ifunc 0: xGESC2 (scaloc < 1
// scales the whole block and multiplies into scaloc); 1: xLATDF into y.dsum / y.dscale.
// Returns xGETC2's INFO (> 0: a pivot was raised).
template <class R>
XTG_HD int tgsy2_sub(SylvG<R> &y, int is0, int ie0, int js0, int je0, int ifunc, R &scaloc)
{
    auto a = [&](int i, int k) { return y.A[(size_t)i + (size_t)k * y.lda]; };
    auto d = [&](int i, int k) { return y.D[(size_t)i + (size_t)k * y.ldd]; };
    auto b = [&](int i, int k) { return y.B[(size_t)i + (size_t)k * y.ldb]; };
    auto e = [&](int i, int k) { return y.E[(size_t)i + (size_t)k * y.lde]; };
    auto C = [&](int i, int k) -> R & { return y.C[(size_t)i + (size_t)k * y.ldc]; };
    auto F = [&](int i, int k) -> R & { return y.F[(size_t)i + (size_t)k * y.ldf]; };
    int ist[5], jst[5], np = 0, nq = 0;
    for (int i = is0; i <= ie0;) {
        ist[np++] = i;
        i += (i < ie0 && a(i + 1, i) != R(0)) ? 2 : 1;
    }
    ist[np] = ie0 + 1;
    for (int j = js0; j <= je0;) {
        jst[nq++] = j;
        j += (j < je0 && b(j + 1, j) != R(0)) ? 2 : 1;
    }
    jst[nq] = je0 + 1;
    int info = 0;
    for (int jb = 0; jb < nq; jb++) {
        const int js = jst[jb], nb = jst[jb + 1] - js;
        for (int ib = np - 1; ib >= 0; ib--) {
            const int is = ist[ib], mb = ist[ib + 1] - is;
            const int nn = mb * nb, zdim = 2 * nn;
            R Z[64], rhs[8];
            for (int t = 0; t < 64; t++) Z[t] = R(0);
            for (int j = 0; j < nb; j++)
                for (int i = 0; i < mb; i++) {
                    const int k = i + mb * j;
                    for (int p = 0; p < mb; p++) {
                        Z[k + 8 * (p + mb * j)] = a(is + i, is + p);
                        if (p >= i) Z[(nn + k) + 8 * (p + mb * j)] = d(is + i, is + p);
                    }
                    for (int q = 0; q < nb; q++) {
                        Z[k + 8 * (nn + i + mb * q)] = -b(js + q, js + j);
                        if (q <= j) Z[(nn + k) + 8 * (nn + i + mb * q)] = -e(js + q, js + j);
                    }
                    rhs[k] = C(is + i, js + j);
                    rhs[nn + k] = F(is + i, js + j);
                }
            int ipiv[8], jpiv[8];
            const int ierr = getc2(zdim, Z, ipiv, jpiv);
            if (ierr > 0) info = ierr;
            if (ifunc == 0) {
                R sc = R(1);
                gesc2(zdim, Z, rhs, ipiv, jpiv, sc);
                if (sc != R(1)) {
                    for (int k = js0; k <= je0; k++)
                        for (int i = is0; i <= ie0; i++) {
                            C(i, k) *= sc;
                            F(i, k) *= sc;
                        }
                    scaloc *= sc;
                }
            } else {
                latdf(zdim, Z, rhs, y.dsum, y.dscale, ipiv, jpiv);
            }
            for (int j = 0; j < nb; j++)
                for (int i = 0; i < mb; i++) {
                    C(is + i, js + j) = rhs[i + mb * j];
                    F(is + i, js + j) = rhs[nn + i + mb * j];
                }
            // rows [is0, is) of the block: C -= A R, F -= D R
            for (int r = is0; r < is; r++)
                for (int j = 0; j < nb; j++) {
                    R c = C(r, js + j), f = F(r, js + j);
                    for (int p = 0; p < mb; p++) {
                        const R rv = rhs[p + mb * j];
                        c -= a(r, is + p) * rv;
                        f -= d(r, is + p) * rv;
                    }
                    C(r, js + j) = c;
                    F(r, js + j) = f;
                }
            // columns (js + nb, je0] of the block: C += L B, F += L E
            for (int col = js + nb; col <= je0; col++)
                for (int i = 0; i < mb; i++) {
                    R c = C(is + i, col), f = F(is + i, col);
                    for (int q = 0; q < nb; q++) {
                        const R lv = rhs[nn + i + mb * q];
                        c += lv * b(js + q, col);
                        f += lv * e(js + q, col);
                    }
                    C(is + i, col) = c;
                    F(is + i, col) = f;
                }
        }
    }
    return info;
}

// xTGSYL's block starts of an order-m quasi-triangular matrix T (2-row blocks, one row more
// where a cut would split a 2x2 block); returns the count, starts[count] = m.  starts has
// room for m / 2 + 2 entries.  m <= 2 and n <= 2 (the caller's test): one block.
template <class R>
XTG_HD int tgsyl_cuts(int m, const R *T, int ldt, int *starts)
{
    int p = 0, i = 1;  // 1-based as xTGSYL
    while (i <= m) {
        starts[p++] = i - 1;
        i += 2;
        if (i >= m) break;
        if (T[(size_t)(i - 1) + (size_t)(i - 2) * ldt] != R(0)) i++;
    }
    starts[p] = m;
    if (starts[p - 1] == starts[p]) p--;
    return p;
}

// the CTA's shared state of tgsyl_cta (shared memory on the GPU); lac: xLACN2's state when the
// solver is driven by the 1-norm estimator
template <class R>
struct Lacn2 {
    int kase, jump, j, iter;
    R est, estold;
};

template <class R>
struct SylvShared {
    SylvG<R> y;
    R scaloc, scale;
    int info, np, nq;
    Lacn2<R> lac;
};

// One round of xTGSYL over every block (ifunc 0: solve, 1: estimate) on one CTA.  rows /
// cols: the block starts of A and B (tgsyl_cuts, or {0, m} / {0, n}).  Ends with a barrier.
template <class R, class Cta>
XTG_HD void tgsyl_round(const Cta &c, SylvShared<R> &sh, const int *rows, const int *cols, int ifunc)
{
    const int tid = c.tid(), nth = c.nth();
    SylvG<R> &y = sh.y;
    const int np = sh.np, nq = sh.nq, m = y.m, n = y.n;
    for (int jb = 0; jb < nq; jb++) {
        const int js = cols[jb], je = cols[jb + 1] - 1;
        for (int ib = np - 1; ib >= 0; ib--) {
            const int is = rows[ib], ie = rows[ib + 1] - 1;
            if (tid == 0) {
                R sl = R(1);
                const int li = tgsy2_sub(y, is, ie, js, je, ifunc, sl);
                if (li > 0) sh.info = li;
                sh.scaloc = sl;
            }
            c.sync();  // the block's solution and scaloc are in memory
            const R sl = sh.scaloc;
            if (sl != R(1)) {  // every entry outside the block
                for (size_t t = tid; t < (size_t)m * n; t += nth) {
                    const int i = (int)(t % m), k = (int)(t / m);
                    if (k >= js && k <= je && i >= is && i <= ie) continue;
                    y.C[(size_t)i + (size_t)k * y.ldc] *= sl;
                    y.F[(size_t)i + (size_t)k * y.ldf] *= sl;
                }
                if (tid == 0) sh.scale *= sl;
                c.sync();  // scaled before the updates read and write the same entries
            }
            // rows above the block (C -= A R, F -= D R) and columns right of it (C += L B,
            // F += L E): disjoint, one pass; R, L read from the block, which nobody writes
            const int nbk = je - js + 1, mbk = ie - is + 1;
            const size_t above = (size_t)is * nbk, right = (size_t)mbk * (n - 1 - je);
            for (size_t t = tid; t < above + right; t += nth) {
                if (t < above) {
                    const int r = (int)(t % is), k = js + (int)(t / is);
                    R cv = y.C[(size_t)r + (size_t)k * y.ldc], fv = y.F[(size_t)r + (size_t)k * y.ldf];
                    for (int p = is; p <= ie; p++) {
                        const R rv = y.C[(size_t)p + (size_t)k * y.ldc];
                        cv -= y.A[(size_t)r + (size_t)p * y.lda] * rv;
                        fv -= y.D[(size_t)r + (size_t)p * y.ldd] * rv;
                    }
                    y.C[(size_t)r + (size_t)k * y.ldc] = cv;
                    y.F[(size_t)r + (size_t)k * y.ldf] = fv;
                } else {
                    const size_t u = t - above;
                    const int i = is + (int)(u % mbk), k = je + 1 + (int)(u / mbk);
                    R cv = y.C[(size_t)i + (size_t)k * y.ldc], fv = y.F[(size_t)i + (size_t)k * y.ldf];
                    for (int q = js; q <= je; q++) {
                        const R lv = y.F[(size_t)i + (size_t)q * y.ldf];
                        cv += lv * y.B[(size_t)q + (size_t)k * y.ldb];
                        fv += lv * y.E[(size_t)q + (size_t)k * y.lde];
                    }
                    y.C[(size_t)i + (size_t)k * y.ldc] = cv;
                    y.F[(size_t)i + (size_t)k * y.ldf] = fv;
                }
            }
            c.sync();  // the updates are in memory before the next block is solved
        }
    }
}

// xTGSYL (TRANS = 'N', IJOB 0, 1 or 3) on one CTA.  sh.y holds the operands on entry (m, n
// >= 1); cuts: room for m / 2 + n / 2 + 4 ints; work (IJOB 1 only): 2 m n elements for the
// saved solution.  On return (every thread, after a barrier): sh.scale, sh.info, and *dif for
// IJOB 1 and 3 (left as it was when the estimate's accumulator stayed 0, as xTGSYL does).
template <class R, class Cta>
XTG_HD void tgsyl_cta(const Cta &c, SylvShared<R> &sh, int ijob, int *cuts, R *work, R *dif)
{
    const int tid = c.tid(), nth = c.nth();
    SylvG<R> &y = sh.y;
    const int m = y.m, n = y.n;
    int *rows = cuts, *cols = cuts + m / 2 + 2;
    if (tid == 0) {
        if (m <= 2 && n <= 2) {
            rows[0] = 0;
            rows[1] = m;
            cols[0] = 0;
            cols[1] = n;
            sh.np = sh.nq = 1;
        } else {
            sh.np = tgsyl_cuts(m, y.A, y.lda, rows);
            sh.nq = tgsyl_cuts(n, y.B, y.ldb, cols);
        }
        sh.info = 0;
        sh.scale = R(1);
        y.dsum = R(1);
        y.dscale = R(0);
    }
    if (ijob == 3)  // only the estimate: C, F start at zero
        for (size_t t = tid; t < (size_t)m * n; t += nth) {
            y.C[(t % m) + (t / m) * (size_t)y.ldc] = R(0);
            y.F[(t % m) + (t / m) * (size_t)y.ldf] = R(0);
        }
    c.sync();
    tgsyl_round(c, sh, rows, cols, ijob == 3 ? 1 : 0);
    if (ijob == 1) {  // keep the solution, estimate from zero right-hand sides, put it back
        const R scale1 = sh.scale;
        for (size_t t = tid; t < (size_t)m * n; t += nth) {
            R &cv = y.C[(t % m) + (t / m) * (size_t)y.ldc];
            R &fv = y.F[(t % m) + (t / m) * (size_t)y.ldf];
            work[t] = cv;
            work[(size_t)m * n + t] = fv;
            cv = R(0);
            fv = R(0);
        }
        c.sync();
        if (tid == 0) {
            y.dsum = R(1);
            y.dscale = R(0);
            sh.scale = R(1);
        }
        c.sync();
        tgsyl_round(c, sh, rows, cols, 1);
        for (size_t t = tid; t < (size_t)m * n; t += nth) {
            y.C[(t % m) + (t / m) * (size_t)y.ldc] = work[t];
            y.F[(t % m) + (t / m) * (size_t)y.ldf] = work[(size_t)m * n + t];
        }
        if (tid == 0) sh.scale = scale1;
    }
    if (ijob != 0 && tid == 0 && y.dscale != R(0)) *dif = xsqrt(R(2 * m) * R(n)) / (y.dscale * xsqrt(y.dsum));
    c.sync();
}

// ---- the transposed equation (xTGSYL with TRANS = 'T', IJOB 0) ------------------------------
//     A^T R + D^T L = scale C,   R B^T + L E^T = -scale F
// the blocks visited in the other order (row blocks top to bottom, column blocks right to
// left), each small system the transpose of the one for TRANS = 'N', and the solution
// substituted into the rows below (C -= A^T R + D^T L) and the columns left (F += R B^T + L E^T).

// xTGSY2 with TRANS = 'T' on the block rows [is0, ie0] x columns [js0, je0]
template <class R>
XTG_HD int tgsy2_sub_t(SylvG<R> &y, int is0, int ie0, int js0, int je0, R &scaloc)
{
    auto a = [&](int i, int k) { return y.A[(size_t)i + (size_t)k * y.lda]; };
    auto d = [&](int i, int k) { return y.D[(size_t)i + (size_t)k * y.ldd]; };
    auto b = [&](int i, int k) { return y.B[(size_t)i + (size_t)k * y.ldb]; };
    auto e = [&](int i, int k) { return y.E[(size_t)i + (size_t)k * y.lde]; };
    auto C = [&](int i, int k) -> R & { return y.C[(size_t)i + (size_t)k * y.ldc]; };
    auto F = [&](int i, int k) -> R & { return y.F[(size_t)i + (size_t)k * y.ldf]; };
    int ist[5], jst[5], np = 0, nq = 0;
    for (int i = is0; i <= ie0;) {
        ist[np++] = i;
        i += (i < ie0 && a(i + 1, i) != R(0)) ? 2 : 1;
    }
    ist[np] = ie0 + 1;
    for (int j = js0; j <= je0;) {
        jst[nq++] = j;
        j += (j < je0 && b(j + 1, j) != R(0)) ? 2 : 1;
    }
    jst[nq] = je0 + 1;
    int info = 0;
    for (int ib = 0; ib < np; ib++) {
        const int is = ist[ib], mb = ist[ib + 1] - is, ie = is + mb - 1;
        for (int jb = nq - 1; jb >= 0; jb--) {
            const int js = jst[jb], nb = jst[jb + 1] - js;
            const int nn = mb * nb, zdim = 2 * nn;
            R Zn[64], Z[64], rhs[8];
            for (int t = 0; t < 64; t++) Zn[t] = R(0);
            for (int j = 0; j < nb; j++)
                for (int i = 0; i < mb; i++) {
                    const int k = i + mb * j;
                    for (int p = 0; p < mb; p++) {
                        Zn[k + 8 * (p + mb * j)] = a(is + i, is + p);
                        if (p >= i) Zn[(nn + k) + 8 * (p + mb * j)] = d(is + i, is + p);
                    }
                    for (int q = 0; q < nb; q++) {
                        Zn[k + 8 * (nn + i + mb * q)] = -b(js + q, js + j);
                        if (q <= j) Zn[(nn + k) + 8 * (nn + i + mb * q)] = -e(js + q, js + j);
                    }
                    rhs[k] = C(is + i, js + j);
                    rhs[nn + k] = F(is + i, js + j);
                }
            for (int r = 0; r < 8; r++)
                for (int q = 0; q < 8; q++) Z[r + 8 * q] = Zn[q + 8 * r];
            int ipiv[8], jpiv[8];
            const int ierr = getc2(zdim, Z, ipiv, jpiv);
            if (ierr > 0) info = ierr;
            R sc = R(1);
            gesc2(zdim, Z, rhs, ipiv, jpiv, sc);
            if (sc != R(1)) {
                for (int k = js0; k <= je0; k++)
                    for (int i = is0; i <= ie0; i++) {
                        C(i, k) *= sc;
                        F(i, k) *= sc;
                    }
                scaloc *= sc;
            }
            for (int j = 0; j < nb; j++)
                for (int i = 0; i < mb; i++) {
                    C(is + i, js + j) = rhs[i + mb * j];
                    F(is + i, js + j) = rhs[nn + i + mb * j];
                }
            // columns [js0, js) of the block: F += R B^T, then F += L E^T
            for (int col = js0; col < js; col++)
                for (int i = 0; i < mb; i++) {
                    R f = F(is + i, col);
                    for (int q = 0; q < nb; q++) f += rhs[i + mb * q] * b(col, js + q);
                    for (int q = 0; q < nb; q++) f += rhs[nn + i + mb * q] * e(col, js + q);
                    F(is + i, col) = f;
                }
            // rows (ie, ie0] of the block: C -= A^T R, then C -= D^T L
            for (int row = ie + 1; row <= ie0; row++)
                for (int j = 0; j < nb; j++) {
                    R cv = C(row, js + j);
                    for (int p = 0; p < mb; p++) cv -= a(is + p, row) * rhs[p + mb * j];
                    for (int p = 0; p < mb; p++) cv -= d(is + p, row) * rhs[nn + p + mb * j];
                    C(row, js + j) = cv;
                }
        }
    }
    return info;
}

// One pass of xTGSYL with TRANS = 'T' over every block on one CTA.  Ends with a barrier.
template <class R, class Cta>
XTG_HD void tgsyl_round_t(const Cta &c, SylvShared<R> &sh, const int *rows, const int *cols)
{
    const int tid = c.tid(), nth = c.nth();
    SylvG<R> &y = sh.y;
    const int np = sh.np, nq = sh.nq, m = y.m, n = y.n;
    for (int ib = 0; ib < np; ib++) {
        const int is = rows[ib], ie = rows[ib + 1] - 1;
        for (int jb = nq - 1; jb >= 0; jb--) {
            const int js = cols[jb], je = cols[jb + 1] - 1;
            if (tid == 0) {
                R sl = R(1);
                const int li = tgsy2_sub_t(y, is, ie, js, je, sl);
                if (li > 0) sh.info = li;
                sh.scaloc = sl;
            }
            c.sync();
            const R sl = sh.scaloc;
            if (sl != R(1)) {
                for (size_t t = tid; t < (size_t)m * n; t += nth) {
                    const int i = (int)(t % m), k = (int)(t / m);
                    if (k >= js && k <= je && i >= is && i <= ie) continue;
                    y.C[(size_t)i + (size_t)k * y.ldc] *= sl;
                    y.F[(size_t)i + (size_t)k * y.ldf] *= sl;
                }
                if (tid == 0) sh.scale *= sl;
                c.sync();
            }
            // columns left of the block in its rows (F += R B^T + L E^T) and rows below it in
            // its columns (C -= A^T R + D^T L): disjoint, one pass
            const int nbk = je - js + 1, mbk = ie - is + 1;
            const size_t left = (size_t)mbk * js, below = (size_t)(m - 1 - ie) * nbk;
            for (size_t t = tid; t < left + below; t += nth) {
                if (t < left) {
                    const int i = is + (int)(t % mbk), col = (int)(t / mbk);
                    R f = y.F[(size_t)i + (size_t)col * y.ldf];
                    for (int q = js; q <= je; q++)
                        f += y.C[(size_t)i + (size_t)q * y.ldc] * y.B[(size_t)col + (size_t)q * y.ldb];
                    for (int q = js; q <= je; q++)
                        f += y.F[(size_t)i + (size_t)q * y.ldf] * y.E[(size_t)col + (size_t)q * y.lde];
                    y.F[(size_t)i + (size_t)col * y.ldf] = f;
                } else {
                    const size_t u = t - left;
                    const int row = ie + 1 + (int)(u % (m - 1 - ie)), k = js + (int)(u / (m - 1 - ie));
                    R cv = y.C[(size_t)row + (size_t)k * y.ldc];
                    for (int p = is; p <= ie; p++)
                        cv -= y.A[(size_t)p + (size_t)row * y.lda] * y.C[(size_t)p + (size_t)k * y.ldc];
                    for (int p = is; p <= ie; p++)
                        cv -= y.D[(size_t)p + (size_t)row * y.ldd] * y.F[(size_t)p + (size_t)k * y.ldf];
                    y.C[(size_t)row + (size_t)k * y.ldc] = cv;
                }
            }
            c.sync();
        }
    }
}

// xTGSYL with TRANS = 'T' (IJOB 0: the solve) on one CTA; sh.y and cuts as for tgsyl_cta.  On
// return (every thread, after a barrier): sh.scale, sh.info.
template <class R, class Cta>
XTG_HD void tgsyl_t_cta(const Cta &c, SylvShared<R> &sh, int *cuts)
{
    const int tid = c.tid();
    SylvG<R> &y = sh.y;
    const int m = y.m, n = y.n;
    int *rows = cuts, *cols = cuts + m / 2 + 2;
    if (tid == 0) {
        if (m <= 2 && n <= 2) {
            rows[0] = 0;
            rows[1] = m;
            cols[0] = 0;
            cols[1] = n;
            sh.np = sh.nq = 1;
        } else {
            sh.np = tgsyl_cuts(m, y.A, y.lda, rows);
            sh.nq = tgsyl_cuts(n, y.B, y.ldb, cols);
        }
        sh.info = 0;
        sh.scale = R(1);
    }
    c.sync();
    tgsyl_round_t(c, sh, rows, cols);
}

// ---- the 1-norm estimator (xLACN2, N. J. Higham, ACM TOMS 14 (1988) 381-396) --------------
// Reverse communication: on kase = 0 the caller starts; the estimator sets x and kase = 1
// (the caller overwrites x by the operator applied to x) or kase = 2 (by its transpose) and is
// called again, until it returns kase = 0 with est the estimate.  At most 5 iterations.
template <class R>
XTG_HD void lacn2(int n, R *v, R *x, int *isgn, Lacn2<R> &s)
{
    const int itmax = 5;
    auto asum = [&](const R *w) {
        R t = R(0);
        for (int i = 0; i < n; i++) t += xabs(w[i]);
        return t;
    };
    auto amax = [&]() {
        int k = 0;
        for (int i = 1; i < n; i++)
            if (xabs(x[i]) > xabs(x[k])) k = i;
        return k;
    };
    auto signs = [&]() {
        for (int i = 0; i < n; i++) {
            x[i] = x[i] >= R(0) ? R(1) : R(-1);
            isgn[i] = x[i] > R(0) ? 1 : -1;
        }
    };
    auto unit = [&]() {  // x = e_j, the operator next
        for (int i = 0; i < n; i++) x[i] = R(0);
        x[s.j] = R(1);
        s.kase = 1;
        s.jump = 3;
    };
    auto final_stage = [&]() {
        R altsgn = R(1);
        for (int i = 0; i < n; i++) {
            x[i] = altsgn * (R(1) + R(i) / R(n - 1));
            altsgn = -altsgn;
        }
        s.kase = 1;
        s.jump = 5;
    };
    if (s.kase == 0) {
        for (int i = 0; i < n; i++) x[i] = R(1) / R(n);
        s.kase = 1;
        s.jump = 1;
        return;
    }
    switch (s.jump) {
    case 1:  // x = A x, first iteration
        if (n == 1) {
            v[0] = x[0];
            s.est = xabs(v[0]);
            s.kase = 0;
            return;
        }
        s.est = asum(x);
        signs();
        s.kase = 2;
        s.jump = 2;
        return;
    case 2:  // x = A^T x, first iteration
        s.j = amax();
        s.iter = 2;
        unit();
        return;
    case 3: {  // x = A x
        for (int i = 0; i < n; i++) v[i] = x[i];
        s.estold = s.est;
        s.est = asum(v);
        bool same = true;
        for (int i = 0; i < n; i++)
            if ((x[i] >= R(0) ? 1 : -1) != isgn[i]) {
                same = false;
                break;
            }
        if (same || s.est <= s.estold) {  // repeated sign vector, or cycling: converged
            final_stage();
            return;
        }
        signs();
        s.kase = 2;
        s.jump = 4;
        return;
    }
    case 4: {  // x = A^T x
        const int jlast = s.j;
        s.j = amax();
        if (x[jlast] != xabs(x[s.j]) && s.iter < itmax) {
            s.iter++;
            unit();
            return;
        }
        final_stage();
        return;
    }
    default: {  // case 5: x = A x, final stage
        const R temp = R(2) * (asum(x) / R(3 * n));
        if (temp > s.est) {
            for (int i = 0; i < n; i++) v[i] = x[i];
            s.est = temp;
        }
        s.kase = 0;
        return;
    }
    }
}

// ---- complex pencils (Z/CTGSYL, TRANS = 'N') -------------------------------------------------

// Solve Z x = scale rhs with zgetc2's 2 x 2 factors, scale <= 1 chosen against overflow
// (ZGESC2: the largest entry by |re| + |im|, its modulus against the last pivot's)
template <class R>
XTG_HD void zgesc2(const zc<R> *Z, zc<R> *rhs, const int *ipiv, const int *jpiv, R &scale)
{
    const int n = 2;
    const R eps = Mach<R>::prec, smlnum = Mach<R>::sfmin / eps;
    for (int i = 0; i < n - 1; i++)
        if (ipiv[i] != i) {
            const zc<R> t = rhs[i];
            rhs[i] = rhs[ipiv[i]];
            rhs[ipiv[i]] = t;
        }
    for (int i = 0; i < n - 1; i++)
        for (int j = i + 1; j < n; j++) rhs[j] = rhs[j] - Z[j + 2 * i] * rhs[i];
    scale = R(1);
    int imax = 0;
    for (int i = 1; i < n; i++)
        if (xabs(rhs[i].re) + xabs(rhs[i].im) > xabs(rhs[imax].re) + xabs(rhs[imax].im)) imax = i;
    if (R(2) * smlnum * cabs(rhs[imax]) > cabs(Z[(n - 1) + 2 * (n - 1)])) {
        const R t = R(0.5) / cabs(rhs[imax]);
        for (int i = 0; i < n; i++) rhs[i] = t * rhs[i];
        scale *= t;
    }
    const zc<R> one = mk(R(1), R(0));
    for (int i = n - 1; i >= 0; i--) {
        const zc<R> t = cdiv(one, Z[i + 2 * i]);
        rhs[i] = rhs[i] * t;
        for (int j = i + 1; j < n; j++) rhs[i] = rhs[i] - rhs[j] * (Z[i + 2 * j] * t);
    }
    for (int i = n - 2; i >= 0; i--)
        if (jpiv[i] != i) {
            const zc<R> t = rhs[i];
            rhs[i] = rhs[jpiv[i]];
            rhs[jpiv[i]] = t;
        }
}

template <class R>
struct ZSylvG {
    int m, n;
    const zc<R> *A, *D, *B, *E;
    int lda, ldd, ldb, lde;
    zc<R> *C, *F;
    int ldc, ldf;
    R dsum, dscale;
};

// ZTGSY2 on the block rows [is0, ie0] x columns [js0, je0] (as tgsy2_sub, 1x1 blocks)
template <class R>
XTG_HD int ztgsy2_sub(ZSylvG<R> &y, int is0, int ie0, int js0, int je0, int ifunc, R &scaloc)
{
    auto a = [&](int i, int k) { return y.A[(size_t)i + (size_t)k * y.lda]; };
    auto d = [&](int i, int k) { return y.D[(size_t)i + (size_t)k * y.ldd]; };
    auto b = [&](int i, int k) { return y.B[(size_t)i + (size_t)k * y.ldb]; };
    auto e = [&](int i, int k) { return y.E[(size_t)i + (size_t)k * y.lde]; };
    auto C = [&](int i, int k) -> zc<R> & { return y.C[(size_t)i + (size_t)k * y.ldc]; };
    auto F = [&](int i, int k) -> zc<R> & { return y.F[(size_t)i + (size_t)k * y.ldf]; };
    int info = 0;
    for (int j = js0; j <= je0; j++)
        for (int i = ie0; i >= is0; i--) {
            zc<R> Z[4] = {a(i, i), d(i, i), -b(j, j), -e(j, j)}, rhs[2] = {C(i, j), F(i, j)};
            int ipiv[2], jpiv[2];
            const int ierr = zgetc2(Z, ipiv, jpiv);
            if (ierr > 0) info = ierr;
            if (ifunc == 0) {
                R sc = R(1);
                zgesc2(Z, rhs, ipiv, jpiv, sc);
                if (sc != R(1)) {
                    for (int k = js0; k <= je0; k++)
                        for (int r = is0; r <= ie0; r++) {
                            C(r, k) = sc * C(r, k);
                            F(r, k) = sc * F(r, k);
                        }
                    scaloc *= sc;
                }
            } else {
                zlatdf(Z, rhs, y.dsum, y.dscale, ipiv, jpiv);
            }
            C(i, j) = rhs[0];
            F(i, j) = rhs[1];
            const zc<R> alpha = -rhs[0];
            for (int r = is0; r < i; r++) {
                C(r, j) = C(r, j) + alpha * a(r, i);
                F(r, j) = F(r, j) + alpha * d(r, i);
            }
            for (int col = j + 1; col <= je0; col++) {
                C(i, col) = C(i, col) + rhs[1] * b(j, col);
                F(i, col) = F(i, col) + rhs[1] * e(j, col);
            }
        }
    return info;
}

template <class R>
struct ZLacn2 {
    int kase, jump, j, iter;
    R est, estold;
};

template <class R>
struct ZSylvShared {
    ZSylvG<R> y;
    R scaloc, scale;
    int info, np, nq;
    ZLacn2<R> lac;
};

// One round of ZTGSYL over every block on one CTA (as tgsyl_round).  Ends with a barrier.
template <class R, class Cta>
XTG_HD void ztgsyl_round(const Cta &c, ZSylvShared<R> &sh, const int *rows, const int *cols, int ifunc)
{
    const int tid = c.tid(), nth = c.nth();
    ZSylvG<R> &y = sh.y;
    const int np = sh.np, nq = sh.nq, m = y.m, n = y.n;
    for (int jb = 0; jb < nq; jb++) {
        const int js = cols[jb], je = cols[jb + 1] - 1;
        for (int ib = np - 1; ib >= 0; ib--) {
            const int is = rows[ib], ie = rows[ib + 1] - 1;
            if (tid == 0) {
                R sl = R(1);
                const int li = ztgsy2_sub(y, is, ie, js, je, ifunc, sl);
                if (li > 0) sh.info = li;
                sh.scaloc = sl;
            }
            c.sync();
            const R sl = sh.scaloc;
            if (sl != R(1)) {
                for (size_t t = tid; t < (size_t)m * n; t += nth) {
                    const int i = (int)(t % m), k = (int)(t / m);
                    if (k >= js && k <= je && i >= is && i <= ie) continue;
                    zc<R> &cv = y.C[(size_t)i + (size_t)k * y.ldc];
                    zc<R> &fv = y.F[(size_t)i + (size_t)k * y.ldf];
                    cv = sl * cv;
                    fv = sl * fv;
                }
                if (tid == 0) sh.scale *= sl;
                c.sync();
            }
            const int nbk = je - js + 1, mbk = ie - is + 1;
            const size_t above = (size_t)is * nbk, right = (size_t)mbk * (n - 1 - je);
            for (size_t t = tid; t < above + right; t += nth) {
                if (t < above) {
                    const int r = (int)(t % is), k = js + (int)(t / is);
                    zc<R> cv = y.C[(size_t)r + (size_t)k * y.ldc], fv = y.F[(size_t)r + (size_t)k * y.ldf];
                    for (int p = is; p <= ie; p++) {
                        const zc<R> rv = y.C[(size_t)p + (size_t)k * y.ldc];
                        cv = cv - y.A[(size_t)r + (size_t)p * y.lda] * rv;
                        fv = fv - y.D[(size_t)r + (size_t)p * y.ldd] * rv;
                    }
                    y.C[(size_t)r + (size_t)k * y.ldc] = cv;
                    y.F[(size_t)r + (size_t)k * y.ldf] = fv;
                } else {
                    const size_t u = t - above;
                    const int i = is + (int)(u % mbk), k = je + 1 + (int)(u / mbk);
                    zc<R> cv = y.C[(size_t)i + (size_t)k * y.ldc], fv = y.F[(size_t)i + (size_t)k * y.ldf];
                    for (int q = js; q <= je; q++) {
                        const zc<R> lv = y.F[(size_t)i + (size_t)q * y.ldf];
                        cv = cv + lv * y.B[(size_t)q + (size_t)k * y.ldb];
                        fv = fv + lv * y.E[(size_t)q + (size_t)k * y.lde];
                    }
                    y.C[(size_t)i + (size_t)k * y.ldc] = cv;
                    y.F[(size_t)i + (size_t)k * y.ldf] = fv;
                }
            }
            c.sync();
        }
    }
}

// ZTGSYL (TRANS = 'N', IJOB 0, 1 or 3) on one CTA, as tgsyl_cta (blocks of 2 rows and 2
// columns, ZTGSYL's unblocked case for m, n <= 2).
template <class R, class Cta>
XTG_HD void ztgsyl_cta(const Cta &c, ZSylvShared<R> &sh, int ijob, int *cuts, zc<R> *work, R *dif)
{
    const int tid = c.tid(), nth = c.nth();
    ZSylvG<R> &y = sh.y;
    const int m = y.m, n = y.n;
    int *rows = cuts, *cols = cuts + m / 2 + 2;
    const zc<R> zero = mk(R(0), R(0));
    if (tid == 0) {
        if (m <= 2 && n <= 2) {
            rows[0] = 0;
            rows[1] = m;
            cols[0] = 0;
            cols[1] = n;
            sh.np = sh.nq = 1;
        } else {
            sh.np = ztgsyl_blocks(m, rows);
            sh.nq = ztgsyl_blocks(n, cols);
        }
        sh.info = 0;
        sh.scale = R(1);
        y.dsum = R(1);
        y.dscale = R(0);
    }
    if (ijob == 3)
        for (size_t t = tid; t < (size_t)m * n; t += nth) {
            y.C[(t % m) + (t / m) * (size_t)y.ldc] = zero;
            y.F[(t % m) + (t / m) * (size_t)y.ldf] = zero;
        }
    c.sync();
    ztgsyl_round(c, sh, rows, cols, ijob == 3 ? 1 : 0);
    if (ijob == 1) {
        const R scale1 = sh.scale;
        for (size_t t = tid; t < (size_t)m * n; t += nth) {
            zc<R> &cv = y.C[(t % m) + (t / m) * (size_t)y.ldc];
            zc<R> &fv = y.F[(t % m) + (t / m) * (size_t)y.ldf];
            work[t] = cv;
            work[(size_t)m * n + t] = fv;
            cv = zero;
            fv = zero;
        }
        c.sync();
        if (tid == 0) {
            y.dsum = R(1);
            y.dscale = R(0);
            sh.scale = R(1);
        }
        c.sync();
        ztgsyl_round(c, sh, rows, cols, 1);
        for (size_t t = tid; t < (size_t)m * n; t += nth) {
            y.C[(t % m) + (t / m) * (size_t)y.ldc] = work[t];
            y.F[(t % m) + (t / m) * (size_t)y.ldf] = work[(size_t)m * n + t];
        }
        if (tid == 0) sh.scale = scale1;
    }
    if (ijob != 0 && tid == 0 && y.dscale != R(0)) *dif = xsqrt(R(2 * m) * R(n)) / (y.dscale * xsqrt(y.dsum));
    c.sync();
}

// ---- the conjugate-transposed equation (Z/CTGSYL with TRANS = 'C', IJOB 0) -----------------
//     A^H R + D^H L = scale C,   R B^H + L E^H = -scale F
// entries of A top to bottom, of B right to left (within and across the 2 x 2 blocks of
// rows / columns), each 2 x 2 system Z^H of ZTGSY2, the solution substituted into the rows
// below (C -= A^H R + D^H L) and the columns left (F += R B^H + L E^H).

template <class R>
XTG_HD int ztgsy2_sub_c(ZSylvG<R> &y, int is0, int ie0, int js0, int je0, R &scaloc)
{
    auto a = [&](int i, int k) { return y.A[(size_t)i + (size_t)k * y.lda]; };
    auto d = [&](int i, int k) { return y.D[(size_t)i + (size_t)k * y.ldd]; };
    auto b = [&](int i, int k) { return y.B[(size_t)i + (size_t)k * y.ldb]; };
    auto e = [&](int i, int k) { return y.E[(size_t)i + (size_t)k * y.lde]; };
    auto C = [&](int i, int k) -> zc<R> & { return y.C[(size_t)i + (size_t)k * y.ldc]; };
    auto F = [&](int i, int k) -> zc<R> & { return y.F[(size_t)i + (size_t)k * y.ldf]; };
    int info = 0;
    for (int i = is0; i <= ie0; i++)
        for (int j = je0; j >= js0; j--) {
            zc<R> Z[4] = {conj(a(i, i)), -conj(b(j, j)), conj(d(i, i)), -conj(e(j, j))}, rhs[2] = {C(i, j), F(i, j)};
            int ipiv[2], jpiv[2];
            const int ierr = zgetc2(Z, ipiv, jpiv);
            if (ierr > 0) info = ierr;
            R sc = R(1);
            zgesc2(Z, rhs, ipiv, jpiv, sc);
            if (sc != R(1)) {
                for (int k = js0; k <= je0; k++)
                    for (int r = is0; r <= ie0; r++) {
                        C(r, k) = sc * C(r, k);
                        F(r, k) = sc * F(r, k);
                    }
                scaloc *= sc;
            }
            C(i, j) = rhs[0];
            F(i, j) = rhs[1];
            for (int k = js0; k < j; k++) F(i, k) = F(i, k) + rhs[0] * conj(b(k, j)) + rhs[1] * conj(e(k, j));
            for (int k = i + 1; k <= ie0; k++) C(k, j) = C(k, j) - conj(a(i, k)) * rhs[0] - conj(d(i, k)) * rhs[1];
        }
    return info;
}

template <class R, class Cta>
XTG_HD void ztgsyl_round_c(const Cta &c, ZSylvShared<R> &sh, const int *rows, const int *cols)
{
    const int tid = c.tid(), nth = c.nth();
    ZSylvG<R> &y = sh.y;
    const int np = sh.np, nq = sh.nq, m = y.m, n = y.n;
    for (int ib = 0; ib < np; ib++) {
        const int is = rows[ib], ie = rows[ib + 1] - 1;
        for (int jb = nq - 1; jb >= 0; jb--) {
            const int js = cols[jb], je = cols[jb + 1] - 1;
            if (tid == 0) {
                R sl = R(1);
                const int li = ztgsy2_sub_c(y, is, ie, js, je, sl);
                if (li > 0) sh.info = li;
                sh.scaloc = sl;
            }
            c.sync();
            const R sl = sh.scaloc;
            if (sl != R(1)) {
                for (size_t t = tid; t < (size_t)m * n; t += nth) {
                    const int i = (int)(t % m), k = (int)(t / m);
                    if (k >= js && k <= je && i >= is && i <= ie) continue;
                    zc<R> &cv = y.C[(size_t)i + (size_t)k * y.ldc];
                    zc<R> &fv = y.F[(size_t)i + (size_t)k * y.ldf];
                    cv = sl * cv;
                    fv = sl * fv;
                }
                if (tid == 0) sh.scale *= sl;
                c.sync();
            }
            const int nbk = je - js + 1, mbk = ie - is + 1;
            const size_t left = (size_t)mbk * js, below = (size_t)(m - 1 - ie) * nbk;
            for (size_t t = tid; t < left + below; t += nth) {
                if (t < left) {  // F += R B^H, then F += L E^H
                    const int i = is + (int)(t % mbk), col = (int)(t / mbk);
                    zc<R> f = y.F[(size_t)i + (size_t)col * y.ldf];
                    for (int q = js; q <= je; q++)
                        f = f + y.C[(size_t)i + (size_t)q * y.ldc] * conj(y.B[(size_t)col + (size_t)q * y.ldb]);
                    for (int q = js; q <= je; q++)
                        f = f + y.F[(size_t)i + (size_t)q * y.ldf] * conj(y.E[(size_t)col + (size_t)q * y.lde]);
                    y.F[(size_t)i + (size_t)col * y.ldf] = f;
                } else {  // C -= A^H R, then C -= D^H L
                    const size_t u = t - left;
                    const int row = ie + 1 + (int)(u % (m - 1 - ie)), k = js + (int)(u / (m - 1 - ie));
                    zc<R> cv = y.C[(size_t)row + (size_t)k * y.ldc];
                    for (int p = is; p <= ie; p++)
                        cv = cv - conj(y.A[(size_t)p + (size_t)row * y.lda]) * y.C[(size_t)p + (size_t)k * y.ldc];
                    for (int p = is; p <= ie; p++)
                        cv = cv - conj(y.D[(size_t)p + (size_t)row * y.ldd]) * y.F[(size_t)p + (size_t)k * y.ldf];
                    y.C[(size_t)row + (size_t)k * y.ldc] = cv;
                }
            }
            c.sync();
        }
    }
}

// Z/CTGSYL with TRANS = 'C' (the solve) on one CTA, as tgsyl_t_cta
template <class R, class Cta>
XTG_HD void ztgsyl_c_cta(const Cta &c, ZSylvShared<R> &sh, int *cuts)
{
    const int tid = c.tid();
    ZSylvG<R> &y = sh.y;
    const int m = y.m, n = y.n;
    int *rows = cuts, *cols = cuts + m / 2 + 2;
    if (tid == 0) {
        if (m <= 2 && n <= 2) {
            rows[0] = 0;
            rows[1] = m;
            cols[0] = 0;
            cols[1] = n;
            sh.np = sh.nq = 1;
        } else {
            sh.np = ztgsyl_blocks(m, rows);
            sh.nq = ztgsyl_blocks(n, cols);
        }
        sh.info = 0;
        sh.scale = R(1);
    }
    c.sync();
    ztgsyl_round_c(c, sh, rows, cols);
}

// ZLACN2 (Higham's estimator for complex operators): as lacn2, with x / |x| (1 where |x| <=
// safmin) in place of the signs and no repeated-sign test; |.| the modulus throughout.
template <class R>
XTG_HD void zlacn2(int n, zc<R> *v, zc<R> *x, ZLacn2<R> &s)
{
    const int itmax = 5;
    const R safmin = Mach<R>::sfmin;
    const zc<R> one = mk(R(1), R(0)), zero = mk(R(0), R(0));
    auto asum = [&](const zc<R> *w) {
        R t = R(0);
        for (int i = 0; i < n; i++) t += cabs(w[i]);
        return t;
    };
    auto amax = [&]() {
        int k = 0;
        R best = cabs(x[0]);
        for (int i = 1; i < n; i++) {
            const R v_ = cabs(x[i]);
            if (v_ > best) {
                best = v_;
                k = i;
            }
        }
        return k;
    };
    auto phases = [&]() {
        for (int i = 0; i < n; i++) {
            const R ax = cabs(x[i]);
            x[i] = ax > safmin ? mk(x[i].re / ax, x[i].im / ax) : one;
        }
    };
    auto unit = [&]() {
        for (int i = 0; i < n; i++) x[i] = zero;
        x[s.j] = one;
        s.kase = 1;
        s.jump = 3;
    };
    auto final_stage = [&]() {
        R altsgn = R(1);
        for (int i = 0; i < n; i++) {
            x[i] = mk(altsgn * (R(1) + R(i) / R(n - 1)), R(0));
            altsgn = -altsgn;
        }
        s.kase = 1;
        s.jump = 5;
    };
    if (s.kase == 0) {
        for (int i = 0; i < n; i++) x[i] = mk(R(1) / R(n), R(0));
        s.kase = 1;
        s.jump = 1;
        return;
    }
    switch (s.jump) {
    case 1:
        if (n == 1) {
            v[0] = x[0];
            s.est = cabs(v[0]);
            s.kase = 0;
            return;
        }
        s.est = asum(x);
        phases();
        s.kase = 2;
        s.jump = 2;
        return;
    case 2:
        s.j = amax();
        s.iter = 2;
        unit();
        return;
    case 3:
        for (int i = 0; i < n; i++) v[i] = x[i];
        s.estold = s.est;
        s.est = asum(v);
        if (s.est <= s.estold) {  // cycling: converged
            final_stage();
            return;
        }
        phases();
        s.kase = 2;
        s.jump = 4;
        return;
    case 4: {
        const int jlast = s.j;
        s.j = amax();
        if (cabs(x[jlast]) != cabs(x[s.j]) && s.iter < itmax) {
            s.iter++;
            unit();
            return;
        }
        final_stage();
        return;
    }
    default: {
        const R temp = R(2) * (asum(x) / R(3 * n));
        if (temp > s.est) {
            for (int i = 0; i < n; i++) v[i] = x[i];
            s.est = temp;
        }
        s.kase = 0;
        return;
    }
    }
}

}  // namespace rb
}  // namespace xtg
