// Reordering a generalized Schur pencil by a selection: the selected eigenvalues move to the
// leading rows (LAPACK D/S/Z/CTGSEN with IJOB = 0, the step xGGES takes when SORT = 'S', its
// SELECT being SELCTG of the QZ eigenvalues), and xTGSEN's estimates for IJOB 1-5 on the
// reordered pencil (tgsen_real_estimates / tgsen_cplx_estimates, on the solvers of
// tgsyl.cuh).  Host and device code: the kernels in qz.cu run these bodies on one CTA
// (rb::CtaDev); the tests run them on host threads and on one thread.
//
// Real pencils (DTGSEN): the diagonal blocks are visited from the top, a 2x2 block counting as
// selected when either of its rows is; each selected block moves up to the next free leading
// row by the xTGEXC walk of tgexc_real_blocks.cuh (walk_cta), and the first rejected swap ends
// the reordering (INFO = 1).  Then, whether or not every move was done, the eigenvalues are
// recomputed from the final pencil: xLAG2 on each 2x2 block (alphar = the two real parts,
// alphai = +-wi, beta = the two scales), and each 1x1 block whose B(k, k) has its sign bit set
// has row k of A and B and column k of Q negated, then alphar = A(k, k), alphai = 0,
// beta = B(k, k).
//
// Complex pencils (ZTGSEN): alpha and beta start as the diagonals of the input.  With M
// selected eigenvalues and 0 < M < n, each selected one moves up to the next free leading row
// by the single swaps of tgsna_dif_cplx.cuh (zswap11, here also applied to Q and Z), and the
// first rejected swap ends the call (INFO = 1, alpha and beta as they started).  After a
// complete reordering every row is normalised so that B(k, k) is real and non-negative: with
// d = |B(k, k)| > safmin, row k of A (columns k..n) and of B (columns k+1..n) is multiplied by
// t = conj(B(k, k) / d), B(k, k) = d and column k of Q is multiplied by conj(t); with
// d <= safmin, B(k, k) = 0.  Then alpha = diag(A), beta = diag(B).  M = 0 or M = n leaves the
// pencil as it is.
//
// B200 form: one CTA.  The decisions (which block moves, and where) read only the selection
// and the subdiagonal, so every thread takes them alike between barriers; each swap is computed
// by thread 0 and applied by the whole CTA.  The final passes spread the rows over the threads,
// with the per-row facts (block kind, sign, scale factor) written first to the eigenvalue
// arrays, which receive their final values in the last pass.
#pragma once

#include "tgsna_dif_cplx.cuh"
#include "tgsyl.cuh"

namespace xtg {
namespace rb {

// ---- real pencils: DTGSEN with IJOB = 0 -----------------------------------------------------

// The moves: returns INFO, 0, 1 (a swap was rejected) or 3 (a walk reached its bound, which
// the walk's own argument rules out).  Every thread returns the same value, after a barrier.
template <class R, class Cta>
XTG_HD int tgsen_real_reorder(const Cta &c, WalkShared<R> &sh, const Pencil<R> &p, const int *select)
{
    const int n = p.n;
    auto A = [&](int i, int j) -> R & { return p.A[(size_t)i + (size_t)j * p.lda]; };
    int info = 0, ks = 0;  // ks: the next free leading row (0-based)
    for (int k = 0; k < n; k++) {
        const bool pair = k + 1 < n && A(k + 1, k) != R(0);
        if (select[k] != 0 || (pair && select[k + 1] != 0)) {
            if (k != ks) {
                walk_cta(c, sh, p, k + 1, ks + 1);  // ends with a barrier
                const int wi = sh.info;
                c.sync();  // every thread has read the walk's state before the next walk rewrites it
                if (wi != 0) {
                    info = wi;
                    break;
                }
            }
            ks += pair ? 2 : 1;
        }
        if (pair) k++;
    }
    c.sync();  // the last swap is in memory
    return info;
}

// DTGSEN's M: the selected eigenvalues, a 2x2 block counting 2 when either of its rows is
template <class R>
XTG_HD int tgsen_real_m(const Pencil<R> &p, const int *select)
{
    int m = 0;
    for (int k = 0; k < p.n; k++) {
        if (k + 1 < p.n && p.A[(size_t)(k + 1) + (size_t)k * p.lda] != R(0)) {
            m += (select[k] != 0 || select[k + 1] != 0) ? 2 : 0;
            k++;
        } else {
            m += select[k] != 0 ? 1 : 0;
        }
    }
    return m;
}

// The eigenvalues of the (reordered) pencil, 1x1 blocks made non-negative in B.  Ends with a
// barrier.
template <class R, class Cta>
XTG_HD void tgsen_real_finish(const Cta &c, const Pencil<R> &p, R *alphar, R *alphai, R *beta)
{
    const int n = p.n, tid = c.tid(), nth = c.nth();
    auto A = [&](int i, int j) -> R & { return p.A[(size_t)i + (size_t)j * p.lda]; };
    auto B = [&](int i, int j) -> R & { return p.B[(size_t)i + (size_t)j * p.ldb]; };
    auto Q = [&](int i, int j) -> R & { return p.Q[(size_t)i + (size_t)j * p.ldq]; };
    // pass 1: block kind of each row (0: 1x1, 1: first row of a 2x2 block, 2: its second row)
    // into alphai, B(k, k) into beta, by the same top-down scan as the reordering's
    for (int k = 0; k < n; k++) {
        const bool pair = k + 1 < n && A(k + 1, k) != R(0);
        if (k % nth == tid) {
            alphai[k] = pair ? R(1) : R(0);
            beta[k] = B(k, k);
        }
        if (pair) {
            if ((k + 1) % nth == tid) alphai[k + 1] = R(2);
            k++;
        }
    }
    c.sync();
    // pass 2: 1x1 blocks whose B(k, k) has its sign bit set: rows k of A and B, column k of Q
    // negated (column i by thread i mod nth)
    for (int k = 0; k < n; k++) {
        if (alphai[k] != R(0) || !(xsign(R(1), beta[k]) < R(0))) continue;
        for (int i = tid; i < n; i += nth) {
            A(k, i) = -A(k, i);
            B(k, i) = -B(k, i);
            if (p.wantq) Q(i, k) = -Q(i, k);
        }
    }
    c.sync();
    // pass 3: the eigenvalues, row k by thread k mod nth (both rows of a 2x2 block evaluate
    // xLAG2 on it, each keeping its own row's values)
    for (int k = tid; k < n; k += nth) {
        const R kind = alphai[k];
        if (kind == R(0)) {
            alphar[k] = A(k, k);
            alphai[k] = R(0);
            beta[k] = B(k, k);
        } else {
            const int k0 = kind == R(1) ? k : k - 1;
            R a[2 * LD], b[2 * LD];
            a[0] = A(k0, k0);
            a[1] = A(k0 + 1, k0);
            a[LD] = A(k0, k0 + 1);
            a[LD + 1] = A(k0 + 1, k0 + 1);
            b[0] = B(k0, k0);
            b[1] = B(k0 + 1, k0);
            b[LD] = B(k0, k0 + 1);
            b[LD + 1] = B(k0 + 1, k0 + 1);
            R s1, s2, wr1, wr2, wi;
            lag2(a, b, Mach<R>::sfmin, s1, s2, wr1, wr2, wi);
            if (k == k0) {
                beta[k] = s1;
                alphar[k] = wr1;
                alphai[k] = wi;
            } else {
                beta[k] = s2;
                alphar[k] = wr2;
                alphai[k] = -wi;
            }
        }
    }
    c.sync();
}

// DTGSEN with IJOB = 0: returns INFO as tgsen_real_reorder (the eigenvalues recomputed in
// every case).  alphar, alphai, beta: n each.
template <class R, class Cta>
XTG_HD int tgsen_real_cta(const Cta &c, WalkShared<R> &sh, const Pencil<R> &p, const int *select, R *alphar,
                          R *alphai, R *beta)
{
    const int info = tgsen_real_reorder(c, sh, p, select);
    tgsen_real_finish(c, p, alphar, alphai, beta);
    return info;
}

// DTGSEN's estimates on the reordered pencil (IJOB 1 to 5; m = M, info the reordering's):
// est[0], est[1] = PL, PR (IJOB 1, 4, 5: 1 / sqrt(1 + ||R||^2 / scale^2) and the same with L,
// from xTGSYL's solution of A11 R - L A22 = A12, B11 R - L B22 = B12), est[2], est[3] = DIF(1),
// DIF(2): IJOB 2 and 4 xTGSYL's Frobenius-norm estimates (its IJOB = 3) of Difu on (A11, B11),
// (A22, B22) and of Difl with the two swapped; IJOB 3 and 5 scale / xLACN2's 1-norm estimate
// of the inverse of the same operators (xTGSYL solves with TRANS = 'N' and 'T').  M = 0 or n:
// PL = PR = 1, DIF = ||(A, B)||_F; a rejected swap: all 0.  work: 4 M (n - M) elements (2 M
// (n - M) for IJOB 1, 2, 4); iwork: 2 M (n - M) ints (IJOB 3, 5); cuts: n / 2 + 4 ints.  Ends
// with a barrier.
template <class R, class Cta>
XTG_HD void tgsen_real_estimates(const Cta &c, SylvShared<R> &sh, const Pencil<R> &p, int m, int ijob, int info,
                                 R *work, int *iwork, int *cuts, R *est)
{
    const int n = p.n, tid = c.tid(), nth = c.nth();
    const bool wantp = ijob == 1 || ijob == 4 || ijob == 5, wantd1 = ijob == 2 || ijob == 4,
               wantd2 = ijob == 3 || ijob == 5, wantd = wantd1 || wantd2;
    if (tid == 0)
        for (int k = 0; k < 4; k++) est[k] = R(0);
    if (info != 0 || (!wantp && !wantd)) {
        c.sync();
        return;
    }
    if (m == 0 || m == n) {
        if (tid == 0) {
            if (wantp) est[0] = est[1] = R(1);
            if (wantd) {
                R sc = R(0), sq = R(1);
                for (int j = 0; j < n; j++) {
                    lassq(n, p.A + (size_t)j * p.lda, sc, sq);
                    lassq(n, p.B + (size_t)j * p.ldb, sc, sq);
                }
                est[2] = est[3] = sc * xsqrt(sq);
            }
        }
        c.sync();
        return;
    }
    const int n1 = m, n2 = n - m;
    const size_t mn = (size_t)n1 * n2;
    R *W = work, *V = work + mn;
    const R *A11 = p.A, *B11 = p.B;
    const R *A22 = p.A + n1 + (size_t)n1 * p.lda, *B22 = p.B + n1 + (size_t)n1 * p.ldb;
    // xTGSYL's operands: (a, d) the mm x mm pencil, (b, e) the nn x nn one; a, b in A (lda),
    // d, e in B (ldb); C, F = W, V with leading dimension mm
    auto setup = [&](int mm, int nn, const R *a, const R *d, const R *b, const R *e) {
        if (tid == 0) {
            SylvG<R> &y = sh.y;
            y.m = mm;
            y.n = nn;
            y.A = a;
            y.D = d;
            y.B = b;
            y.E = e;
            y.lda = y.ldb = p.lda;
            y.ldd = y.lde = p.ldb;
            y.C = W;
            y.F = V;
            y.ldc = y.ldf = mm;
        }
        c.sync();
    };
    if (wantp) {
        for (size_t t = tid; t < mn; t += nth) {  // C = A12, F = B12
            const int i = (int)(t % n1), j = n1 + (int)(t / n1);
            W[t] = p.A[(size_t)i + (size_t)j * p.lda];
            V[t] = p.B[(size_t)i + (size_t)j * p.ldb];
        }
        setup(n1, n2, A11, B11, A22, B22);
        R unused = R(0);
        tgsyl_cta(c, sh, 0, cuts, (R *)nullptr, &unused);
        if (tid == 0) {
            const R dscale = sh.scale;
            for (int k = 0; k < 2; k++) {
                R sc = R(0), sq = R(1);
                lassq((int)mn, k == 0 ? W : V, sc, sq);
                R v = sc * xsqrt(sq);
                v = v == R(0) ? R(1) : dscale / (xsqrt(dscale * dscale / v + v) * xsqrt(v));
                est[k] = v;
            }
        }
        c.sync();
    }
    if (wantd1) {
        setup(n1, n2, A11, B11, A22, B22);
        tgsyl_cta(c, sh, 3, cuts, (R *)nullptr, est + 2);
        setup(n2, n1, A22, B22, A11, B11);
        tgsyl_cta(c, sh, 3, cuts, (R *)nullptr, est + 3);
    }
    if (wantd2) {  // xLACN2 on [vec C; vec F] = work[0, 2 mn), its v in work[2 mn, 4 mn)
        const int mn2 = (int)(2 * mn);
        R *Vl = work + 2 * mn;
        for (int which = 0; which < 2; which++) {
            if (tid == 0) {
                sh.lac.kase = 0;
                lacn2(mn2, Vl, W, iwork, sh.lac);
            }
            c.sync();
            R dscale = R(1);
            for (int step = 0; step < 16; step++) {  // xLACN2 asks for at most 11 products
                const int kase = sh.lac.kase;
                if (kase == 0) break;
                if (which == 0) setup(n1, n2, A11, B11, A22, B22);
                else setup(n2, n1, A22, B22, A11, B11);
                R unused = R(0);
                if (kase == 1) tgsyl_cta(c, sh, 0, cuts, (R *)nullptr, &unused);
                else tgsyl_t_cta(c, sh, cuts);
                if (tid == 0) {
                    dscale = sh.scale;
                    lacn2(mn2, Vl, W, iwork, sh.lac);
                }
                c.sync();
            }
            if (tid == 0) est[2 + which] = dscale / sh.lac.est;
            c.sync();
        }
    }
}

// DTGSEN with IJOB 0 to 5 (tgsen_real_estimates): M (into *m_out from thread 0), the moves,
// the estimates on the reordered pencil, the eigenvalues.  Returns INFO as tgsen_real_reorder.
// est: PL, PR, DIF(1), DIF(2).
template <class R, class Cta>
XTG_HD int tgsen_real_full_cta(const Cta &c, WalkShared<R> &shw, SylvShared<R> &shs, const Pencil<R> &p,
                               const int *select, int ijob, R *alphar, R *alphai, R *beta, R *work, int *iwork,
                               int *cuts, R *est, int *m_out)
{
    const int m = tgsen_real_m(p, select);  // reads the subdiagonal before the first swap's barrier
    if (m_out && c.tid() == 0) *m_out = m;
    const int info = tgsen_real_reorder(c, shw, p, select);
    tgsen_real_estimates(c, shs, p, m, ijob, info, work, iwork, cuts, est);
    tgsen_real_finish(c, p, alphar, alphai, beta);
    return info;
}

// ---- complex pencils: ZTGSEN with IJOB = 0 --------------------------------------------------

template <class R>
struct ZPencil {
    int n, wantq, wantz;
    zc<R> *A, *B, *Q, *Z;
    int lda, ldb, ldq, ldz;
};

// the CTA's shared state (shared memory on the GPU)
template <class R>
struct ZSortShared {
    ZSwap<R> s;
    int rej;
};

// The swap of rows / columns (j, j + 1), j = s.j: its rotations and tests (one thread)
template <class R>
XTG_HD void zsort_prepare(const ZPencil<R> &p, ZSwap<R> &s)
{
    const int j = s.j;
    auto a = [&](int i, int k) { return p.A[(size_t)(j + i) + (size_t)(j + k) * p.lda]; };
    auto b = [&](int i, int k) { return p.B[(size_t)(j + i) + (size_t)(j + k) * p.ldb]; };
    s.ok = zswap11(a(0, 0), a(1, 0), a(0, 1), a(1, 1), b(0, 0), b(1, 0), b(0, 1), b(1, 1), s.cz, s.szc, s.cq, s.sq)
               ? 1
               : 0;
}

// Applying a done swap by thread tid of nth: phase 0 rotates columns j, j+1 (rows [0, j + 2)
// of A and B, every row of Z), phase 1 (after a barrier) rows j, j+1 (columns [j, n) of A and
// B) and columns j, j+1 of Q with the conjugate rotation, phase 2 (after a barrier, one
// thread) zeroes the two subdiagonal entries, as ZTGEX2 does.
template <class R>
XTG_HD void zsort_apply(const ZPencil<R> &p, const ZSwap<R> &s, int phase, int tid, int nth)
{
    const int j = s.j, n = p.n;
    auto at = [](zc<R> *M, int ld, int i, int k) -> zc<R> & { return M[(size_t)i + (size_t)k * ld]; };
    if (phase == 0) {
        const int r = j + 2, cnt = 2 * r + (p.wantz ? n : 0);
        for (int i = tid; i < cnt; i += nth) {
            if (i < r) zrot(at(p.A, p.lda, i, j), at(p.A, p.lda, i, j + 1), s.cz, s.szc);
            else if (i < 2 * r) zrot(at(p.B, p.ldb, i - r, j), at(p.B, p.ldb, i - r, j + 1), s.cz, s.szc);
            else zrot(at(p.Z, p.ldz, i - 2 * r, j), at(p.Z, p.ldz, i - 2 * r, j + 1), s.cz, s.szc);
        }
    } else if (phase == 1) {
        const int c = n - j, cnt = 2 * c + (p.wantq ? n : 0);
        const zc<R> sqc = conj(s.sq);
        for (int i = tid; i < cnt; i += nth) {
            if (i < c) zrot(at(p.A, p.lda, j, j + i), at(p.A, p.lda, j + 1, j + i), s.cq, s.sq);
            else if (i < 2 * c) zrot(at(p.B, p.ldb, j, j + i - c), at(p.B, p.ldb, j + 1, j + i - c), s.cq, s.sq);
            else zrot(at(p.Q, p.ldq, i - 2 * c, j), at(p.Q, p.ldq, i - 2 * c, j + 1), s.cq, sqc);
        }
    } else if (tid == 0) {
        at(p.A, p.lda, j + 1, j) = mk(R(0), R(0));
        at(p.B, p.ldb, j + 1, j) = mk(R(0), R(0));
    }
}

// The moves of ZTGSEN: alpha, beta first the input diagonals; with 0 < M < n each selected
// eigenvalue walks up to the next free leading row.  Returns INFO, 0 or 1 (a swap was
// rejected).  Every thread returns the same value, after a barrier.
template <class R, class Cta>
XTG_HD int tgsen_cplx_reorder(const Cta &c, ZSortShared<R> &sh, const ZPencil<R> &p, const int *select, zc<R> *alpha,
                              zc<R> *beta)
{
    const int n = p.n, tid = c.tid(), nth = c.nth();
    auto A = [&](int i, int j) -> zc<R> & { return p.A[(size_t)i + (size_t)j * p.lda]; };
    auto B = [&](int i, int j) -> zc<R> & { return p.B[(size_t)i + (size_t)j * p.ldb]; };
    for (int k = tid; k < n; k += nth) {
        alpha[k] = A(k, k);
        beta[k] = B(k, k);
    }
    int m = 0;
    for (int k = 0; k < n; k++) m += select[k] != 0 ? 1 : 0;
    c.sync();  // the diagonals are read before the first swap writes A and B
    if (m == 0 || m == n) return 0;
    int ks = 0;
    for (int k = 0; k < n; k++) {
        if (select[k] == 0) continue;
        for (int j = k - 1; j >= ks; j--) {
            if (tid == 0) {
                sh.s.j = j;
                zsort_prepare(p, sh.s);
                sh.rej = sh.s.ok ? 0 : 1;
            }
            c.sync();  // thread 0 writes s / rej again only after this swap's last barrier
            if (sh.rej) {
                c.sync();
                return 1;
            }
            zsort_apply(p, sh.s, 0, tid, nth);
            c.sync();  // the 2x2 block takes the column rotation before the row rotation
            zsort_apply(p, sh.s, 1, tid, nth);
            c.sync();
            zsort_apply(p, sh.s, 2, tid, nth);
            c.sync();
        }
        ks++;
    }
    return 0;
}

// ZTGSEN's normalisation after a complete reordering (0 < M < n): B(k, k) made real and
// non-negative row by row, Q's columns with it; alpha = diag(A), beta = diag(B).  Ends with a
// barrier.
template <class R, class Cta>
XTG_HD void tgsen_cplx_normalize(const Cta &c, const ZPencil<R> &p, zc<R> *alpha, zc<R> *beta)
{
    const int n = p.n, tid = c.tid(), nth = c.nth();
    auto A = [&](int i, int j) -> zc<R> & { return p.A[(size_t)i + (size_t)j * p.lda]; };
    auto B = [&](int i, int j) -> zc<R> & { return p.B[(size_t)i + (size_t)j * p.ldb]; };
    auto Q = [&](int i, int j) -> zc<R> & { return p.Q[(size_t)i + (size_t)j * p.ldq]; };
    // pass 1: each row's factor t into alpha and d into beta (d = -1: no scaling)
    const R safmin = Mach<R>::sfmin;
    for (int k = tid; k < n; k += nth) {
        const zc<R> bkk = B(k, k);
        const R d = cabs(bkk);
        if (d > safmin) {
            alpha[k] = conj(mk(bkk.re / d, bkk.im / d));
            beta[k] = mk(d, R(0));
        } else {
            beta[k] = mk(R(-1), R(0));
        }
    }
    c.sync();
    // pass 2: the row scalings (column by column, row k by thread k mod nth) and Q's columns
    for (int col = 0; col < n; col++) {
        for (int k = tid; k <= col; k += nth) {
            const R d = beta[k].re;
            if (d < R(0)) {
                if (k == col) B(k, k) = mk(R(0), R(0));
                continue;
            }
            const zc<R> t = alpha[k];
            A(k, col) = t * A(k, col);
            B(k, col) = k == col ? mk(d, R(0)) : t * B(k, col);
        }
    }
    if (p.wantq)
        for (int k = 0; k < n; k++) {
            if (beta[k].re < R(0)) continue;
            const zc<R> t2 = conj(alpha[k]);
            for (int i = tid; i < n; i += nth) Q(i, k) = t2 * Q(i, k);
        }
    c.sync();
    // pass 3: alpha = diag(A), beta = diag(B)
    for (int k = tid; k < n; k += nth) {
        alpha[k] = A(k, k);
        beta[k] = B(k, k);
    }
    c.sync();
}

// ZTGSEN with IJOB = 0: returns INFO, 0 or 1 (a swap was rejected).  Every thread returns the
// same value, after a barrier.  alpha, beta: n each.
template <class R, class Cta>
XTG_HD int tgsen_cplx_cta(const Cta &c, ZSortShared<R> &sh, const ZPencil<R> &p, const int *select, zc<R> *alpha,
                          zc<R> *beta)
{
    const int info = tgsen_cplx_reorder(c, sh, p, select, alpha, beta);
    int m = 0;
    for (int k = 0; k < p.n; k++) m += select[k] != 0 ? 1 : 0;
    if (info == 0 && m > 0 && m < p.n) tgsen_cplx_normalize(c, p, alpha, beta);
    return info;
}

// ZTGSEN's estimates (IJOB 1 to 5) on the reordered pencil before its normalisation, as
// tgsen_real_estimates with ZTGSYL (TRANS = 'N' and 'C') and ZLACN2.  work: 4 M (n - M)
// complex elements (2 M (n - M) for IJOB 1, 2, 4); cuts n / 2 + 4 ints.
template <class R, class Cta>
XTG_HD void tgsen_cplx_estimates(const Cta &c, ZSylvShared<R> &sh, const ZPencil<R> &p, int m, int ijob, int info,
                                 zc<R> *work, int *cuts, R *est)
{
    const int n = p.n, tid = c.tid(), nth = c.nth();
    const bool wantp = ijob == 1 || ijob == 4 || ijob == 5, wantd1 = ijob == 2 || ijob == 4,
               wantd2 = ijob == 3 || ijob == 5, wantd = wantd1 || wantd2;
    if (tid == 0)
        for (int k = 0; k < 4; k++) est[k] = R(0);
    if (info != 0 || (!wantp && !wantd)) {
        c.sync();
        return;
    }
    if (m == 0 || m == n) {
        if (tid == 0) {
            if (wantp) est[0] = est[1] = R(1);
            if (wantd) {
                R sc = R(0), sq = R(1);
                for (int j = 0; j < n; j++) {
                    zlassq(n, p.A + (size_t)j * p.lda, sc, sq);
                    zlassq(n, p.B + (size_t)j * p.ldb, sc, sq);
                }
                est[2] = est[3] = sc * xsqrt(sq);
            }
        }
        c.sync();
        return;
    }
    const int n1 = m, n2 = n - m;
    const size_t mn = (size_t)n1 * n2;
    zc<R> *W = work, *V = work + mn;
    const zc<R> *A11 = p.A, *B11 = p.B;
    const zc<R> *A22 = p.A + n1 + (size_t)n1 * p.lda, *B22 = p.B + n1 + (size_t)n1 * p.ldb;
    auto setup = [&](int mm, int nn, const zc<R> *a, const zc<R> *d, const zc<R> *b, const zc<R> *e) {
        if (tid == 0) {
            ZSylvG<R> &y = sh.y;
            y.m = mm;
            y.n = nn;
            y.A = a;
            y.D = d;
            y.B = b;
            y.E = e;
            y.lda = y.ldb = p.lda;
            y.ldd = y.lde = p.ldb;
            y.C = W;
            y.F = V;
            y.ldc = y.ldf = mm;
        }
        c.sync();
    };
    if (wantp) {
        for (size_t t = tid; t < mn; t += nth) {  // C = A12, F = B12
            const int i = (int)(t % n1), j = n1 + (int)(t / n1);
            W[t] = p.A[(size_t)i + (size_t)j * p.lda];
            V[t] = p.B[(size_t)i + (size_t)j * p.ldb];
        }
        setup(n1, n2, A11, B11, A22, B22);
        R unused = R(0);
        ztgsyl_cta(c, sh, 0, cuts, (zc<R> *)nullptr, &unused);
        if (tid == 0) {
            const R dscale = sh.scale;
            for (int k = 0; k < 2; k++) {
                R sc = R(0), sq = R(1);
                zlassq((int)mn, k == 0 ? W : V, sc, sq);
                R v = sc * xsqrt(sq);
                v = v == R(0) ? R(1) : dscale / (xsqrt(dscale * dscale / v + v) * xsqrt(v));
                est[k] = v;
            }
        }
        c.sync();
    }
    if (wantd1) {
        setup(n1, n2, A11, B11, A22, B22);
        ztgsyl_cta(c, sh, 3, cuts, (zc<R> *)nullptr, est + 2);
        setup(n2, n1, A22, B22, A11, B11);
        ztgsyl_cta(c, sh, 3, cuts, (zc<R> *)nullptr, est + 3);
    }
    if (wantd2) {  // ZLACN2 on [vec C; vec F] = work[0, 2 mn), its v in work[2 mn, 4 mn)
        const int mn2 = (int)(2 * mn);
        zc<R> *Vl = work + 2 * mn;
        for (int which = 0; which < 2; which++) {
            if (tid == 0) {
                sh.lac.kase = 0;
                zlacn2(mn2, Vl, W, sh.lac);
            }
            c.sync();
            R dscale = R(1);
            for (int step = 0; step < 16; step++) {  // ZLACN2 asks for at most 11 products
                const int kase = sh.lac.kase;
                if (kase == 0) break;
                if (which == 0) setup(n1, n2, A11, B11, A22, B22);
                else setup(n2, n1, A22, B22, A11, B11);
                R unused = R(0);
                if (kase == 1) ztgsyl_cta(c, sh, 0, cuts, (zc<R> *)nullptr, &unused);
                else ztgsyl_c_cta(c, sh, cuts);
                if (tid == 0) {
                    dscale = sh.scale;
                    zlacn2(mn2, Vl, W, sh.lac);
                }
                c.sync();
            }
            if (tid == 0) est[2 + which] = dscale / sh.lac.est;
            c.sync();
        }
    }
}

// ZTGSEN with IJOB 0, 1, 2 or 4: M (into *m_out from thread 0), the moves, the estimates, the
// normalisation.  Returns INFO.  est: PL, PR, DIF(1), DIF(2).
template <class R, class Cta>
XTG_HD int tgsen_cplx_full_cta(const Cta &c, ZSortShared<R> &shs, ZSylvShared<R> &shy, const ZPencil<R> &p,
                               const int *select, int ijob, zc<R> *alpha, zc<R> *beta, zc<R> *work, int *cuts, R *est,
                               int *m_out)
{
    int m = 0;
    for (int k = 0; k < p.n; k++) m += select[k] != 0 ? 1 : 0;
    if (m_out && c.tid() == 0) *m_out = m;
    const int info = tgsen_cplx_reorder(c, shs, p, select, alpha, beta);
    tgsen_cplx_estimates(c, shy, p, m, ijob, info, work, cuts, est);
    if (info == 0 && m > 0 && m < p.n) tgsen_cplx_normalize(c, p, alpha, beta);
    return info;
}

// ---- xGGES's check of the reordered eigenvalues (host code) ---------------------------------

// Real pencils (DGGES): SELCTG on every eigenvalue after the reordering; returns SDIM, the
// number selected (a complex pair counts 2 when either of its values is selected), and sets
// *info = n + 2 when a selected eigenvalue follows one that is not.
template <class R, class SEL>
int gges_sdim_real(int n, SEL sel, const R *alphar, const R *alphai, const R *beta, int *info)
{
    bool lastsl = true, lst2sl = true;
    int sdim = 0, ip = 0;
    for (int i = 0; i < n; i++) {
        bool cursl = sel(&alphar[i], &alphai[i], &beta[i]) != 0;
        if (alphai[i] == R(0)) {
            if (cursl) sdim++;
            ip = 0;
            if (cursl && !lastsl) *info = n + 2;
        } else if (ip == 1) {  // the second value of a complex pair
            cursl = cursl || lastsl;
            lastsl = cursl;
            if (cursl) sdim += 2;
            ip = -1;
            if (cursl && !lst2sl) *info = n + 2;
        } else {  // the first value of a complex pair
            ip = 1;
        }
        lst2sl = lastsl;
        lastsl = cursl;
    }
    return sdim;
}

// Complex pencils (ZGGES): the same with one value per eigenvalue; alpha and beta as (re, im)
// pairs, SELCTG(alpha(i), beta(i)).
template <class R, class SEL>
int gges_sdim_cplx(int n, SEL sel, const zc<R> *alpha, const zc<R> *beta, int *info)
{
    bool lastsl = true;
    int sdim = 0;
    for (int i = 0; i < n; i++) {
        const bool cursl = sel(&alpha[i].re, &beta[i].re) != 0;
        if (cursl) sdim++;
        if (cursl && !lastsl) *info = n + 2;
        lastsl = cursl;
    }
    return sdim;
}

}  // namespace rb
}  // namespace xtg
