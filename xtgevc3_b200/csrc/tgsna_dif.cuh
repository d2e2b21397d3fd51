// DIF of LAPACK D/STGSNA (JOB = 'V' / 'B'): the estimated reciprocal condition number of the
// eigenvectors of a real generalized Schur pencil (A, B), per selected eigenvalue (1x1 block)
// or complex pair (2x2 block), following DTGSNA's own steps:
//   1. a copy of (A, B) reordered so that the block comes first (xTGEXC, no Q or Z; a
//      rejected swap gives DIF = 0);
//   2. with (A11, B11) that n1 x n1 block and (A22, B22) the rest, the generalized Sylvester
//      operator  (R, L) -> (A22 R - L A11, B22 R - L B11)  and xTGSYL's Frobenius-norm
//      estimate of its smallest singular value (IJOB = 3): the substitution of xTGSYL /
//      xTGSY2 over A22's diagonal blocks, bottom to top, where each block's Kronecker system
//      (LU with complete pivoting, xGETC2) is solved by xLATDF for a right-hand side of the
//      current residual plus +-1 entries chosen by look-ahead to make the solution large;
//      DIF = sqrt(2 n1 n2) / ||all solutions||_F;
//   3. for a complex pair, DIF = min(DIF, the pair's own bound from its 2x2 eigenvalue
//      problem, xLAG2); n2 = 0 gives that bound alone; n = 1 gives |(A, B)|.
// xTGSYL's blocks are those of LAPACK's ILAENV for xTGSYL (2 rows, one more when the cut
// would split a 2x2 block; the 1x1 / 2x2 block A11 is one block); inside a block xTGSY2
// substitutes its 1x1 / 2x2 diagonal blocks and updates the block's own rows, then the rows
// above the block take the block's solution at once.  The +-1 choices depend on the
// residuals, so the estimate agrees with LAPACK's to rounding as long as no choice is a
// near tie.
//
// Host and device code like tgexc_real_blocks.cuh: the GPU kernel runs one CTA per
// eigenvalue (thread 0 for the small systems, the CTA for the O(n) row updates); the tests
// compile this header for the CPU and compare with LAPACK.
#pragma once

#include "tgexc_real_blocks.cuh"

namespace xtg {
namespace rb {

// Sum-of-squares accumulation scale^2 * sumsq += sum x_i^2 (xLASSQ)
template <class R>
XTG_HD void lassq(int n, const R *x, R &scale, R &sumsq)
{
    for (int i = 0; i < n; i++) {
        if (x[i] != R(0)) {
            const R a = xabs(x[i]);
            if (scale < a) {
                const R q = scale / a;
                sumsq = R(1) + sumsq * q * q;
                scale = a;
            } else {
                const R q = a / scale;
                sumsq += q * q;
            }
        }
    }
}

// xLATDF with the look-ahead strategy (IJOB != 2): with Z = P^T L U Q^T from getc2, solve
// Z x = b where b = rhs + (+-1 entries) is chosen entry by entry to make x large, x into rhs,
// and add ||x||^2 to (rdscal, rdsum).
template <class R>
XTG_HD void latdf(int n, const R *Z, R *rhs, R &rdsum, R &rdscal, const int *ipiv, const int *jpiv)
{
    for (int i = 0; i < n - 1; i++)
        if (ipiv[i] != i) {
            const R t = rhs[i];
            rhs[i] = rhs[ipiv[i]];
            rhs[ipiv[i]] = t;
        }
    R pmone = R(-1);
    for (int j = 0; j < n - 1; j++) {
        const R bp = rhs[j] + R(1), bm = rhs[j] - R(1);
        R splus = R(1), sminu = R(0);
        for (int k = j + 1; k < n; k++) splus += Z[k + 8 * j] * Z[k + 8 * j];
        for (int k = j + 1; k < n; k++) sminu += Z[k + 8 * j] * rhs[k];
        splus *= rhs[j];
        if (splus > sminu) {
            rhs[j] = bp;
        } else if (sminu > splus) {
            rhs[j] = bm;
        } else {  // equal updating sums: -1 the first time, +1 after that
            rhs[j] += pmone;
            pmone = R(1);
        }
        const R t = -rhs[j];
        for (int k = j + 1; k < n; k++) rhs[k] += t * Z[k + 8 * j];
    }
    R xp[8];
    for (int i = 0; i < n - 1; i++) xp[i] = rhs[i];
    xp[n - 1] = rhs[n - 1] + R(1);
    rhs[n - 1] -= R(1);
    R splus = R(0), sminu = R(0);
    for (int i = n - 1; i >= 0; i--) {
        const R t = R(1) / Z[i + 8 * i];
        xp[i] *= t;
        rhs[i] *= t;
        for (int k = i + 1; k < n; k++) {
            xp[i] -= xp[k] * (Z[i + 8 * k] * t);
            rhs[i] -= rhs[k] * (Z[i + 8 * k] * t);
        }
        splus += xabs(xp[i]);
        sminu += xabs(rhs[i]);
    }
    if (splus > sminu)
        for (int i = 0; i < n; i++) rhs[i] = xp[i];
    for (int i = n - 2; i >= 0; i--)
        if (jpiv[i] != i) {
            const R t = rhs[i];
            rhs[i] = rhs[jpiv[i]];
            rhs[jpiv[i]] = t;
        }
    lassq(n, rhs, rdscal, rdsum);
}

// The reordered pencil seen as xTGSYL's operands (column-major, leading dimension ld):
// A22 = A[n1:, n1:], B22 = B[n1:, n1:] (the n2 x n2 rest), A11, B11 (n1 x n1, in A11s / B11s
// with leading dimension LD), and the n2 x n1 right-hand sides C, F (leading dimension ldc).
template <class R>
struct Sylv {
    int n1, n2, ld, ldc;
    const R *A22, *B22;
    R A11s[16], B11s[16];
    R *C, *F;
    R dsum, dscale;
};

// One xTGSYL block: rows [is, ie] of A22 (0-based), xTGSY2 with IJOB = 1 over it: its 1x1 /
// 2x2 diagonal blocks bottom to top, each solved by getc2 + latdf, the block's own rows above
// it updated.  Returns getc2's INFO (> 0: a pivot was raised).
template <class R>
XTG_HD int tgsyl_block(Sylv<R> &y, int is, int ie)
{
    const int n1 = y.n1, ld = y.ld, ldc = y.ldc;
    auto a = [&](int i, int k) { return y.A22[(size_t)i + (size_t)k * ld]; };
    auto d = [&](int i, int k) { return y.B22[(size_t)i + (size_t)k * ld]; };
    int starts[4], nb = 0;
    for (int i = is; i <= ie;) {
        starts[nb++] = i;
        i += (i < ie && a(i + 1, i) != R(0)) ? 2 : 1;
    }
    int info = 0;
    for (int b = nb - 1; b >= 0; b--) {
        const int s0 = starts[b], mb = (b + 1 < nb ? starts[b + 1] : ie + 1) - s0;
        const int nn = mb * n1, zdim = 2 * nn;
        R Z[64], rhs[8];
        for (int i = 0; i < 64; i++) Z[i] = R(0);
        for (int j = 0; j < n1; j++)
            for (int i = 0; i < mb; i++) {
                const int k = i + mb * j;
                for (int p = 0; p < mb; p++) {
                    Z[k + 8 * (p + mb * j)] = a(s0 + i, s0 + p);
                    if (p >= i) Z[(nn + k) + 8 * (p + mb * j)] = d(s0 + i, s0 + p);
                }
                for (int q = 0; q < n1; q++) {
                    Z[k + 8 * (nn + i + mb * q)] = -y.A11s[q + LD * j];
                    if (q <= j) Z[(nn + k) + 8 * (nn + i + mb * q)] = -y.B11s[q + LD * j];
                }
                rhs[k] = y.C[(s0 + i) + (size_t)j * ldc];
                rhs[nn + k] = y.F[(s0 + i) + (size_t)j * ldc];
            }
        int ipiv[8], jpiv[8];
        const int ierr = getc2(zdim, Z, ipiv, jpiv);
        if (ierr > 0) info = ierr;
        latdf(zdim, Z, rhs, y.dsum, y.dscale, ipiv, jpiv);
        for (int j = 0; j < n1; j++)
            for (int i = 0; i < mb; i++) {
                y.C[(s0 + i) + (size_t)j * ldc] = rhs[i + mb * j];
                y.F[(s0 + i) + (size_t)j * ldc] = rhs[nn + i + mb * j];
            }
        // rows [is, s0) of this xTGSYL block: C -= A22 R, F -= B22 R
        for (int r = is; r < s0; r++)
            for (int j = 0; j < n1; j++) {
                R c = y.C[r + (size_t)j * ldc], f = y.F[r + (size_t)j * ldc];
                for (int p = 0; p < mb; p++) {
                    const R rv = rhs[p + mb * j];
                    c -= a(r, s0 + p) * rv;
                    f -= d(r, s0 + p) * rv;
                }
                y.C[r + (size_t)j * ldc] = c;
                y.F[r + (size_t)j * ldc] = f;
            }
    }
    return info;
}

// Rows [0, is) after the xTGSYL block [is, ie]: C -= A22[:, is:ie] R, F -= B22[:, is:ie] R,
// rows tid, tid + nth, ...
template <class R>
XTG_HD void tgsyl_update_above(Sylv<R> &y, int is, int ie, int tid, int nth)
{
    const int ld = y.ld, ldc = y.ldc;
    for (int r = tid; r < is; r += nth)
        for (int j = 0; j < y.n1; j++) {
            R c = y.C[r + (size_t)j * ldc], f = y.F[r + (size_t)j * ldc];
            for (int p = is; p <= ie; p++) {
                const R rv = y.C[p + (size_t)j * ldc];
                c -= y.A22[(size_t)r + (size_t)p * ld] * rv;
                f -= y.B22[(size_t)r + (size_t)p * ld] * rv;
            }
            y.C[r + (size_t)j * ldc] = c;
            y.F[r + (size_t)j * ldc] = f;
        }
}

// xTGSYL's block starts of A22 (ILAENV's 2-row blocks, one row more where a cut would split a
// 2x2 block); returns the count, starts[count] = n2.  starts has room for n2 / 2 + 2 entries.
template <class R>
XTG_HD int tgsyl_blocks(const Sylv<R> &y, int *starts)
{
    const int m = y.n2, ld = y.ld;
    if (m <= 2) {  // M <= MB and N <= NB: xTGSYL's unblocked solver, one block
        starts[0] = 0;
        starts[1] = m;
        return 1;
    }
    int p = 0, i = 1;  // 1-based as xTGSYL
    while (i <= m) {
        starts[p++] = i - 1;
        i += 2;
        if (i >= m) break;
        if (y.A22[(size_t)(i - 1) + (size_t)(i - 2) * ld] != R(0)) i++;
    }
    starts[p] = m;
    if (starts[p - 1] == starts[p]) p--;
    return p;
}

// The bound of a complex pair from its own 2x2 block (DTGSNA): min singular value of the
// 2x2 pencil's Kronecker form from alpha / beta of xLAG2.
template <class R>
XTG_HD R pair_cond(R a00, R a10, R a01, R a11, R b00, R b10, R b01, R b11)
{
    R A[16] = {}, B[16] = {};
    A[0] = a00;
    A[1] = a10;
    A[LD] = a01;
    A[1 + LD] = a11;
    B[0] = b00;
    B[1] = b10;
    B[LD] = b01;
    B[1 + LD] = b11;
    R beta, scale2, alphar, wr2, alphai;
    lag2(A, B, Mach<R>::sfmin, beta, scale2, alphar, wr2, alphai);
    const R c1 = R(2) * (alphar * alphar + alphai * alphai + beta * beta);
    const R c2 = R(4) * beta * beta * alphai * alphai;
    const R root1 = (c1 + xsqrt(c1 * c1 - R(4) * c2)) / R(2);
    const R root2 = c2 / root1;
    return xmin(xsqrt(root1), xsqrt(root2));
}

// DIF from the reordered copy (A, B with the block first, leading dimension ld) on one thread
// (the tests' CPU build; the kernel splits the same steps between thread 0 and the CTA).
// C, F: scratch of n rows x 2 (leading dimension ldc >= n); starts: n / 2 + 2 ints.
template <class R>
XTG_HD R dif_reordered_serial(int n, const R *A, const R *B, int ld, R *C, R *F, int ldc, int *starts)
{
    Sylv<R> y;
    y.n1 = (n > 1 && A[1] != R(0)) ? 2 : 1;
    y.n2 = n - y.n1;
    y.ld = ld;
    y.ldc = ldc;
    y.A22 = A + y.n1 + (size_t)y.n1 * ld;
    y.B22 = B + y.n1 + (size_t)y.n1 * ld;
    for (int k = 0; k < 16; k++) {
        y.A11s[k] = R(0);
        y.B11s[k] = R(0);
    }
    for (int j = 0; j < y.n1; j++)
        for (int i = 0; i < y.n1; i++) {
            y.A11s[i + LD * j] = A[i + (size_t)j * ld];
            y.B11s[i + LD * j] = B[i + (size_t)j * ld];
        }
    y.C = C;
    y.F = F;
    for (int j = 0; j < y.n1; j++)
        for (int i = 0; i < y.n2; i++) C[i + (size_t)j * ldc] = F[i + (size_t)j * ldc] = R(0);
    y.dsum = R(1);
    y.dscale = R(0);
    const int nbk = tgsyl_blocks(y, starts);
    for (int b = nbk - 1; b >= 0; b--) {
        tgsyl_block(y, starts[b], starts[b + 1] - 1);
        tgsyl_update_above(y, starts[b], starts[b + 1] - 1, 0, 1);
    }
    return xsqrt(R(2 * y.n1 * y.n2)) / (y.dscale * xsqrt(y.dsum));
}

// ---- the GPU kernel's body, one CTA ---------------------------------------------------------
// Written against a CTA context (see walk_cta in tgexc_real_blocks.cuh) so that the kernel
// (tgsna_dif.cu: shared memory, __syncthreads) and the tests (host threads with a barrier)
// run the same code.

// one selected block: its first row (0-based), the index of its DIF, whether a 2x2 block
struct DifItem {
    int k, ks, pair;
};

// workspace of one CTA in elements of R: the reordered copy (2 n^2), C and F (n x 2 each),
// xTGSYL's block starts (n / 2 + 4 ints in n + 8 elements of room)
XTG_HD inline size_t dif_work_elems(int n) { return 2 * (size_t)n * n + 4 * (size_t)n + (size_t)n + 8; }

// the CTA's shared state (shared memory on the GPU)
template <class R>
struct DifShared {
    WalkShared<R> walk;
    Sylv<R> y;
    int nbk;
    R cond, d;
};

// DIF of the items it = c.cta(), c.cta() + c.ncta(), ... of a real pencil (A, B): copy, walk
// the block to the top (walk_cta; *err = 1 if its swap bound were reached), xTGSYL's estimate
// (thread 0 solves each block, the CTA updates the rows above it).
template <class R, class Cta>
XTG_HD void dif_cta(const Cta &c, DifShared<R> &sh, int n, const R *A, int lda, const R *B, int ldb,
                    const DifItem *items, int count, R *dif, R *work, size_t per_cta, int *err)
{
    const int tid = c.tid(), nth = c.nth();
    R *Aw = work + (size_t)c.cta() * per_cta;
    R *Bw = Aw + (size_t)n * n;
    R *Cw = Bw + (size_t)n * n;
    R *Fw = Cw + 2 * (size_t)n;
    int *starts = reinterpret_cast<int *>(Fw + 2 * (size_t)n);
    for (int it = c.cta(); it < count; it += c.ncta()) {
        const DifItem item = items[it];
        if (n == 1) {
            if (tid == 0) dif[item.ks] = lapy2(A[0], B[0]);
            continue;
        }
        for (size_t e = tid; e < (size_t)n * n; e += nth) {
            const size_t i = e % n, j = e / n;
            Aw[e] = A[i + j * lda];
            Bw[e] = B[i + j * ldb];
        }
        for (int e = tid; e < 2 * n; e += nth) {
            Cw[e] = R(0);
            Fw[e] = R(0);
        }
        const Pencil<R> p{n, 0, 0, Aw, Bw, nullptr, nullptr, n, n, 1, 1};
        if (tid == 0) {
            const int k = item.k;
            sh.cond = R(0);
            if (item.pair)
                sh.cond = pair_cond(A[k + (size_t)k * lda], A[k + 1 + (size_t)k * lda], A[k + (size_t)(k + 1) * lda],
                                    A[k + 1 + (size_t)(k + 1) * lda], B[k + (size_t)k * ldb], B[k + 1 + (size_t)k * ldb],
                                    B[k + (size_t)(k + 1) * ldb], B[k + 1 + (size_t)(k + 1) * ldb]);
        }
        c.sync();  // the copy is complete before thread 0 reads it
        walk_cta(c, sh.walk, p, item.k + 1, 1);  // ends with a barrier
        if (tid == 0) {
            sh.nbk = 0;
            sh.d = R(0);  // a rejected swap: DIF = 0
            if (sh.walk.info == 3) *err = 1;
            if (sh.walk.info == 0) {
                const int n1 = Aw[1] != R(0) ? 2 : 1;
                if (n - n1 == 0) {
                    sh.d = sh.cond;
                } else {
                    Sylv<R> &y = sh.y;
                    y.n1 = n1;
                    y.n2 = n - n1;
                    y.ld = n;
                    y.ldc = n;
                    y.A22 = Aw + n1 + (size_t)n1 * n;
                    y.B22 = Bw + n1 + (size_t)n1 * n;
                    for (int q = 0; q < 16; q++) {
                        y.A11s[q] = R(0);
                        y.B11s[q] = R(0);
                    }
                    for (int j = 0; j < n1; j++)
                        for (int i = 0; i < n1; i++) {
                            y.A11s[i + LD * j] = Aw[i + (size_t)j * n];
                            y.B11s[i + LD * j] = Bw[i + (size_t)j * n];
                        }
                    y.C = Cw;
                    y.F = Fw;
                    y.dsum = R(1);
                    y.dscale = R(0);
                    sh.nbk = tgsyl_blocks(y, starts);
                }
            }
        }
        c.sync();
        const int nbk = sh.nbk;
        for (int b = nbk - 1; b >= 0; b--) {
            if (tid == 0) tgsyl_block(sh.y, starts[b], starts[b + 1] - 1);
            c.sync();
            tgsyl_update_above(sh.y, starts[b], starts[b + 1] - 1, tid, nth);
            c.sync();
        }
        if (tid == 0) {
            R d = sh.d;
            if (nbk > 0) {
                d = xsqrt(R(2 * sh.y.n1 * sh.y.n2)) / (sh.y.dscale * xsqrt(sh.y.dsum));
                if (item.pair) d = xmin(d, sh.cond);
            }
            dif[item.ks] = d;
            if (item.pair) dif[item.ks + 1] = d;
        }
        c.sync();  // the workspace is reused by the next item
    }
}

}  // namespace rb
}  // namespace xtg
