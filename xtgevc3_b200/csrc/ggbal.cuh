// Permutation balancing of a pencil (LAPACK xGGBAL with JOB = 'P', the first step of xGGES) and
// its back-transformation of the Schur vectors (xGGBAK with JOB = 'P').  Host and device code:
// the kernels in qz.cu run these bodies on one CTA; the tests run them on host threads.
//
// xGGBAL 'P' isolates eigenvalues: with the active rows / columns [K, L] (1-based, start 1, n),
// it looks for a row I (from L down to 1) whose entries in columns 1..L of A and B are zero
// except in at most one column J; it swaps rows I and L (columns K..n) and columns J and L
// (rows 1..L), records LSCALE(L) = I, RSCALE(L) = J and repeats with L - 1 (L = 1: done).  When
// no row qualifies it looks for a column J (from K up to L) whose entries in rows K..L are zero
// except in at most one row I; it swaps rows I and K and columns J and K, records LSCALE(K) =
// I, RSCALE(K) = J and repeats with K + 1.  ILO = K, IHI = L: outside [ILO, IHI] the pencil is
// upper triangular, so those eigenvalues are isolated.  LSCALE = RSCALE = 1 on [ILO, IHI], as
// xGGBAL with JOB = 'P' leaves them; the permuted rows and columns are exact copies.
//
// B200 form: one CTA.  Each search step checks every candidate row (or column) in parallel,
// a shared reduction picks the one xGGBAL's loop meets first (the largest row, the smallest
// column), and the CTA swaps the two rows and the two columns; at most n steps.
#pragma once

#include "tgsna_dif_cplx.cuh"

namespace xtg {
namespace rb {

XTG_HD inline bool nz_(double v) { return v != 0.0; }
XTG_HD inline bool nz_(float v) { return v != 0.0f; }
template <class R>
XTG_HD inline bool nz_(zc<R> v)
{
    return v.re != R(0) || v.im != R(0);
}

template <class E>
struct BalPencil {
    int n;
    E *A, *B;
    int lda, ldb;
};

// the CTA's shared state of ggbal_cta
struct BalShared {
    int k, l, best, bestj, phase;  // phase 1: rows, 2: columns, 0: done
};

// Row I of the active block qualifies when A(I, 1..L), B(I, 1..L) hold at most one nonzero
// column; *j the column (L when there is none), as xGGBAL's scan finds it
template <class E>
XTG_HD bool row_isolated(const BalPencil<E> &p, int i, int l, int *j)
{
    int first = -1;
    for (int c = 0; c < l; c++)
        if (nz_(p.A[(size_t)i + (size_t)c * p.lda]) || nz_(p.B[(size_t)i + (size_t)c * p.ldb])) {
            if (first >= 0) return false;
            first = c;
        }
    *j = (first < 0 || first == l - 1) ? l - 1 : first;
    return true;
}

// Column J qualifies when A(K..L, J), B(K..L, J) hold at most one nonzero row; *i the row
// (L when there is none)
template <class E>
XTG_HD bool col_isolated(const BalPencil<E> &p, int j, int k, int l, int *i)
{
    int first = -1;
    for (int r = k; r < l; r++)
        if (nz_(p.A[(size_t)r + (size_t)j * p.lda]) || nz_(p.B[(size_t)r + (size_t)j * p.ldb])) {
            if (first >= 0) return false;
            first = r;
        }
    *i = (first < 0 || first == l - 1) ? l - 1 : first;
    return true;
}

// xGGBAL 'P' on one CTA: lscale, rscale (n each, 1-based indices as xGGBAL stores them) for
// the isolated rows / columns; *ilo, *ihi (1-based) from thread 0; red: 2 nth ints of scratch
// for the per-thread candidates.  Ends with a barrier.
template <class E, class R, class Cta>
XTG_HD void ggbal_cta(const Cta &c, BalShared &sh, const BalPencil<E> &p, R *lscale, R *rscale, int *ilo, int *ihi,
                      int *red)
{
    const int n = p.n, tid = c.tid(), nth = c.nth();
    auto A = [&](int i, int j) -> E & { return p.A[(size_t)i + (size_t)j * p.lda]; };
    auto B = [&](int i, int j) -> E & { return p.B[(size_t)i + (size_t)j * p.ldb]; };
    if (tid == 0) {
        sh.k = 0;      // 0-based K
        sh.l = n;      // L as a count: active rows / columns [k, l)
        sh.phase = n == 1 ? 0 : 1;
        if (n == 1) {
            lscale[0] = R(1);
            rscale[0] = R(1);
        }
    }
    c.sync();
    for (int step = 0; step < 2 * n + 2; step++) {
        const int phase = sh.phase, k = sh.k, l = sh.l;
        if (phase == 0) break;
        // candidates: rows l-1 .. 0 (the largest qualifying wins), or columns k .. l-1 (the
        // smallest wins); thread t checks candidates t, t + nth, ...
        const int count = phase == 1 ? l : l - k;
        int mine = phase == 1 ? -1 : n, minej = -1;
        for (int t = tid; t < count; t += nth) {
            int other;
            if (phase == 1) {
                const int i = t;
                if (i > mine && row_isolated(p, i, l, &other)) {
                    mine = i;
                    minej = other;
                }
            } else {
                const int j = k + t;
                if (j < mine && col_isolated(p, j, k, l, &other)) {
                    mine = j;
                    minej = other;
                }
            }
        }
        red[2 * tid] = mine;
        red[2 * tid + 1] = minej;
        c.sync();  // every candidate is in red before thread 0 picks the first in xGGBAL's order
        if (tid == 0) {
            int b = phase == 1 ? -1 : n, bj = -1;
            for (int t = 0; t < nth; t++)
                if ((phase == 1 && red[2 * t] > b) || (phase == 2 && red[2 * t] < b)) {
                    b = red[2 * t];
                    bj = red[2 * t + 1];
                }
            sh.best = b;
            sh.bestj = bj;
        }
        c.sync();
        const int best = sh.best, bestj = sh.bestj;
        if ((phase == 1 && best < 0) || (phase == 2 && best >= n)) {  // no candidate
            if (tid == 0) sh.phase = phase == 1 ? 2 : 0;
            c.sync();
            continue;
        }
        // rows: I = best <-> L - 1 over columns k..n-1, then columns J = bestj <-> L - 1 over
        // rows 0..l-1; columns: row bestj <-> K (columns k..n-1), column best <-> K (rows 0..l-1)
        const int ri = phase == 1 ? best : bestj, cj = phase == 1 ? bestj : best, m = phase == 1 ? l - 1 : k;
        if (ri != m)
            for (int col = k + tid; col < n; col += nth) {
                E t1 = A(ri, col), t2 = B(ri, col);
                A(ri, col) = A(m, col);
                B(ri, col) = B(m, col);
                A(m, col) = t1;
                B(m, col) = t2;
            }
        c.sync();
        if (cj != m)
            for (int row = tid; row < l; row += nth) {
                E t1 = A(row, cj), t2 = B(row, cj);
                A(row, cj) = A(row, m);
                B(row, cj) = B(row, m);
                A(row, m) = t1;
                B(row, m) = t2;
            }
        if (tid == 0) {
            lscale[m] = R(ri + 1);
            rscale[m] = R(cj + 1);
            if (phase == 1) {
                sh.l = l - 1;
                if (l - 1 == 1) {  // xGGBAL: L = 1 ends the search with ILO = IHI = 1
                    lscale[0] = R(1);
                    rscale[0] = R(1);
                    sh.phase = 0;
                }
            } else {
                sh.k = k + 1;
            }
        }
        c.sync();
    }
    if (tid == 0) {
        *ilo = sh.k + 1;
        *ihi = sh.l;
    }
    for (int i = sh.k + tid; i < sh.l; i += nth) {
        lscale[i] = R(1);
        rscale[i] = R(1);
    }
    c.sync();
}

// xGGBAK 'P' for V (n x m, leading dimension ldv; m = n for the Schur vectors): rows ilo-1 .. 1
// and ihi+1 .. n (1-based) swapped with the rows scale records, in that order.  Ends with a
// barrier.
template <class E, class R, class Cta>
XTG_HD void ggbak_cta(const Cta &c, int n, int ilo, int ihi, const R *scale, E *V, int ldv, int m = -1)
{
    const int tid = c.tid(), nth = c.nth();
    const int cols = m < 0 ? n : m;
    auto swap_rows = [&](int i, int k) {
        for (int col = tid; col < cols; col += nth) {
            E t = V[(size_t)i + (size_t)col * ldv];
            V[(size_t)i + (size_t)col * ldv] = V[(size_t)k + (size_t)col * ldv];
            V[(size_t)k + (size_t)col * ldv] = t;
        }
        c.sync();
    };
    // a recorded row outside 1..n (scales not made by xGGBAL) is skipped: no access outside V
    for (int i = ilo - 1; i >= 1; i--) {
        const int k = (int)scale[i - 1];
        if (k != i && k >= 1 && k <= n) swap_rows(i - 1, k - 1);
    }
    for (int i = ihi + 1; i <= n; i++) {
        const int k = (int)scale[i - 1];
        if (k != i && k >= 1 && k <= n) swap_rows(i - 1, k - 1);
    }
    c.sync();
}

}  // namespace rb
}  // namespace xtg
