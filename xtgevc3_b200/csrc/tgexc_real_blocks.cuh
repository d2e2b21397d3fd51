// Eigenvalue reordering of a real generalized Schur pencil across 2x2 diagonal blocks (LAPACK
// D/STGEXC with its swaps D/STGEX2, general case): the swap of two adjacent diagonal blocks of
// sizes n1, n2 in {1, 2}, and the walk that moves a block from IFST to ILST swap by swap,
// including the case where a 2x2 block splits into two 1x1 blocks on the way.
//
// One swap of blocks (S11, S22), (T11, T22) with m = n1 + n2 > 2 is the direct swapping method
// (B. Kagstrom, "A direct method for reordering eigenvalues in the generalized real Schur form
// of a regular matrix pair (A, B)", 1993; B. Kagstrom and P. Poromaa, 1996):
//   1. solve the generalized Sylvester equation  S11 R - L S22 = scale S12,
//      T11 R - L T22 = scale T12  (a 2 n1 n2 Kronecker system, LU with complete pivoting);
//   2. orthogonal QL from the QR factorisation of [-L; scale I], QR from the RQ factorisation
//      of [scale I, R]; the tentative swap is (QL^T S QR^T, QL^T T QR^T);
//   3. re-triangularise T by an RQ and by a QR factorisation, keep the one whose S21 block is
//      smaller (the weak test: ||S21||_F <= 20 eps ||S||_F), then the strong test: the swapped
//      blocks transformed back must equal the originals within 20 eps ||.||_F;
//   4. standardise each new 2x2 block (LAPACK xLAGV2: B's block diagonal and positive for a
//      complex pair, or both triangular when its eigenvalues have become real).
// A rejected swap leaves the pencil as it is (INFO = 1).  Swaps of two 1x1 blocks use the two
// rotations of the 1x1 method.  The small-block arithmetic follows LAPACK's routines step by
// step (xTGSY2 with xGETC2 / xGESC2, xGEQR2 / xORG2R / xORM2R, xGERQ2 / xORGR2 / xORMR2,
// xLAGV2 with xLAG2 and xLASV2, xLARTG, xLARFG) so that the results agree with LAPACK's to
// rounding.
//
// Everything here is host and device code: the reordering kernel runs one swap's small-block
// arithmetic on one thread and the O(n) updates of the swap on the whole CTA; the tests also
// compile this header for the CPU and compare single swaps and whole moves with LAPACK.
#pragma once

#include <math.h>

#ifdef __CUDACC__
#define XTG_HD __host__ __device__
#else
#define XTG_HD
#endif

namespace xtg {
namespace rb {

// LAPACK's machine constants: xLAMCH('P') (eps * base), xLAMCH('E') (eps), xLAMCH('S').
template <class R> struct Mach;
template <> struct Mach<double> {
    static constexpr double prec = 2.220446049250313080847e-16;   // 2^-52
    static constexpr double epsr = 1.110223024625156540424e-16;   // 2^-53
    static constexpr double sfmin = 2.225073858507201383090e-308; // 2^-1022
};
template <> struct Mach<float> {
    static constexpr float prec = 1.1920928955078125e-7f;  // 2^-23
    static constexpr float epsr = 5.9604644775390625e-8f;  // 2^-24
    static constexpr float sfmin = 1.1754943508222875e-38f; // 2^-126
};

XTG_HD inline double xsqrt(double x) { return sqrt(x); }
XTG_HD inline float xsqrt(float x) { return sqrtf(x); }
XTG_HD inline double xabs(double x) { return fabs(x); }
XTG_HD inline float xabs(float x) { return fabsf(x); }
XTG_HD inline double xsign(double a, double b) { return copysign(a, b); }
XTG_HD inline float xsign(float a, float b) { return copysignf(a, b); }
XTG_HD inline double xmax(double a, double b) { return fmax(a, b); }
XTG_HD inline float xmax(float a, float b) { return fmaxf(a, b); }
XTG_HD inline double xmin(double a, double b) { return fmin(a, b); }
XTG_HD inline float xmin(float a, float b) { return fminf(a, b); }
XTG_HD inline double xhypot(double a, double b) { return hypot(a, b); }
XTG_HD inline float xhypot(float a, float b) { return hypotf(a, b); }
XTG_HD inline bool xfinite(double a) { return isfinite(a); }
XTG_HD inline bool xfinite(float a) { return isfinite(a); }
// products and differences rounded one by one (no fused multiply-add), as LAPACK forms the
// 1x1 swap's F and G
XTG_HD inline double mul_rn(double a, double b)
{
#ifdef __CUDA_ARCH__
    return __dmul_rn(a, b);
#else
    return a * b;
#endif
}
XTG_HD inline float mul_rn(float a, float b)
{
#ifdef __CUDA_ARCH__
    return __fmul_rn(a, b);
#else
    return a * b;
#endif
}
XTG_HD inline double sub_rn(double a, double b)
{
#ifdef __CUDA_ARCH__
    return __dsub_rn(a, b);
#else
    return a - b;
#endif
}
XTG_HD inline float sub_rn(float a, float b)
{
#ifdef __CUDA_ARCH__
    return __fsub_rn(a, b);
#else
    return a - b;
#endif
}

// Small matrices are column-major with leading dimension 4 (m <= 4).
constexpr int LD = 4;

// sqrt(x^2 + y^2) without overflow (xLAPY2)
template <class R>
XTG_HD R lapy2(R x, R y)
{
    if (x != x) return x;
    if (y != y) return y;
    const R xa = xabs(x), ya = xabs(y), w = xmax(xa, ya), z = xmin(xa, ya);
    if (z == R(0) || !xfinite(w)) return w;
    const R q = z / w;
    return w * xsqrt(R(1) + q * q);
}

// Frobenius norm of cnt values at p[0], p[inc], ... by a running scaled sum of squares
template <class R>
XTG_HD R fro(const R *p, int cnt, int inc = 1)
{
    R scale = R(0), ssq = R(1);
    for (int i = 0; i < cnt; i++) {
        const R v = p[i * inc];
        if (v != R(0)) {
            const R a = xabs(v);
            if (scale < a) {
                const R q = scale / a;
                ssq = R(1) + ssq * q * q;
                scale = a;
            } else {
                const R q = a / scale;
                ssq += q * q;
            }
        }
    }
    return scale * xsqrt(ssq);
}

// Frobenius norm of the rows x cols block at M (leading dimension LD)
template <class R>
XTG_HD R fro_block(const R *M, int rows, int cols)
{
    R v[16];
    int k = 0;
    for (int j = 0; j < cols; j++)
        for (int i = 0; i < rows; i++) v[k++] = M[i + LD * j];
    return fro(v, k);
}

// Plane rotation [c s; -s c] [f; g] = [r; 0], c >= 0, r of f's sign, computed in range (xLARTG)
template <class R>
XTG_HD void lartg(R f, R g, R &c, R &s, R &r)
{
    const R safmin = Mach<R>::sfmin, safmax = R(1) / safmin;
    const R rtmin = xsqrt(safmin), rtmax = xsqrt(safmax / R(2));
    const R f1 = xabs(f), g1 = xabs(g);
    if (g == R(0)) {
        c = R(1);
        s = R(0);
        r = f;
    } else if (f == R(0)) {
        c = R(0);
        s = xsign(R(1), g);
        r = g1;
    } else if (f1 > rtmin && f1 < rtmax && g1 > rtmin && g1 < rtmax) {
        const R d = xsqrt(f * f + g * g);
        c = f1 / d;
        r = xsign(d, f);
        s = g / r;
    } else {
        const R u = xmin(safmax, xmax(safmin, xmax(f1, g1)));
        const R fs = f / u, gs = g / u, d = xsqrt(fs * fs + gs * gs);
        c = xabs(fs) / d;
        r = xsign(d, f);
        s = gs / r;
        r = r * u;
    }
}

// (x, y) <- (c x + s y, c y - s x)
template <class R>
XTG_HD inline void rot(R &x, R &y, R c, R s)
{
    const R xn = c * x + s * y, yn = c * y - s * x;
    x = xn;
    y = yn;
}

// Elementary reflector H = I - tau v v^T with H [alpha; x] = [beta; 0], v = [1; x'] (xLARFG):
// alpha becomes beta, x becomes x'.
template <class R>
XTG_HD void larfg(int n, R &alpha, R *x, int incx, R &tau)
{
    if (n <= 1) {
        tau = R(0);
        return;
    }
    R xnorm = fro(x, n - 1, incx);
    if (xnorm == R(0)) {
        tau = R(0);
        return;
    }
    R beta = -xsign(lapy2(alpha, xnorm), alpha);
    const R safmin = Mach<R>::sfmin / Mach<R>::epsr;
    int knt = 0;
    if (xabs(beta) < safmin) {
        const R rsafmn = R(1) / safmin;
        do {
            knt++;
            for (int i = 0; i < n - 1; i++) x[i * incx] *= rsafmn;
            beta *= rsafmn;
            alpha *= rsafmn;
        } while (xabs(beta) < safmin && knt < 20);
        xnorm = fro(x, n - 1, incx);
        beta = -xsign(lapy2(alpha, xnorm), alpha);
    }
    tau = (beta - alpha) / beta;
    const R sc = R(1) / (alpha - beta);
    for (int i = 0; i < n - 1; i++) x[i * incx] *= sc;
    for (int j = 0; j < knt; j++) beta *= safmin;
    alpha = beta;
}

// C (m x n at C, leading dimension LD) <- H C with H = I - tau v v^T (xLARF, side L)
template <class R>
XTG_HD void larf_left(int m, int n, const R *v, int incv, R tau, R *C)
{
    if (tau == R(0)) return;
    for (int j = 0; j < n; j++) {
        R w = R(0);
        for (int i = 0; i < m; i++) w += C[i + LD * j] * v[i * incv];
        const R t = -tau * w;
        for (int i = 0; i < m; i++) C[i + LD * j] += v[i * incv] * t;
    }
}

// C (m x n) <- C H (xLARF, side R)
template <class R>
XTG_HD void larf_right(int m, int n, const R *v, int incv, R tau, R *C)
{
    if (tau == R(0)) return;
    R w[4];
    for (int i = 0; i < m; i++) w[i] = R(0);
    for (int j = 0; j < n; j++)
        for (int i = 0; i < m; i++) w[i] += C[i + LD * j] * v[j * incv];
    for (int j = 0; j < n; j++) {
        const R t = -tau * v[j * incv];
        for (int i = 0; i < m; i++) C[i + LD * j] += w[i] * t;
    }
}

// QR factorisation of the m x n matrix A = Q R, Q = H(0) ... H(k-1) (xGEQR2): R in the upper
// triangle, reflector i below the diagonal of column i.
template <class R>
XTG_HD void geqr2(int m, int n, R *A, R *tau)
{
    const int k = m < n ? m : n;
    for (int i = 0; i < k; i++) {
        larfg(m - i, A[i + LD * i], &A[(i + 1 < m ? i + 1 : m - 1) + LD * i], 1, tau[i]);
        if (i < n - 1) {
            const R aii = A[i + LD * i];
            A[i + LD * i] = R(1);
            larf_left(m - i, n - i - 1, &A[i + LD * i], 1, tau[i], &A[i + LD * (i + 1)]);
            A[i + LD * i] = aii;
        }
    }
}

// The first n columns of Q = H(0) ... H(k-1) from geqr2, in place (xORG2R)
template <class R>
XTG_HD void org2r(int m, int n, int k, R *A, const R *tau)
{
    for (int j = k; j < n; j++) {
        for (int l = 0; l < m; l++) A[l + LD * j] = R(0);
        A[j + LD * j] = R(1);
    }
    for (int i = k - 1; i >= 0; i--) {
        if (i < n - 1) {
            A[i + LD * i] = R(1);
            larf_left(m - i, n - i - 1, &A[i + LD * i], 1, tau[i], &A[i + LD * (i + 1)]);
        }
        for (int l = i + 1; l < m; l++) A[l + LD * i] *= -tau[i];
        A[i + LD * i] = R(1) - tau[i];
        for (int l = 0; l < i; l++) A[l + LD * i] = R(0);
    }
}

// RQ factorisation of the m x n matrix A = R Q, Q = H(0) ... H(k-1) (xGERQ2): reflector i in
// row m - k + i left of column n - k + i (where its unit entry is).
template <class R>
XTG_HD void gerq2(int m, int n, R *A, R *tau)
{
    const int k = m < n ? m : n;
    for (int i = k - 1; i >= 0; i--) {
        const int r = m - k + i, c = n - k + i;
        larfg(c + 1, A[r + LD * c], &A[r], LD, tau[i]);
        const R aii = A[r + LD * c];
        A[r + LD * c] = R(1);
        larf_right(r, c + 1, &A[r], LD, tau[i], A);
        A[r + LD * c] = aii;
    }
}

// The last m rows of Q = H(0) ... H(k-1) (n x n) from gerq2's reflectors in rows m - k .. m - 1,
// in place (xORGR2)
template <class R>
XTG_HD void orgr2(int m, int n, int k, R *A, const R *tau)
{
    if (k < m) {
        for (int j = 0; j < n; j++) {
            for (int l = 0; l < m - k; l++) A[l + LD * j] = R(0);
            if (j + 1 > n - m && j + 1 <= n - k) A[(m - n + j) + LD * j] = R(1);
        }
    }
    for (int i = 0; i < k; i++) {
        const int ii = m - k + i, col = n - m + ii;
        A[ii + LD * col] = R(1);
        larf_right(ii, col + 1, &A[ii], LD, tau[i], A);
        for (int l = 0; l < col; l++) A[ii + LD * l] *= -tau[i];
        A[ii + LD * col] = R(1) - tau[i];
        for (int l = col + 1; l < n; l++) A[ii + LD * l] = R(0);
    }
}

// C (m x m) <- C Q^T with Q from gerq2 of the m x m matrix F (xORMR2, side R, trans T)
template <class R>
XTG_HD void ormr2_rt(int m, R *F, const R *tau, R *C)
{
    for (int i = m - 1; i >= 0; i--) {
        const R aii = F[i + LD * i];
        F[i + LD * i] = R(1);
        larf_right(m, i + 1, &F[i], LD, tau[i], C);
        F[i + LD * i] = aii;
    }
}

// C (m x m) <- Q C with Q from gerq2 of F (xORMR2, side L, trans N)
template <class R>
XTG_HD void ormr2_ln(int m, R *F, const R *tau, R *C)
{
    for (int i = m - 1; i >= 0; i--) {
        const R aii = F[i + LD * i];
        F[i + LD * i] = R(1);
        larf_left(i + 1, m, &F[i], LD, tau[i], C);
        F[i + LD * i] = aii;
    }
}

// C (m x m) <- Q^T C with Q from geqr2 of F (xORM2R, side L, trans T)
template <class R>
XTG_HD void orm2r_lt(int m, R *F, const R *tau, R *C)
{
    for (int i = 0; i < m; i++) {
        const R aii = F[i + LD * i];
        F[i + LD * i] = R(1);
        larf_left(m - i, m, &F[i + LD * i], 1, tau[i], &C[i]);
        F[i + LD * i] = aii;
    }
}

// C (m x m) <- C Q with Q from geqr2 of F (xORM2R, side R, trans N)
template <class R>
XTG_HD void orm2r_rn(int m, R *F, const R *tau, R *C)
{
    for (int i = 0; i < m; i++) {
        const R aii = F[i + LD * i];
        F[i + LD * i] = R(1);
        larf_right(m, m - i, &F[i + LD * i], 1, tau[i], &C[LD * i]);
        F[i + LD * i] = aii;
    }
}

// LU factorisation with complete pivoting of the n x n matrix Z (leading dimension 8),
// P Z Q = L U, tiny pivots raised to smin (xGETC2).  Returns 0, or the first (1-based) pivot
// that was raised.
template <class R>
XTG_HD int getc2(int n, R *Z, int *ipiv, int *jpiv)
{
    const R eps = Mach<R>::prec, smlnum = Mach<R>::sfmin / eps;
    int info = 0;
    R smin = R(0);
    for (int i = 0; i < n - 1; i++) {
        R xmx = R(0);
        int ipv = i, jpv = i;
        for (int ip = i; ip < n; ip++)
            for (int jp = i; jp < n; jp++)
                if (xabs(Z[ip + 8 * jp]) >= xmx) {
                    xmx = xabs(Z[ip + 8 * jp]);
                    ipv = ip;
                    jpv = jp;
                }
        if (i == 0) smin = xmax(eps * xmx, smlnum);
        if (ipv != i)
            for (int j = 0; j < n; j++) {
                const R t = Z[ipv + 8 * j];
                Z[ipv + 8 * j] = Z[i + 8 * j];
                Z[i + 8 * j] = t;
            }
        ipiv[i] = ipv;
        if (jpv != i)
            for (int j = 0; j < n; j++) {
                const R t = Z[j + 8 * jpv];
                Z[j + 8 * jpv] = Z[j + 8 * i];
                Z[j + 8 * i] = t;
            }
        jpiv[i] = jpv;
        if (xabs(Z[i + 8 * i]) < smin) {
            info = i + 1;
            Z[i + 8 * i] = smin;
        }
        for (int j = i + 1; j < n; j++) Z[j + 8 * i] /= Z[i + 8 * i];
        for (int jj = i + 1; jj < n; jj++) {
            const R t = -Z[i + 8 * jj];
            for (int ii = i + 1; ii < n; ii++) Z[ii + 8 * jj] += Z[ii + 8 * i] * t;
        }
    }
    if (xabs(Z[(n - 1) + 8 * (n - 1)]) < smin) {
        info = n;
        Z[(n - 1) + 8 * (n - 1)] = smin;
    }
    ipiv[n - 1] = n - 1;
    jpiv[n - 1] = n - 1;
    return info;
}

// Solve Z x = scale rhs with getc2's factors, scale <= 1 chosen against overflow (xGESC2)
template <class R>
XTG_HD void gesc2(int n, const R *Z, R *rhs, const int *ipiv, const int *jpiv, R &scale)
{
    const R eps = Mach<R>::prec, smlnum = Mach<R>::sfmin / eps;
    for (int i = 0; i < n - 1; i++)
        if (ipiv[i] != i) {
            const R t = rhs[i];
            rhs[i] = rhs[ipiv[i]];
            rhs[ipiv[i]] = t;
        }
    for (int i = 0; i < n - 1; i++)
        for (int j = i + 1; j < n; j++) rhs[j] -= Z[j + 8 * i] * rhs[i];
    scale = R(1);
    int imax = 0;
    for (int i = 1; i < n; i++)
        if (xabs(rhs[i]) > xabs(rhs[imax])) imax = i;
    if (R(2) * smlnum * xabs(rhs[imax]) > xabs(Z[(n - 1) + 8 * (n - 1)])) {
        const R t = R(0.5) / xabs(rhs[imax]);
        for (int i = 0; i < n; i++) rhs[i] *= t;
        scale *= t;
    }
    for (int i = n - 1; i >= 0; i--) {
        const R t = R(1) / Z[i + 8 * i];
        rhs[i] *= t;
        for (int j = i + 1; j < n; j++) rhs[i] -= rhs[j] * (Z[i + 8 * j] * t);
    }
    for (int i = n - 2; i >= 0; i--)
        if (jpiv[i] != i) {
            const R t = rhs[i];
            rhs[i] = rhs[jpiv[i]];
            rhs[jpiv[i]] = t;
        }
}

// Generalized Sylvester equation of one pair of diagonal blocks (xTGSY2, TRANS = 'N',
// IJOB = 0, with A and B each a single 1x1 or 2x2 block):
//     A R - L B = scale C,   D R - L E = scale F
// A (n1 x n1), B (n2 x n2), D, E upper triangular; C, F (n1 x n2, leading dimension 2) are
// overwritten by R and L.  The unknowns [vec R; vec L] (column-major) solve the 2 n1 n2
// Kronecker system.  Returns 0, or > 0 when a pivot had to be raised (close eigenvalues).
template <class R>
XTG_HD int tgsy2(int n1, int n2, const R *A, const R *B, const R *D, const R *E, R *C, R *F, R &scale)
{
    const int nn = n1 * n2, zdim = 2 * nn;
    R Z[64], rhs[8];
    for (int i = 0; i < 64; i++) Z[i] = R(0);
    for (int j = 0; j < n2; j++)
        for (int i = 0; i < n1; i++) {
            const int k = i + n1 * j;
            for (int p = 0; p < n1; p++) {
                Z[k + 8 * (p + n1 * j)] = A[i + LD * p];                       // (A R)(i, j)
                if (p >= i) Z[(nn + k) + 8 * (p + n1 * j)] = D[i + LD * p];    // (D R)(i, j)
            }
            for (int q = 0; q < n2; q++) {
                Z[k + 8 * (nn + i + n1 * q)] = -B[q + LD * j];                 // (L B)(i, j)
                if (q <= j) Z[(nn + k) + 8 * (nn + i + n1 * q)] = -E[q + LD * j];  // (L E)(i, j)
            }
            rhs[k] = C[i + 2 * j];
            rhs[nn + k] = F[i + 2 * j];
        }
    int ipiv[8], jpiv[8];
    const int info = getc2(zdim, Z, ipiv, jpiv);
    gesc2(zdim, Z, rhs, ipiv, jpiv, scale);
    for (int j = 0; j < n2; j++)
        for (int i = 0; i < n1; i++) {
            C[i + 2 * j] = rhs[i + n1 * j];
            F[i + 2 * j] = rhs[nn + i + n1 * j];
        }
    return info;
}

// Eigenvalues of the 2x2 pencil A - w B, B upper triangular, with scaling against over- and
// underflow (xLAG2): real pair (wr1, wr2, wi = 0; wr1 the one closer to the (2,2) entry of
// A B^-1) or complex pair wr1 +- i wi; scale1 w1 = the first eigenvalue's numerator scale.
template <class R>
XTG_HD void lag2(const R *A, const R *B, R safmin, R &scale1, R &scale2, R &wr1, R &wr2, R &wi)
{
    const R rtmin = xsqrt(safmin), rtmax = R(1) / rtmin, safmax = R(1) / safmin;
    const R fuzzy1 = R(1) + R(1.0e-5);
    const R anorm = xmax(xmax(xabs(A[0]) + xabs(A[1]), xabs(A[LD]) + xabs(A[1 + LD])), safmin);
    const R ascale = R(1) / anorm;
    const R a11 = ascale * A[0], a21 = ascale * A[1], a12 = ascale * A[LD], a22 = ascale * A[1 + LD];
    R b11 = B[0], b12 = B[LD], b22 = B[1 + LD];
    const R bmin = rtmin * xmax(xmax(xabs(b11), xabs(b12)), xmax(xabs(b22), rtmin));
    if (xabs(b11) < bmin) b11 = xsign(bmin, b11);
    if (xabs(b22) < bmin) b22 = xsign(bmin, b22);
    const R bnorm = xmax(xmax(xabs(b11), xabs(b12) + xabs(b22)), safmin);
    const R bsize = xmax(xabs(b11), xabs(b22));
    const R bscale = R(1) / bsize;
    b11 *= bscale;
    b12 *= bscale;
    b22 *= bscale;
    const R binv11 = R(1) / b11, binv22 = R(1) / b22;
    const R s1 = a11 * binv11, s2 = a22 * binv22;
    R as12, ss, abi22, pp, shift;
    if (xabs(s1) <= xabs(s2)) {
        as12 = a12 - s1 * b12;
        const R as22 = a22 - s1 * b22;
        ss = a21 * (binv11 * binv22);
        abi22 = as22 * binv22 - ss * b12;
        pp = R(0.5) * abi22;
        shift = s1;
    } else {
        as12 = a12 - s2 * b12;
        const R as11 = a11 - s2 * b11;
        ss = a21 * (binv11 * binv22);
        abi22 = -ss * b12;
        pp = R(0.5) * (as11 * binv11 + abi22);
        shift = s2;
    }
    const R qq = ss * as12;
    R discr, r;
    if (xabs(pp * rtmin) >= R(1)) {
        discr = (rtmin * pp) * (rtmin * pp) + qq * safmin;
        r = xsqrt(xabs(discr)) * rtmax;
    } else if (pp * pp + xabs(qq) <= safmin) {
        discr = (rtmax * pp) * (rtmax * pp) + qq * safmax;
        r = xsqrt(xabs(discr)) * rtmin;
    } else {
        discr = pp * pp + qq;
        r = xsqrt(xabs(discr));
    }
    if (discr >= R(0) || r == R(0)) {
        const R sum = pp + xsign(r, pp), diff = pp - xsign(r, pp);
        const R wbig = shift + sum;
        R wsmall = shift + diff;
        if (R(0.5) * xabs(wbig) > xmax(xabs(wsmall), safmin)) {
            const R wdet = (a11 * a22 - a12 * a21) * (binv11 * binv22);
            wsmall = wdet / wbig;
        }
        if (pp > abi22) {
            wr1 = xmin(wbig, wsmall);
            wr2 = xmax(wbig, wsmall);
        } else {
            wr1 = xmax(wbig, wsmall);
            wr2 = xmin(wbig, wsmall);
        }
        wi = R(0);
    } else {
        wr1 = shift + pp;
        wr2 = wr1;
        wi = r;
    }
    const R c1 = bsize * (safmin * xmax(R(1), ascale));
    const R c2 = safmin * xmax(R(1), bnorm);
    const R c3 = bsize * safmin;
    const R c4 = (ascale <= R(1) && bsize <= R(1)) ? xmin(R(1), (ascale / safmin) * bsize) : R(1);
    const R c5 = (ascale <= R(1) || bsize <= R(1)) ? xmin(R(1), ascale * bsize) : R(1);
    const R wabs = xabs(wr1) + xabs(wi);
    R wsize = xmax(xmax(safmin, c1), xmax(fuzzy1 * (wabs * c2 + c3), xmin(c4, R(0.5) * xmax(wabs, c5))));
    if (wsize != R(1)) {
        const R wscale = R(1) / wsize;
        if (wsize > R(1)) scale1 = (xmax(ascale, bsize) * wscale) * xmin(ascale, bsize);
        else scale1 = (xmin(ascale, bsize) * wscale) * xmax(ascale, bsize);
        wr1 *= wscale;
        if (wi != R(0)) {
            wi *= wscale;
            wr2 = wr1;
            scale2 = scale1;
        }
    } else {
        scale1 = ascale * bsize;
        scale2 = scale1;
    }
    if (wi == R(0)) {
        wsize = xmax(xmax(safmin, c1), xmax(fuzzy1 * (xabs(wr2) * c2 + c3), xmin(c4, R(0.5) * xmax(xabs(wr2), c5))));
        if (wsize != R(1)) {
            const R wscale = R(1) / wsize;
            if (wsize > R(1)) scale2 = (xmax(ascale, bsize) * wscale) * xmin(ascale, bsize);
            else scale2 = (xmin(ascale, bsize) * wscale) * xmax(ascale, bsize);
            wr2 *= wscale;
        } else {
            scale2 = ascale * bsize;
        }
    }
}

// SVD of the 2x2 upper triangular [f g; 0 h] (xLASV2):
// [csl snl; -snl csl] [f g; 0 h] [csr -snr; snr csr] = [ssmax 0; 0 ssmin]
template <class R>
XTG_HD void lasv2(R f, R g, R h, R &ssmin, R &ssmax, R &snr, R &csr, R &snl, R &csl)
{
    R ft = f, fa = xabs(ft), ht = h, ha = xabs(h);
    int pmax = 1;
    const bool swap = ha > fa;
    if (swap) {
        pmax = 3;
        R t = ft;
        ft = ht;
        ht = t;
        t = fa;
        fa = ha;
        ha = t;
    }
    const R gt = g, ga = xabs(gt);
    R clt, crt, slt, srt;
    if (ga == R(0)) {
        ssmin = ha;
        ssmax = fa;
        clt = R(1);
        crt = R(1);
        slt = R(0);
        srt = R(0);
    } else {
        bool gasmal = true;
        if (ga > fa) {
            pmax = 2;
            if (fa / ga < Mach<R>::epsr) {
                gasmal = false;
                ssmax = ga;
                if (ha > R(1)) ssmin = fa / (ga / ha);
                else ssmin = (fa / ga) * ha;
                clt = R(1);
                slt = ht / gt;
                srt = R(1);
                crt = ft / gt;
            }
        }
        if (gasmal) {
            const R d = fa - ha;
            R l = (d == fa) ? R(1) : d / fa;
            const R mq = gt / ft;
            R t = R(2) - l;
            const R mm = mq * mq, tt = t * t;
            const R s = xsqrt(tt + mm);
            const R r = (l == R(0)) ? xabs(mq) : xsqrt(l * l + mm);
            const R a = R(0.5) * (s + r);
            ssmin = ha / a;
            ssmax = fa * a;
            if (mm == R(0)) {
                if (l == R(0)) t = xsign(R(2), ft) * xsign(R(1), gt);
                else t = gt / xsign(d, ft) + mq / t;
            } else {
                t = (mq / (s + t) + mq / (r + l)) * (R(1) + a);
            }
            l = xsqrt(t * t + R(4));
            crt = R(2) / l;
            srt = t / l;
            clt = (crt + srt * mq) / a;
            slt = (ht / ft) * srt / a;
        }
    }
    if (swap) {
        csl = srt;
        snl = crt;
        csr = slt;
        snr = clt;
    } else {
        csl = clt;
        snl = slt;
        csr = crt;
        snr = srt;
    }
    R tsign = R(1);
    if (pmax == 1) tsign = xsign(R(1), csr) * xsign(R(1), csl) * xsign(R(1), f);
    if (pmax == 2) tsign = xsign(R(1), snr) * xsign(R(1), csl) * xsign(R(1), g);
    if (pmax == 3) tsign = xsign(R(1), snr) * xsign(R(1), snl) * xsign(R(1), h);
    ssmax = xsign(ssmax, tsign);
    ssmin = xsign(ssmin, tsign * xsign(R(1), f) * xsign(R(1), h));
}

// Generalized Schur form of the 2x2 pencil (A, B), B upper triangular, in place (xLAGV2):
// rows take [csl snl; -snl csl], columns [csr -snr; snr csr].  Real eigenvalues: both become
// upper triangular; a complex pair: B becomes diagonal (positive), A stays full.
template <class R>
XTG_HD void lagv2(R *A, R *B, R &csl, R &snl, R &csr, R &snr)
{
    const R safmin = Mach<R>::sfmin, ulp = Mach<R>::prec;
    const R anorm = xmax(xmax(xabs(A[0]) + xabs(A[1]), xabs(A[LD]) + xabs(A[1 + LD])), safmin);
    const R ascale = R(1) / anorm;
    A[0] *= ascale;
    A[LD] *= ascale;
    A[1] *= ascale;
    A[1 + LD] *= ascale;
    const R bnorm = xmax(xmax(xabs(B[0]), xabs(B[LD]) + xabs(B[1 + LD])), safmin);
    const R bscale = R(1) / bnorm;
    B[0] *= bscale;
    B[LD] *= bscale;
    B[1 + LD] *= bscale;
    R r;
    auto rows = [&](R c, R s) {
        rot(A[0], A[1], c, s);
        rot(A[LD], A[1 + LD], c, s);
        rot(B[0], B[1], c, s);
        rot(B[LD], B[1 + LD], c, s);
    };
    auto cols = [&](R c, R s) {
        rot(A[0], A[LD], c, s);
        rot(A[1], A[1 + LD], c, s);
        rot(B[0], B[LD], c, s);
        rot(B[1], B[1 + LD], c, s);
    };
    if (xabs(A[1]) <= ulp) {
        csl = R(1);
        snl = R(0);
        csr = R(1);
        snr = R(0);
        A[1] = R(0);
        B[1] = R(0);
    } else if (xabs(B[0]) <= ulp) {
        lartg(A[0], A[1], csl, snl, r);
        csr = R(1);
        snr = R(0);
        rows(csl, snl);
        A[1] = R(0);
        B[0] = R(0);
        B[1] = R(0);
    } else if (xabs(B[1 + LD]) <= ulp) {
        lartg(A[1 + LD], A[1], csr, snr, r);
        snr = -snr;
        cols(csr, snr);
        csl = R(1);
        snl = R(0);
        A[1] = R(0);
        B[1] = R(0);
        B[1 + LD] = R(0);
    } else {
        R scale1, scale2, wr1, wr2, wi;
        lag2(A, B, safmin, scale1, scale2, wr1, wr2, wi);
        if (wi == R(0)) {
            R h1 = scale1 * A[0] - wr1 * B[0];
            R h2 = scale1 * A[LD] - wr1 * B[LD];
            const R h3 = scale1 * A[1 + LD] - wr1 * B[1 + LD];
            const R rr = lapy2(h1, h2), qq = lapy2(scale1 * A[1], h3);
            if (rr > qq) lartg(h2, h1, csr, snr, r);
            else lartg(h3, scale1 * A[1], csr, snr, r);
            snr = -snr;
            cols(csr, snr);
            h1 = xmax(xabs(A[0]) + xabs(A[LD]), xabs(A[1]) + xabs(A[1 + LD]));
            h2 = xmax(xabs(B[0]) + xabs(B[LD]), xabs(B[1]) + xabs(B[1 + LD]));
            if (scale1 * h1 >= xabs(wr1) * h2) lartg(B[0], B[1], csl, snl, r);
            else lartg(A[0], A[1], csl, snl, r);
            rows(csl, snl);
            A[1] = R(0);
            B[1] = R(0);
        } else {
            R t;
            lasv2(B[0], B[LD], B[1 + LD], r, t, snr, csr, snl, csl);
            rows(csl, snl);
            cols(csr, snr);
            B[1] = R(0);
            B[LD] = R(0);
        }
    }
    A[0] *= anorm;
    A[1] *= anorm;
    A[LD] *= anorm;
    A[1 + LD] *= anorm;
    B[0] *= bnorm;
    B[1] *= bnorm;
    B[LD] *= bnorm;
    B[1 + LD] *= bnorm;
}

// The swap of two 1x1 blocks at the 2x2 blocks (a, b) of A and B: the column rotation
// (cz, sz) and the row rotation (cq, sq), both applied as (x, y) <- (c x + s y, c y - s x),
// and whether the swap passes the weak and the strong test (the real xTGEX2's 1x1 case:
// F = a11 b00 - b11 a00, G = a11 b01 - b11 a01 rounded term by term, [cs sn; -sn cs] [F; G]
// = [r; 0], columns (sn, -cs), rows the rotation that zeroes the new (1, 0) entry of A or B).
template <class R>
XTG_HD bool swap11(R a00, R a10, R a01, R a11, R b00, R b10, R b01, R b11, R &cz, R &sz, R &cq, R &sq)
{
    const R eps = Mach<R>::prec, smlnum = Mach<R>::sfmin / eps;
    const R tha = xmax(R(20) * eps * xhypot(xhypot(a00, a10), xhypot(a01, a11)), smlnum);
    const R thb = xmax(R(20) * eps * xhypot(xhypot(b00, b10), xhypot(b01, b11)), smlnum);
    const R f = sub_rn(mul_rn(a11, b00), mul_rn(b11, a00));
    const R g = sub_rn(mul_rn(a11, b01), mul_rn(b11, a01));
    const R sa = xabs(a11) * xabs(b00), sb = xabs(a00) * xabs(b11);
    R cs, sn, r;
    lartg(f, g, cs, sn, r);
    cz = sn;
    sz = -cs;
    R s00 = a00, s01 = a01, s10 = a10, s11 = a11, t00 = b00, t01 = b01, t10 = b10, t11 = b11;
    rot(s00, s01, cz, sz);
    rot(s10, s11, cz, sz);
    rot(t00, t01, cz, sz);
    rot(t10, t11, cz, sz);
    if (sa >= sb) lartg(s00, s10, cq, sq, r);
    else lartg(t00, t10, cq, sq, r);
    rot(s00, s10, cq, sq);
    rot(s01, s11, cq, sq);
    rot(t00, t10, cq, sq);
    rot(t01, t11, cq, sq);
    bool ok = xabs(s10) <= tha && xabs(t10) <= thb && xfinite(cz) && xfinite(sz) && xfinite(cq) && xfinite(sq) &&
              xfinite(s00) && xfinite(s01) && xfinite(s11) && xfinite(t00) && xfinite(t01) && xfinite(t11);
    if (ok) {  // undo both rotations on the swapped blocks: the originals must come back
        R w00 = s00, w01 = s01, w10 = s10, w11 = s11, v00 = t00, v01 = t01, v10 = t10, v11 = t11;
        rot(w00, w10, cq, -sq);
        rot(w01, w11, cq, -sq);
        rot(v00, v10, cq, -sq);
        rot(v01, v11, cq, -sq);
        rot(w00, w01, cz, -sz);
        rot(w10, w11, cz, -sz);
        rot(v00, v01, cz, -sz);
        rot(v10, v11, cz, -sz);
        ok = xhypot(xhypot(w00 - a00, w10 - a10), xhypot(w01 - a01, w11 - a11)) <= tha &&
             xhypot(xhypot(v00 - b00, v10 - b10), xhypot(v01 - b01, v11 - b11)) <= thb;
    }
    return ok;
}

// C = op(X) op(Y) for m x m matrices (leading dimension LD); ta / tb transpose X / Y
template <class R>
XTG_HD void mm(int m, const R *X, bool ta, const R *Y, bool tb, R *C)
{
    for (int j = 0; j < m; j++)
        for (int i = 0; i < m; i++) {
            R s = R(0);
            for (int k = 0; k < m; k++) s += (ta ? X[k + LD * i] : X[i + LD * k]) * (tb ? Y[j + LD * k] : Y[k + LD * j]);
            C[i + LD * j] = s;
        }
}

// One swap of an n1 block and an n2 block, m = n1 + n2 in {3, 4} (the real xTGEX2's general
// case).  In: the m x m diagonal blocks S, T of A and B (leading dimension LD).  Out, when the
// swap passes both tests: S, T the new blocks (standardised), LI and IR (m x m) with
//     rows of the block row     <- LI^T rows,    Q's m columns <- Q LI,
//     columns of the block col  <- columns IR,   Z's m columns <- Z IR.
// Returns false (nothing to apply) when the swap is rejected.
template <class R>
XTG_HD bool swap_blocks(int n1, int n2, R *S, R *T, R *LI, R *IR)
{
    const int m = n1 + n2;
    const R eps = Mach<R>::prec, smlnum = Mach<R>::sfmin / eps;
    R A0[16], B0[16];
    for (int i = 0; i < 16; i++) {
        A0[i] = S[i];
        B0[i] = T[i];
    }
    const R thresha = xmax(R(20) * eps * fro_block(S, m, m), smlnum);
    const R threshb = xmax(R(20) * eps * fro_block(T, m, m), smlnum);
    // 1. S11 R - L S22 = scale S12, T11 R - L T22 = scale T12
    R Rm[4], Lm[4], scale;
    for (int j = 0; j < n2; j++)
        for (int i = 0; i < n1; i++) {
            Rm[i + 2 * j] = S[i + LD * (n1 + j)];
            Lm[i + 2 * j] = T[i + LD * (n1 + j)];
        }
    if (tgsy2(n1, n2, S, &S[n1 + LD * n1], T, &T[n1 + LD * n1], Rm, Lm, scale) != 0) return false;
    // 2. QL from the QR factorisation of [-L; scale I] (m x n2), QR from the RQ factorisation
    //    of [scale I, R] (n1 x m, rows n2 .. m - 1 of IR)
    R taul[4], taur[4];
    for (int i = 0; i < 16; i++) {
        LI[i] = R(0);
        IR[i] = R(0);
    }
    for (int j = 0; j < n2; j++) {
        for (int i = 0; i < n1; i++) LI[i + LD * j] = -Lm[i + 2 * j];
        LI[n1 + j + LD * j] = scale;
    }
    geqr2(m, n2, LI, taul);
    org2r(m, m, n2, LI, taul);
    for (int i = 0; i < n1; i++) {
        IR[n2 + i + LD * i] = scale;
        for (int j = 0; j < n2; j++) IR[n2 + i + LD * (n1 + j)] = Rm[i + 2 * j];
    }
    gerq2(n1, m, &IR[n2], taur);
    orgr2(m, m, n1, IR, taur);
    // the tentative swap: S <- LI^T S IR^T, T <- LI^T T IR^T
    R W[16], Scp[16], Tcp[16], IRcp[16], LIcp[16];
    mm(m, LI, true, S, false, W);
    mm(m, W, false, IR, true, S);
    mm(m, LI, true, T, false, W);
    mm(m, W, false, IR, true, T);
    for (int i = 0; i < 16; i++) {
        Scp[i] = S[i];
        Tcp[i] = T[i];
        IRcp[i] = IR[i];
        LIcp[i] = LI[i];
    }
    // 3. re-triangularise T: by RQ (S <- S Q^T, IR <- Q IR) and by QR (Scp <- Q^T Scp,
    //    LIcp <- LIcp Q); keep the smaller S21, then the weak and the strong test
    gerq2(m, m, T, taur);
    ormr2_rt(m, T, taur, S);
    ormr2_ln(m, T, taur, IR);
    const R brqa21 = fro_block(&S[n2], n1, n2);
    geqr2(m, m, Tcp, taul);
    orm2r_lt(m, Tcp, taul, Scp);
    orm2r_rn(m, Tcp, taul, LIcp);
    const R bqra21 = fro_block(&Scp[n2], n1, n2);
    if (bqra21 <= brqa21 && bqra21 <= thresha) {
        for (int i = 0; i < 16; i++) {
            S[i] = Scp[i];
            T[i] = Tcp[i];
            IR[i] = IRcp[i];
            LI[i] = LIcp[i];
        }
    } else if (!(brqa21 < thresha)) {
        return false;
    }
    for (int j = 0; j < m; j++)
        for (int i = j + 1; i < m; i++) T[i + LD * j] = R(0);
    {  // strong test: || A0 - LI S IR ||_F, || B0 - LI T IR ||_F
        R X[16];
        mm(m, LI, false, S, false, W);
        mm(m, W, false, IR, false, X);
        for (int j = 0; j < m; j++)
            for (int i = 0; i < m; i++) X[i + LD * j] = A0[i + LD * j] - X[i + LD * j];
        const R sa = fro_block(X, m, m);
        mm(m, LI, false, T, false, W);
        mm(m, W, false, IR, false, X);
        for (int j = 0; j < m; j++)
            for (int i = 0; i < m; i++) X[i + LD * j] = B0[i + LD * j] - X[i + LD * j];
        const R sb = fro_block(X, m, m);
        if (!(sa <= thresha && sb <= threshb)) return false;
    }
    for (int j = 0; j < n2; j++)
        for (int i = n2; i < m; i++) S[i + LD * j] = R(0);
    // 4. standardise the new diagonal blocks: left WQ, right WZ (block diagonal rotations)
    R WQ[16], WZ[16];
    for (int i = 0; i < 16; i++) {
        WQ[i] = R(0);
        WZ[i] = R(0);
    }
    WQ[0] = R(1);
    WZ[0] = R(1);
    R csl, snl, csr, snr;
    if (n2 > 1) {
        lagv2(S, T, csl, snl, csr, snr);
        WQ[0] = csl;
        WQ[1] = snl;
        WQ[LD] = -snl;
        WQ[1 + LD] = csl;
        WZ[0] = csr;
        WZ[1] = snr;
        WZ[LD] = -snr;
        WZ[1 + LD] = csr;
    }
    WQ[(m - 1) + LD * (m - 1)] = R(1);
    WZ[(m - 1) + LD * (m - 1)] = R(1);
    if (n1 > 1) {
        lagv2(&S[n2 + LD * n2], &T[n2 + LD * n2], csl, snl, csr, snr);
        WQ[n2 + LD * n2] = csl;
        WQ[n2 + 1 + LD * n2] = snl;
        WQ[(m - 2) + LD * (m - 1)] = -snl;
        WQ[(m - 1) + LD * (m - 1)] = csl;
        WZ[n2 + LD * n2] = csr;
        WZ[(m - 1) + LD * (m - 2)] = snr;
        WZ[(m - 2) + LD * (m - 1)] = -snr;
        WZ[(m - 1) + LD * (m - 1)] = csr;
    }
    // off-diagonal blocks: S12 <- WQ11^T S12 WZ22, T12 likewise
    for (int w = 0; w < 2; w++) {
        R *M = w == 0 ? S : T;
        R X[4], Y[4];
        for (int j = 0; j < n1; j++)
            for (int i = 0; i < n2; i++) {
                R s = R(0);
                for (int k = 0; k < n2; k++) s += WQ[k + LD * i] * M[k + LD * (n2 + j)];
                X[i + 2 * j] = s;
            }
        for (int j = 0; j < n1; j++)
            for (int i = 0; i < n2; i++) {
                R s = R(0);
                for (int k = 0; k < n1; k++) s += X[i + 2 * k] * WZ[(n2 + k) + LD * (n2 + j)];
                Y[i + 2 * j] = s;
            }
        for (int j = 0; j < n1; j++)
            for (int i = 0; i < n2; i++) M[i + LD * (n2 + j)] = Y[i + 2 * j];
    }
    // LI <- LI WQ, IR <- IR^T WZ
    mm(m, LI, false, WQ, false, W);
    for (int i = 0; i < 16; i++) LI[i] = W[i];
    mm(m, IR, true, WZ, false, W);
    for (int i = 0; i < 16; i++) IR[i] = W[i];
    return true;
}

// The matrices of one reordering (column-major; Q, Z referenced only when wanted)
template <class R>
struct Pencil {
    int n, wantq, wantz;
    R *A, *B, *Q, *Z;
    int lda, ldb, ldq, ldz;
};

// A(i, j) != 0, 1-based; outside the matrix reads as zero
template <class R>
XTG_HD inline bool nz(const Pencil<R> &p, int i, int j)
{
    return i >= 1 && j >= 1 && i <= p.n && j <= p.n && p.A[(size_t)(i - 1) + (size_t)(j - 1) * p.lda] != R(0);
}

// The walk of xTGEXC: the block at row `here` (1-based) of size nbf (3: a 2x2 block that split
// into two 1x1 blocks, moved one after the other) travels to ilst by swaps with its neighbour
// block; the phases order the swaps of a split block.
struct Walk {
    int here, ilst, nbf, nbnext, phase, fwd;
    int next_here, next_phase, check_split;  // applied when the pending swap is done
};

// xTGEXC's start: IFST and ILST move to the first row of their blocks, ILST is adjusted for
// the block sizes of a downward move.  Returns false when nothing moves.
template <class R>
XTG_HD bool walk_begin(const Pencil<R> &p, Walk &w, int &ifst, int &ilst)
{
    if (ifst > 1 && nz(p, ifst, ifst - 1)) ifst--;
    const int nbf = (ifst < p.n && nz(p, ifst + 1, ifst)) ? 2 : 1;
    if (ilst > 1 && nz(p, ilst, ilst - 1)) ilst--;
    const int nbl = (ilst < p.n && nz(p, ilst + 1, ilst)) ? 2 : 1;
    if (ifst == ilst) return false;
    if (ifst < ilst) {
        if (nbf == 2 && nbl == 1) ilst--;
        if (nbf == 1 && nbl == 2) ilst++;
    }
    w.here = ifst;
    w.ilst = ilst;
    w.nbf = nbf;
    w.nbnext = 1;
    w.phase = 0;
    w.fwd = ifst < ilst ? 1 : 0;
    w.next_here = ifst;
    w.next_phase = 0;
    w.check_split = 0;
    return true;
}

// The next swap (first row j1, 1-based, block sizes n1 above n2), or false when the block has
// arrived (here is then the new ILST).
template <class R>
XTG_HD bool walk_next(const Pencil<R> &p, Walk &w, int &j1, int &n1, int &n2)
{
    const int h = w.here;
    w.check_split = 0;
    if (w.fwd) {
        if (w.phase == 0) {
            if (h >= w.ilst) return false;
            if (w.nbf != 3) {
                w.nbnext = (h + w.nbf + 1 <= p.n && nz(p, h + w.nbf + 1, h + w.nbf)) ? 2 : 1;
                j1 = h, n1 = w.nbf, n2 = w.nbnext;
                w.next_here = h + w.nbnext, w.next_phase = 0, w.check_split = w.nbf == 2;
            } else {
                w.nbnext = (h + 3 <= p.n && nz(p, h + 3, h + 2)) ? 2 : 1;
                j1 = h + 1, n1 = 1, n2 = w.nbnext;
                w.next_here = h, w.next_phase = 1;
            }
        } else if (w.phase == 1) {
            if (w.nbnext == 1) {
                j1 = h, n1 = 1, n2 = 1;
                w.next_here = h + 1, w.next_phase = 0;
            } else {
                if (!nz(p, h + 2, h + 1)) w.nbnext = 1;  // the 2x2 block split
                if (w.nbnext == 2) {
                    j1 = h, n1 = 1, n2 = 2;
                    w.next_here = h + 2, w.next_phase = 0;
                } else {
                    j1 = h, n1 = 1, n2 = 1;
                    w.next_here = h + 1, w.next_phase = 2;
                }
            }
        } else {
            j1 = h, n1 = 1, n2 = 1;
            w.next_here = h + 1, w.next_phase = 0;
        }
    } else {
        if (w.phase == 0) {
            if (h <= w.ilst) return false;
            w.nbnext = (h >= 3 && nz(p, h - 1, h - 2)) ? 2 : 1;
            if (w.nbf != 3) {
                j1 = h - w.nbnext, n1 = w.nbnext, n2 = w.nbf;
                w.next_here = h - w.nbnext, w.next_phase = 0, w.check_split = w.nbf == 2;
            } else {
                j1 = h - w.nbnext, n1 = w.nbnext, n2 = 1;
                w.next_here = h, w.next_phase = 1;
            }
        } else if (w.phase == 1) {
            if (w.nbnext == 1) {
                j1 = h, n1 = 1, n2 = 1;
                w.next_here = h - 1, w.next_phase = 0;
            } else {
                if (!nz(p, h, h - 1)) w.nbnext = 1;  // the 2x2 block split
                if (w.nbnext == 2) {
                    j1 = h - 1, n1 = 2, n2 = 1;
                    w.next_here = h - 2, w.next_phase = 0;
                } else {
                    j1 = h, n1 = 1, n2 = 1;
                    w.next_here = h - 1, w.next_phase = 2;
                }
            }
        } else {
            j1 = h, n1 = 1, n2 = 1;
            w.next_here = h - 1, w.next_phase = 0;
        }
    }
    return true;
}

// After the pending swap was done: advance, and note a moving 2x2 block that split
template <class R>
XTG_HD void walk_after(const Pencil<R> &p, Walk &w)
{
    w.here = w.next_here;
    w.phase = w.next_phase;
    if (w.check_split && !nz(p, w.here + 1, w.here)) w.nbf = 3;
}

// One swap: where (j1 0-based, sizes n1 above n2), whether it is done (ok: 1 applied, 0
// rejected, 2 nothing to do: the blocks reach past row n, as xTGEX2's quick return), and
// its transformations (m = 2: the two rotations; m > 2: the new blocks and LI, IR).
template <class R>
struct Swap {
    int j1, n1, n2, ok;
    R cz, sz, cq, sq;
    R S[16], T[16], LI[16], IR[16];
};

// The small-block arithmetic of a swap (one thread)
template <class R>
XTG_HD void swap_prepare(const Pencil<R> &p, Swap<R> &s)
{
    const int j = s.j1, m = s.n1 + s.n2;
    if (j < 0 || j + s.n1 >= p.n || j + m > p.n) {
        s.ok = 2;
        return;
    }
    auto a = [&](int i, int k) { return p.A[(size_t)(j + i) + (size_t)(j + k) * p.lda]; };
    auto b = [&](int i, int k) { return p.B[(size_t)(j + i) + (size_t)(j + k) * p.ldb]; };
    if (m == 2) {
        s.ok = swap11(a(0, 0), a(1, 0), a(0, 1), a(1, 1), b(0, 0), b(1, 0), b(0, 1), b(1, 1), s.cz, s.sz, s.cq, s.sq)
                   ? 1
                   : 0;
        return;
    }
    for (int k = 0; k < 16; k++) {
        s.S[k] = R(0);
        s.T[k] = R(0);
    }
    for (int k = 0; k < m; k++)
        for (int i = 0; i < m; i++) {
            s.S[i + LD * k] = a(i, k);
            s.T[i + LD * k] = b(i, k);
        }
    s.ok = swap_blocks(s.n1, s.n2, s.S, s.T, s.LI, s.IR) ? 1 : 0;
}

// Applying a done swap, by thread tid of nth (the CTA on the GPU; one thread on the host).
// m = 2, as xTGEX2's 1x1 case: phase 0 rotates columns j, j+1 (rows [0, j + 2) of A and B,
// all rows of Z), phase 1 (after a barrier) rows j, j+1 (columns [j, n) of A and B) and Q's
// columns j, j+1, phase 2 (after a barrier, one thread) zeroes A(j+1, j) and B(j+1, j).
// m > 2: phase 0 does all of it (the rows above the block take IR, the columns right of it
// LI^T, the block is replaced by S, T, Q takes LI and Z takes IR: disjoint parts).
template <class R>
XTG_HD void swap_apply(const Pencil<R> &p, const Swap<R> &s, int phase, int tid, int nth)
{
    const int j = s.j1, m = s.n1 + s.n2, n = p.n;
    auto A = [&](int i, int k) -> R & { return p.A[(size_t)i + (size_t)k * p.lda]; };
    auto B = [&](int i, int k) -> R & { return p.B[(size_t)i + (size_t)k * p.ldb]; };
    auto Q = [&](int i, int k) -> R & { return p.Q[(size_t)i + (size_t)k * p.ldq]; };
    auto Z = [&](int i, int k) -> R & { return p.Z[(size_t)i + (size_t)k * p.ldz]; };
    if (m == 2) {
        if (phase == 0) {
            const int r = j + 2;
            for (int i = tid; i < 2 * r; i += nth) {
                R &x = i < r ? A(i, j) : B(i - r, j);
                R &y = i < r ? A(i, j + 1) : B(i - r, j + 1);
                rot(x, y, s.cz, s.sz);
            }
            if (p.wantz)
                for (int i = tid; i < n; i += nth) rot(Z(i, j), Z(i, j + 1), s.cz, s.sz);
        } else if (phase == 1) {
            const int c = n - j;
            for (int i = tid; i < 2 * c; i += nth) {
                R &x = i < c ? A(j, j + i) : B(j, j + i - c);
                R &y = i < c ? A(j + 1, j + i) : B(j + 1, j + i - c);
                rot(x, y, s.cq, s.sq);
            }
            if (p.wantq)
                for (int i = tid; i < n; i += nth) rot(Q(i, j), Q(i, j + 1), s.cq, s.sq);
        } else if (tid == 0) {
            A(j + 1, j) = R(0);
            B(j + 1, j) = R(0);
        }
        return;
    }
    if (phase != 0) return;
    // rows [0, j) of columns j .. j+m-1 (A then B) <- rows IR
    for (int i = tid; i < 2 * j; i += nth) {
        const bool ia = i < j;
        const int r = ia ? i : i - j;
        R x[4];
        for (int k = 0; k < m; k++) x[k] = ia ? A(r, j + k) : B(r, j + k);
        for (int c = 0; c < m; c++) {
            R v = R(0);
            for (int k = 0; k < m; k++) v += x[k] * s.IR[k + LD * c];
            (ia ? A(r, j + c) : B(r, j + c)) = v;
        }
    }
    // columns [j + m, n) of rows j .. j+m-1 (A then B) <- LI^T columns
    const int nc = n - j - m;
    for (int i = tid; i < 2 * nc; i += nth) {
        const bool ia = i < nc;
        const int c = j + m + (ia ? i : i - nc);
        R x[4];
        for (int k = 0; k < m; k++) x[k] = ia ? A(j + k, c) : B(j + k, c);
        for (int r = 0; r < m; r++) {
            R v = R(0);
            for (int k = 0; k < m; k++) v += s.LI[k + LD * r] * x[k];
            (ia ? A(j + r, c) : B(j + r, c)) = v;
        }
    }
    // the block itself
    for (int e = tid; e < 2 * m * m; e += nth) {
        const int f = e % (m * m), i = f % m, k = f / m;
        if (e < m * m) A(j + i, j + k) = s.S[i + LD * k];
        else B(j + i, j + k) = s.T[i + LD * k];
    }
    // Q's and Z's columns j .. j+m-1
    if (p.wantq || p.wantz)
        for (int i = tid; i < 2 * n; i += nth) {
            const bool iq = i < n;
            if (iq ? !p.wantq : !p.wantz) continue;
            const int r = iq ? i : i - n;
            const R *Mx = iq ? s.LI : s.IR;
            R x[4];
            for (int k = 0; k < m; k++) x[k] = iq ? Q(r, j + k) : Z(r, j + k);
            for (int c = 0; c < m; c++) {
                R v = R(0);
                for (int k = 0; k < m; k++) v += x[k] * Mx[k + LD * c];
                (iq ? Q(r, j + c) : Z(r, j + c)) = v;
            }
        }
}

// ---- the reordering on one CTA ----------------------------------------------------------------
// Written against a CTA context c (c.tid(), c.nth(): this thread and the CTA's size; c.cta(),
// c.ncta(): this CTA and the grid's size; c.sync(): the CTA barrier): the kernels pass
// CtaDev (threadIdx, __syncthreads), the tests host threads with a barrier.
struct CtaDev {
    XTG_HD int tid() const
    {
#ifdef __CUDA_ARCH__
        return (int)threadIdx.x;
#else
        return 0;
#endif
    }
    XTG_HD int nth() const
    {
#ifdef __CUDA_ARCH__
        return (int)blockDim.x;
#else
        return 1;
#endif
    }
    XTG_HD int cta() const
    {
#ifdef __CUDA_ARCH__
        return (int)blockIdx.x;
#else
        return 0;
#endif
    }
    XTG_HD int ncta() const
    {
#ifdef __CUDA_ARCH__
        return (int)gridDim.x;
#else
        return 1;
#endif
    }
    XTG_HD void sync() const
    {
#ifdef __CUDA_ARCH__
        __syncthreads();
#endif
    }
};

// the CTA's shared state of a walk (shared memory on the GPU)
template <class R>
struct WalkShared {
    Swap<R> s;
    Walk w;
    int go, info, ifst, ilst;
};

// The walk of the block at row ifst to row ilst (1-based) on one CTA: thread 0 decides and
// computes each swap, the CTA applies it.  The walk moves the block at least one row every two
// swaps, so it ends within 4 n + 16 swaps; the loop is bounded by that count all the same.  On
// return (every thread, after a barrier): sh.info = 0, 1 (a swap was rejected) or 3 (the
// bound was reached); sh.ifst, sh.ilst as xTGEXC leaves them.
template <class R, class Cta>
XTG_HD void walk_cta(const Cta &c, WalkShared<R> &sh, const Pencil<R> &p, int ifst, int ilst)
{
    const int tid = c.tid(), nth = c.nth();
    if (tid == 0) {
        int f = ifst, l = ilst;
        sh.go = (p.n > 1 && walk_begin(p, sh.w, f, l)) ? 1 : 0;
        sh.ifst = f;
        sh.ilst = l;
        sh.info = 0;
        sh.s.ok = 0;
        sh.s.n1 = sh.s.n2 = 1;
    }
    const int limit = 4 * p.n + 16;
    for (int step = 0;; step++) {
        if (tid == 0 && sh.go) {
            int j1, n1, n2;
            if (step >= limit) {
                sh.go = 0;
                sh.info = 3;
            } else if (!walk_next(p, sh.w, j1, n1, n2)) {
                sh.go = 0;
                sh.ilst = sh.w.here;
            } else {
                sh.s.j1 = j1 - 1;
                sh.s.n1 = n1;
                sh.s.n2 = n2;
                swap_prepare(p, sh.s);
                if (sh.s.ok == 0) {
                    sh.go = 0;
                    sh.ilst = sh.w.here;
                    sh.info = 1;
                }
            }
        }
        c.sync();  // (1): thread 0 writes go / s again only after barrier (2)
        const int go = sh.go, ok = sh.s.ok, m = sh.s.n1 + sh.s.n2;
        if (!go) break;
        if (ok == 1) {
            swap_apply(p, sh.s, 0, tid, nth);
            if (m == 2) {
                c.sync();  // the 2x2 block takes the column rotation before the row rotation
                swap_apply(p, sh.s, 1, tid, nth);
                c.sync();
                swap_apply(p, sh.s, 2, tid, nth);
            }
        }
        c.sync();  // (2): the swap is in memory before thread 0 reads A again
        if (tid == 0) walk_after(p, sh.w);
    }
    c.sync();  // every thread has left the loop before the state is read or reused
}

// The whole reordering on one thread (the tests' CPU build of this header): returns INFO
// (0, or 1 when a swap was rejected), with ifst and ilst as xTGEXC leaves them.
template <class R>
int tgexc_serial(const Pencil<R> &p, int &ifst, int &ilst)
{
    Walk w;
    if (p.n <= 1 || !walk_begin(p, w, ifst, ilst)) return 0;
    Swap<R> s;
    int j1, n1, n2;
    while (walk_next(p, w, j1, n1, n2)) {
        s.j1 = j1 - 1;
        s.n1 = n1;
        s.n2 = n2;
        swap_prepare(p, s);
        if (s.ok == 0) {
            ilst = w.here;
            return 1;
        }
        if (s.ok == 1)
            for (int ph = 0; ph < 3; ph++) swap_apply(p, s, ph, 0, 1);
        walk_after(p, w);
    }
    ilst = w.here;
    return 0;
}

}  // namespace rb
}  // namespace xtg
