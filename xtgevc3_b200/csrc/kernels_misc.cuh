// Auxiliary kernels of the xTGEVC3 path: pencil norms and shift coefficients, the
// reversal/transposition that turns the left problem into a right problem, the
// write-back of untransformed eigenvectors, and the final column normalisation.
#pragma once
#include <climits>
#include "common.cuh"

namespace xtg {

template <class R> __device__ __forceinline__ R absval(R v) { return fabs(v); }
template <class R> __device__ __forceinline__ R absval(cplx<R> v) { return hypot(v.x, v.y); }

// Column sums of |S| and |P| over rows <= min(col + extra, n - 1): the 1-norms behind
// ascale/bscale (src/dtgevc3.cpp:1254-1270 with extra = 1; src/ztgevc3.cpp:528-542
// with extra = 0).  One warp per column.
template <class E, class R>
__global__ void colsum_kernel(const E *S, int lds, const E *P, int ldp, int n, int extra, R *sums)
{
    int col = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    int lane = threadIdx.x & 31;
    if (col >= n) return;
    int last = min(col + extra, n - 1);
    R ss = 0, sp = 0;
    for (int r = lane; r <= last; r += 32) {
        ss += absval(S[(size_t)r + (size_t)col * lds]);
        sp += absval(P[(size_t)r + (size_t)col * ldp]);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        ss += __shfl_xor_sync(0xffffffffu, ss, o);
        sp += __shfl_xor_sync(0xffffffffu, sp, o);
    }
    if (lane == 0) {
        sums[col] = ss;
        sums[n + col] = sp;
    }
}

// norms = {anorm, bnorm} computed by the caller.
template <class R>
__global__ void set_norms_kernel(R *norms, R anorm, R bnorm)
{
    norms[0] = anorm;
    norms[1] = bnorm;
}

// norms[0] = anorm, norms[1] = bnorm (single block).
template <class R>
__global__ void colmax_kernel(const R *sums, int n, R *norms)
{
    __shared__ R sa[32], sb[32];
    R a = 0, b = 0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        a = fmax(a, sums[i]);
        b = fmax(b, sums[n + i]);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        a = fmax(a, __shfl_xor_sync(0xffffffffu, a, o));
        b = fmax(b, __shfl_xor_sync(0xffffffffu, b, o));
    }
    if ((threadIdx.x & 31) == 0) {
        sa[threadIdx.x >> 5] = a;
        sb[threadIdx.x >> 5] = b;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < (int)(blockDim.x >> 5); w++) {
            a = fmax(a, sa[w]);
            b = fmax(b, sb[w]);
        }
        norms[0] = a;
        norms[1] = b;
    }
}

// Shift coefficients of every computed column (src/dtgevc3.cpp:716-725, 1372-1381):
//   t = 1 / max(|ar| ascale + |ai| ascale, |b| bscale, safemin)
//   ac = (t b bscale) ascale,  b_re = (t ar ascale) bscale,  b_im = (t ai ascale) bscale,
// with (ac, b) = (0, 1) for an infinite eigenvalue.  `neg_im` flips ai (the left problem
// solves for the conjugate eigenvalue).  smin is the pivot floor of the shifted solves:
// max(eps * (|ac| anorm + |b| bnorm), safemin).
template <class R>
__global__ void coef_real_kernel(const R *alphar, const R *alphai, const R *beta, const int *src,
                                 const uint8_t *kind, int m, int neg_im, const R *norms, R *coef)
{
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= m) return;
    const R safemin = limits<R>::safemin, eps = limits<R>::eps;
    R anorm = norms[0], bnorm = norms[1];
    R ascale = R(1) / fmax(anorm, safemin), bscale = R(1) / fmax(bnorm, safemin);
    int k = src[c];
    R ar = alphar[k], ai = kind[c] == kReal ? R(0) : alphai[k], b = beta[k];
    if (neg_im) ai = -ai;
    R den = fmax(fmax(fabs(ar) * ascale + fabs(ai) * ascale, fabs(b) * bscale), safemin);
    R t = R(1) / den;
    R ac = (t * b * bscale) * ascale;
    R br = (t * ar * ascale) * bscale;
    R bi = (t * ai * ascale) * bscale;
    if (fabs(b) <= safemin && (fabs(ar) + fabs(ai)) > safemin) {
        ac = R(0);
        br = R(1);
        bi = R(0);
    }
    coef[4 * c + 0] = ac;
    coef[4 * c + 1] = br;
    coef[4 * c + 2] = bi;
    coef[4 * c + 3] = fmax(eps * (fabs(ac) * anorm + (fabs(br) + fabs(bi)) * bnorm), safemin);
}

// Complex form (src/ztgevc3.cpp:148-156): t = 1 / max(|a| ascale, |b| bscale, safemin),
// ac = (t ascale) b bscale, bc = (t bscale) a ascale; `conj_ab` conjugates a and b (left).
template <class R>
__global__ void coef_cplx_kernel(const cplx<R> *alpha, const cplx<R> *beta, const int *src, int m,
                                 int conj_ab, const R *norms, R *coef)
{
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= m) return;
    const R safemin = limits<R>::safemin, eps = limits<R>::eps;
    R anorm = norms[0], bnorm = norms[1];
    R ascale = R(1) / fmax(anorm, safemin), bscale = R(1) / fmax(bnorm, safemin);
    int k = src[c];
    cplx<R> a = alpha[k], b = beta[k];
    if (conj_ab) {
        a = conjg(a);
        b = conjg(b);
    }
    R na = hypot(a.x, a.y), nb = hypot(b.x, b.y);
    R t = R(1) / fmax(fmax(na * ascale, nb * bscale), safemin);
    cplx<R> ac = (cplx<R>(t * ascale, R(0)) * b) * cplx<R>(bscale, R(0));
    cplx<R> bc = (cplx<R>(t * bscale, R(0)) * a) * cplx<R>(ascale, R(0));
    if (nb <= safemin && na > safemin) {
        ac = cplx<R>(0, 0);
        bc = cplx<R>(1, 0);
    }
    coef[6 * c + 0] = ac.x;
    coef[6 * c + 1] = ac.y;
    coef[6 * c + 2] = bc.x;
    coef[6 * c + 3] = bc.y;
    coef[6 * c + 4] = fmax(eps * (l1abs(ac) * anorm + l1abs(bc) * bnorm), safemin);
    coef[6 * c + 5] = R(0);
}

template <class E> __device__ __forceinline__ E maybe_conj(E v, int) { return v; }
template <class R> __device__ __forceinline__ cplx<R> maybe_conj(cplx<R> v, int c) { return c ? conjg(v) : v; }

// out(i, j) = f(in(n-1-j, n-1-i)), f = conj when `cj`: the left problem
// y^H (b S - a P) = 0 becomes the right problem of (F S^H F, F P^H F), F the reversal.
// 32 x 32 tiles through shared memory.  Output columns [c0, c1) only (rows n-c1 .. n-c0-1 of
// in), grid.y = ceil((c1 - c0) / 32); c0 = 0, c1 = n: the whole matrix.
template <class E>
__global__ void rev_transpose_kernel(const E *in, int ldi, E *out, int ldo, int n, int cj, int c0 = 0, int c1 = INT_MAX)
{
    __shared__ E tile[32][33];
    if (c1 > n) c1 = n;
    int i0 = blockIdx.x * 32, j0 = c0 + blockIdx.y * 32;
    // read in(n-1-j, n-1-i) for j in [j0, j0+32) (rows of in), i in [i0, i0+32) (cols of in)
    int tx = threadIdx.x, ty = threadIdx.y;  // 32 x 8
    for (int q = ty; q < 32; q += 8) {
        int j = j0 + tx, i = i0 + q;
        if (i < n && j < c1) tile[q][tx] = in[(size_t)(n - 1 - j) + (size_t)(n - 1 - i) * ldi];
    }
    __syncthreads();
    for (int q = ty; q < 32; q += 8) {
        int i = i0 + tx, j = j0 + q;
        if (i < n && j < c1) out[(size_t)i + (size_t)j * ldo] = maybe_conj(tile[tx][q], cj);
    }
}

// out[:, j] = in[:, n-1-j] for j < n (rows 0..rows-1).
template <class E>
__global__ void rev_columns_kernel(const E *in, int ldi, E *out, int ldo, int rows, int n)
{
    int j = blockIdx.y;
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < rows; r += gridDim.x * blockDim.x)
        out[(size_t)r + (size_t)j * ldo] = in[(size_t)r + (size_t)(n - 1 - j) * ldi];
}

// V[r, ccol[c]] = X[r, c] for r < kext[c], 0 otherwise (upstream write-back,
// src/dtgevc3.cpp:1455-1465).  With `rev` the row order is reversed (left problem):
// V[r, ccol[c]] = X[n-1-r, c].
template <class E>
__global__ void writeback_kernel(const E *X, int ldx, E *V, int ldv, int n, int m, const int *ccol,
                                 const int *kext, int rev)
{
    int c = blockIdx.y;
    if (c >= m) return;
    int ke = kext[c];
    E *out = V + (size_t)ccol[c] * ldv;
    const E *in = X + (size_t)c * ldx;
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
        int src = rev ? n - 1 - r : r;
        out[r] = src < ke ? in[src] : E(0);
    }
}

// Final normalisation (not done by the upstream code; LAPACK xTGEVC convention): every
// eigenvector is scaled so that max_i (|re_i| + |im_i|) = 1, a real pair (Re, Im) jointly.
// One CTA per eigenvector; the column (pair) is read twice, the second time from L2.
template <class R>
__global__ void normalize_real_kernel(R *V, int ldv, int n, const int *outcol, const uint8_t *kind, int m)
{
    int c = blockIdx.x;
    if (c >= m) return;
    uint8_t kd = kind[c];
    if (kd == kPairIm) return;
    R *v0 = V + (size_t)outcol[c] * ldv;  // a pair's (Re, Im) output columns are adjacent
    R *v1 = kd == kPairRe ? v0 + ldv : nullptr;
    R mx = 0;
    for (int r = threadIdx.x; r < n; r += blockDim.x) mx = fmax(mx, fabs(v0[r]) + (v1 ? fabs(v1[r]) : R(0)));
    __shared__ R red[32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = mx;
    __syncthreads();
    if (threadIdx.x < 32) {
        R v = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : R(0);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
        if (threadIdx.x == 0) red[0] = v;
    }
    __syncthreads();
    mx = red[0];
    if (!(mx > R(0))) return;
    R s = R(1) / mx;
    for (int r = threadIdx.x; r < n; r += blockDim.x) {
        v0[r] *= s;
        if (v1) v1[r] *= s;
    }
}

// One-pass normalisation (LAPACK convention: max_i |re| + |im| = 1, a real (Re, Im) pair
// jointly): one CTA of 256 threads per eigenvector (items: its first column), the rows
// (RPT per thread, coalesced) stay in registers between the maximum and the scaling, so
// each entry is read once and written once.  n <= 256 RPT.
template <class R, int RPT>
__global__ void __launch_bounds__(256) normalize_real_1p_kernel(R *V, int ldv, int n, const int *items,
                                                               const int *outcol, const uint8_t *kind, int nitems)
{
    const int it = blockIdx.x;
    if (it >= nitems) return;
    const int c = items[it];
    const bool pair = kind[c] == kPairRe;
    R *v0 = V + (size_t)outcol[c] * ldv;  // a pair's (Re, Im) output columns are adjacent
    R *v1 = v0 + ldv;
    R a[RPT], b[RPT];
    R mx = 0;
#pragma unroll
    for (int q = 0; q < RPT; q++) {
        const int r = threadIdx.x + 256 * q;
        a[q] = r < n ? v0[r] : R(0);
        b[q] = (pair && r < n) ? v1[r] : R(0);
        mx = fmax(mx, fabs(a[q]) + fabs(b[q]));
    }
    __shared__ R red[8];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = mx;
    __syncthreads();
    mx = red[0];
#pragma unroll
    for (int w = 1; w < 8; w++) mx = fmax(mx, red[w]);
    if (!(mx > R(0))) return;
    const R s = R(1) / mx;
#pragma unroll
    for (int q = 0; q < RPT; q++) {
        const int r = threadIdx.x + 256 * q;
        if (r < n) {
            v0[r] = a[q] * s;
            if (pair) v1[r] = b[q] * s;
        }
    }
}

template <class R, int RPT>
__global__ void __launch_bounds__(256) normalize_cplx_1p_kernel(cplx<R> *V, int ldv, int n, const int *outcol, int m)
{
    const int c = blockIdx.x;
    if (c >= m) return;
    cplx<R> *v = V + (size_t)outcol[c] * ldv;
    cplx<R> a[RPT];
    R mx = 0;
#pragma unroll
    for (int q = 0; q < RPT; q++) {
        const int r = threadIdx.x + 256 * q;
        a[q] = r < n ? v[r] : cplx<R>(R(0), R(0));
        mx = fmax(mx, l1abs(a[q]));
    }
    __shared__ R red[8];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = mx;
    __syncthreads();
    mx = red[0];
#pragma unroll
    for (int w = 1; w < 8; w++) mx = fmax(mx, red[w]);
    if (!(mx > R(0))) return;
    const R s = R(1) / mx;
#pragma unroll
    for (int q = 0; q < RPT; q++) {
        const int r = threadIdx.x + 256 * q;
        if (r < n) v[r] = s * a[q];
    }
}

template <class R>
__global__ void normalize_cplx_kernel(cplx<R> *V, int ldv, int n, const int *outcol, int m)
{
    int c = blockIdx.x;
    if (c >= m) return;
    cplx<R> *v = V + (size_t)outcol[c] * ldv;
    R mx = 0;
    for (int r = threadIdx.x; r < n; r += blockDim.x) mx = fmax(mx, l1abs(v[r]));
    __shared__ R red[32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = mx;
    __syncthreads();
    if (threadIdx.x < 32) {
        R w = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : R(0);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) w = fmax(w, __shfl_xor_sync(0xffffffffu, w, o));
        if (threadIdx.x == 0) red[0] = w;
    }
    __syncthreads();
    mx = red[0];
    if (!(mx > R(0))) return;
    R s = R(1) / mx;
    for (int r = threadIdx.x; r < n; r += blockDim.x) v[r] = s * v[r];
}

// Deferred guard scaling (see DiagArgs::pending): rows [0, rows) of every column with a
// pending factor are multiplied by it, and the factor is reset to 1.  One warp per column.
template <class E, class R>
__global__ void apply_pending_kernel(E *X, int ldx, R *pending, int m, int rows)
{
    const int c = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (c >= m) return;
    const R f = pending[c];
    if (f == R(1)) return;
    E *col = X + (size_t)c * ldx;
    for (int i = lane; i < rows; i += 32) col[i] = f * col[i];
    __syncwarp();
    if (lane == 0) pending[c] = R(1);
}

// pending[c] = 1 for every column.
template <class R>
__global__ void fill_one_kernel(R *p, int m)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < m) p[i] = R(1);
}

// Structure check of a real pencil given on the device (the block partition is planned on
// the host from alphai, without reading S): *flag becomes 1 when some subdiagonal entry
// S(k+1, k) is nonzero at a row k that does not start a complex pair, i.e. when the
// upstream partition rule (snap where S(k+1, k) != 0, src/dtgevc3.cpp:32-47) would
// differ from the planned one.  *flag is zeroed by the caller.
template <class R>
__global__ void subdiag_check_kernel(const R *S, int lds, int n, const uint8_t *pairstart, int *flag)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const bool bad = k + 1 < n && S[(size_t)(k + 1) + (size_t)k * lds] != R(0) && !pairstart[k];
    if (__syncthreads_or(bad) && threadIdx.x == 0) atomicExch(flag, 1);
}

// Diagonal of the identity (the rest zeroed by the caller): P of the standard problem.
template <class E>
__global__ void identity_diag_kernel(E *A, int lda, int n)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) A[(size_t)i * lda + i] = E(1);
}

// LAPACK xTREVC3's phase of a real 2x2 pair's eigenvector.  LAPACK seeds the pair (rows k,
// k+1 of T, standardised block, wi = sqrt|T(k,k+1)| sqrt|T(k+1,k)|) with one real and one
// imaginary entry (reference LAPACK dtrevc3.f, complex right / left eigenvector):
//   right: x(k) = 1, x(k+1) = i wi/T(k,k+1)   if |T(k,k+1)| >= |T(k+1,k)|,
//          x(k) = -wi/T(k+1,k), x(k+1) = i     otherwise;
//   left:  y(k) = wi/T(k,k+1), y(k+1) = i      if |T(k,k+1)| >= |T(k+1,k)|,
//          y(k) = 1, y(k+1) = -i wi/T(k+1,k)   otherwise,
// and only ever scales by positive reals after that.  One warp per pair (Re column c, Im
// column c + 1 of X in problem orientation, rows colk[c], colk[c] + 1; the left problem is
// reversed, so original row k is problem row colk[c] + 1 there) multiplies the pair by the
// unit complex number that gives its entry at the real seed row LAPACK's sign (the other
// seed row when that entry underflowed; a pair with neither is left alone).  Sp: S in
// problem orientation, where Sp(kk, kk+1) = T(k, k+1) and Sp(kk+1, kk) = T(k+1, k) for
// both sides.
template <class R>
__global__ void lapack_pair_phase_kernel(R *X, int ldx, int m, const int *colk, const int *kext,
                                         const uint8_t *kind, const R *Sp, int lds, int left)
{
    const int c = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (c >= m || kind[c] != kPairRe) return;  // uniform per warp
    const int kk = colk[c];
    R *xr = X + (size_t)c * ldx, *xi = xr + ldx;
    const R a = Sp[kk + (size_t)(kk + 1) * lds], b = Sp[kk + 1 + (size_t)kk * lds];
    const bool up = fabs(a) >= fabs(b);
    const R wi = sqrt(fabs(a)) * sqrt(fabs(b));
    const int rr = left ? kk + 1 : kk, ri = left ? kk : kk + 1;       // real / imaginary seed rows
    const R tr = left ? (up ? wi / a : R(1)) : (up ? R(1) : -wi / b);  // x(real row) = tr
    const R ti = left ? (up ? R(1) : -wi / b) : (up ? wi / a : R(1));  // x(imaginary row) = i ti
    R cr, ci;  // unit factor: sign(t) conj(x) / |x| at the real row, sign(t) i conj(x) / |x| at the other
    const R x0r = xr[rr], x0i = xi[rr], x0 = hypot(x0r, x0i);
    if (x0 > R(0)) {
        const R sg = tr < R(0) ? R(-1) : R(1);
        cr = sg * x0r / x0;
        ci = -sg * x0i / x0;
    } else {
        const R x1r = xr[ri], x1i = xi[ri], x1 = hypot(x1r, x1i);
        if (!(x1 > R(0))) return;
        const R sg = ti < R(0) ? R(-1) : R(1);
        cr = sg * x1i / x1;
        ci = sg * x1r / x1;
    }
    for (int i = lane; i < kext[c]; i += 32) {
        const R u = xr[i], v = xi[i];
        xr[i] = cr * u - ci * v;
        xi[i] = cr * v + ci * u;
    }
}

// Eigenvalue condition numbers (LAPACK xTGSNA, JOB = 'E'):
//   S(k) = sqrt(|y^H A x|^2 + |y^H B x|^2) / (||x||_2 ||y||_2)
// for the eigenvector columns x = VR(:, c), y = VL(:, c) of one selected eigenvalue, from
// AX = A VR and BX = B VR (columns c of the GEMM outputs).  A real pair (Re, Im columns c,
// c + 1) combines the four real products as LAPACK does (y^H A x = (xr.yr + xi.yi) +
// i (xi.yr - xr.yi)) and gives both columns the same S.  Norms are scaled by the column
// maximum (no overflow for any finite input); S = -1 marks a zero numerator (not for a pair,
// as in LAPACK dtgsna).  One warp per eigenvalue: items[w] is its
// first column, kind 0 real, 1 pair, 2 complex; s[w] and, for a pair, s[w + 1].
template <class R>
__device__ __forceinline__ R warp_sum(R v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

template <class R>
__device__ __forceinline__ R warp_maxabs(const R *col, int n, int lane)
{
    R mx = R(0);
    for (int i = lane; i < n; i += 32) mx = fmax(mx, fabs(col[i]));
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    return mx;
}

// ||(u, v)||_2 of one or two real vectors of length n (v may be null), scaled
template <class R>
__device__ __forceinline__ R warp_norm2(const R *u, const R *v, int n, int lane)
{
    R mx = warp_maxabs(u, n, lane);
    if (v) mx = fmax(mx, warp_maxabs(v, n, lane));
    if (!(mx > R(0))) return R(0);
    R acc = R(0);
    for (int i = lane; i < n; i += 32) {
        const R a = u[i] / mx;
        acc += a * a;
        if (v) {
            const R b = v[i] / mx;
            acc += b * b;
        }
    }
    return mx * sqrt(warp_sum(acc));
}

template <class R>
__global__ void eig_cond_kernel(int nitems, const int *items, const uint8_t *kinds, int n, const R *AX, const R *BX,
                                int ldx, const R *VL, int ldvl, const R *VR, int ldvr, R *s, const int *sidx)
{
    const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (w >= nitems) return;  // uniform per warp
    const int c = items[w], kind = kinds[w];
    R num = R(0), rn = R(0), ln = R(0);
    if (kind == 0) {  // real
        const R *x = VR + (size_t)c * ldvr, *y = VL + (size_t)c * ldvl;
        const R *ax = AX + (size_t)c * ldx, *bx = BX + (size_t)c * ldx;
        R ta = R(0), tb = R(0);
        for (int i = lane; i < n; i += 32) {
            ta += ax[i] * y[i];
            tb += bx[i] * y[i];
        }
        ta = warp_sum(ta);
        tb = warp_sum(tb);
        num = hypot(ta, tb);
        rn = warp_norm2<R>(x, nullptr, n, lane);
        ln = warp_norm2<R>(y, nullptr, n, lane);
    } else if (kind == 1) {  // real pair: (Re, Im) columns c, c + 1
        const R *xr = VR + (size_t)c * ldvr, *xi = xr + ldvr, *yr = VL + (size_t)c * ldvl, *yi = yr + ldvl;
        const R *ar = AX + (size_t)c * ldx, *ai = ar + ldx, *br = BX + (size_t)c * ldx, *bi = br + ldx;
        R a_rr = R(0), a_ri = R(0), a_ii = R(0), a_ir = R(0), b_rr = R(0), b_ri = R(0), b_ii = R(0), b_ir = R(0);
        for (int i = lane; i < n; i += 32) {
            a_rr += ar[i] * yr[i];
            a_ri += ar[i] * yi[i];
            a_ii += ai[i] * yi[i];
            a_ir += ai[i] * yr[i];
            b_rr += br[i] * yr[i];
            b_ri += br[i] * yi[i];
            b_ii += bi[i] * yi[i];
            b_ir += bi[i] * yr[i];
        }
        a_rr = warp_sum(a_rr); a_ri = warp_sum(a_ri); a_ii = warp_sum(a_ii); a_ir = warp_sum(a_ir);
        b_rr = warp_sum(b_rr); b_ri = warp_sum(b_ri); b_ii = warp_sum(b_ii); b_ir = warp_sum(b_ir);
        const R uha = hypot(a_rr + a_ii, a_ir - a_ri), uhb = hypot(b_rr + b_ii, b_ir - b_ri);
        num = hypot(uha, uhb);
        rn = warp_norm2<R>(xr, xi, n, lane);
        ln = warp_norm2<R>(yr, yi, n, lane);
    } else {  // complex: interleaved columns, y^H A x = sum conj(y_i) (A x)_i
        const R *x = VR + 2 * (size_t)c * ldvr, *y = VL + 2 * (size_t)c * ldvl;
        const R *ax = AX + 2 * (size_t)c * ldx, *bx = BX + 2 * (size_t)c * ldx;
        R ar_ = R(0), ai_ = R(0), br_ = R(0), bi_ = R(0);
        for (int i = lane; i < n; i += 32) {
            const R yr = y[2 * i], yi = y[2 * i + 1];
            ar_ += yr * ax[2 * i] + yi * ax[2 * i + 1];
            ai_ += yr * ax[2 * i + 1] - yi * ax[2 * i];
            br_ += yr * bx[2 * i] + yi * bx[2 * i + 1];
            bi_ += yr * bx[2 * i + 1] - yi * bx[2 * i];
        }
        num = hypot(hypot(warp_sum(ar_), warp_sum(ai_)), hypot(warp_sum(br_), warp_sum(bi_)));
        rn = warp_norm2<R>(x, nullptr, 2 * n, lane);
        ln = warp_norm2<R>(y, nullptr, 2 * n, lane);
    }
    if (lane == 0) {
        const R v = (num == R(0) && kind != 1) ? R(-1) : num / (rn * ln);  // LAPACK: no -1 for a pair
        s[sidx[w]] = v;
        if (kind == 1) s[sidx[w] + 1] = v;
    }
}

}  // namespace xtg
