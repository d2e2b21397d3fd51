// Batched form: many independent pencils of uneven order in one persistent launch.
//
// Work is split into units taken from a global queue (one atomic counter) by a grid of
// resident CTAs:
//   * a prep unit per pencil: the norms behind the shift coefficients
//     (src/dtgevc3.cpp:1254-1270), the complex-pair structure of the eigenvalues
//     (src/dtgevc3.cpp:1193-1207), the per-column shift coefficients of both problem
//     orientations (src/dtgevc3.cpp:716-725) and a partition of the columns into tiles
//     that never separate the two columns of a complex pair.  It ends by setting the
//     pencil's ready flag;
//   * a compute unit per (pencil, side, column tile): the whole right-looking blocked
//     substitution of the tile's eigenvectors (at most NT columns) with the tile X[0:c_hi,
//     tile] resident in shared memory, followed by the back-transform V = Z X (right) or
//     V = Q F X (left, F the row reversal) or the plain write-back.  A compute unit waits
//     (bounded) for its pencil's ready flag.
// The queue holds every pencil's prep unit before any compute unit, so a unit only ever
// waits for work that a running CTA has already taken: no deadlock is possible.  A wait
// that runs past its limit sets kErrWaitTimeout in the status word and the unit is
// skipped; the host turns the status into an error return.
//
// The per-tile algorithm is the one of the single-pencil path (left problem = right
// problem of (F S^T F, F P^T F); per-column overflow guards; seeds of the 1x1 and 2x2
// diagonal blocks), restricted to the tile's columns:
//     for each row block I = [r0, r1) of at most H rows, bottom to top from c_hi:
//         solve   (ac_c S_II - b_c P_II) x = X[I, c]     (one warp per eigenvector)
//         update  X[0:r0, tile] += [S[0:r0, I] | P[0:r0, I]] [-ac x ; b x]
// The update and the back-transform are CTA-wide GEMMs: 256 threads, each owning up to
// 4 rows (64 apart) x NT/4 columns of the output, the A operand (strips of S and P, or of
// Z / Q) staged through shared memory in chunks of KC columns by cp.async, double
// buffered; the B operand (the solved block, or X itself) is read from shared memory by
// broadcast.  The left problem's strips are rows of S and P: the stager reads them along
// the row (contiguous in memory) and transposes on the way into shared memory.
#pragma once
#include "common.cuh"
#include "kernels_diag.cuh"
#include "kernels_gemm.cuh"
#include "../../include/xtgevc3.h"

#include <type_traits>

namespace xtg {
namespace batch {

constexpr int THREADS = 256;
constexpr int WARPS = THREADS / 32;
constexpr int KC = 16;          // A-operand columns per staged chunk
constexpr int PASS = 256;       // output rows per GEMM pass: 64 row lanes x 4 row slots
constexpr int ALD = PASS + 1;   // leading dimension of a staged chunk

template <class T> struct PencilOf;
template <> struct PencilOf<double> { using type = xtgevc3_dpencil; };
template <> struct PencilOf<float> { using type = xtgevc3_spencil; };

// Row strides of the shared X tile and of the solved-block operand: 16-byte aligned rows,
// shifted by 16 bytes from one row to the next (conflict-free 16-byte accesses).
template <class T, int NT> struct Lds {
    static constexpr int X = NT + 16 / (int)sizeof(T);
    static constexpr int Y = NT + 16 / (int)sizeof(T);
};

__host__ __device__ inline int max_tiles(int n, int nt) { return (n + nt - 2) / (nt - 1); }

// Per-pencil workspace, written by the prep unit.
template <class T>
struct Work {
    T *coef;          // [2][n][4]: ac, b_re, b_im, smin per column (side 0 right, 1 left)
    T *norms;         // [2]: anorm, bnorm
    int *tiles;       // [2][maxt + 1]: first column of each tile, then n
    int *ntiles;      // [2]
    uint8_t *kind;    // [2][n]: kReal / kPairRe / kPairIm in problem orientation
    uint8_t *splitf;  // [2][n + 1]: rows j-1, j form a 2x2 diagonal block (orientation)
};

__host__ __device__ inline size_t align_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

template <class T>
__host__ __device__ inline size_t work_layout(unsigned char *base, int n, int nt, Work<T> *w)
{
    const int maxt = max_tiles(n, nt);
    size_t off = 0;
    auto take = [&](size_t bytes, size_t al) {
        off = align_up(off, al);
        size_t o = off;
        off += bytes;
        return o;
    };
    const size_t o_coef = take(sizeof(T) * 8 * (size_t)n, 16);
    const size_t o_norm = take(sizeof(T) * 2, 16);
    const size_t o_tiles = take(sizeof(int) * 2 * (size_t)(maxt + 1), 16);
    const size_t o_nt = take(sizeof(int) * 2, 16);
    const size_t o_kind = take(2 * (size_t)n, 16);
    const size_t o_split = take(2 * (size_t)(n + 1), 16);
    if (w) {
        w->coef = reinterpret_cast<T *>(base + o_coef);
        w->norms = reinterpret_cast<T *>(base + o_norm);
        w->tiles = reinterpret_cast<int *>(base + o_tiles);
        w->ntiles = reinterpret_cast<int *>(base + o_nt);
        w->kind = base + o_kind;
        w->splitf = base + o_split;
    }
    return align_up(off, 256);
}

template <class T>
struct Args {
    const typename PencilOf<T>::type *pencils;
    const int4 *units;       // {0: prep | 1: compute, pencil, side, tile}
    int nunits;
    unsigned char *ws;       // per-pencil workspaces
    const long long *woff;   // byte offset of each pencil's workspace
    int *ctrl;               // [0] queue counter, [1] status word, [2 + p] ready flag of pencil p
    int back;                // HOWMNY = 'B'
    int xrows;               // rows of the shared X tile (>= every n)
    long long spin_limit;    // polls of a ready flag before giving up
};

// FP64 runs its GEMMs on the DMMA path with A fragments from global memory (no staging),
// so its union region only holds the diagonal blocks.
template <class T, int NT, int H>
__host__ __device__ constexpr size_t smem_union_bytes()
{
    return std::is_same<T, double>::value
               ? 2 * (size_t)H * (H + 1) * sizeof(T)
               : (2 * (size_t)KC * ALD > 2 * (size_t)H * (H + 1) ? 2 * (size_t)KC * ALD : 2 * (size_t)H * (H + 1)) *
                     sizeof(T);
}

template <class T, int NT, int H>
__host__ __device__ inline size_t smem_bytes(int xrows)
{
    return (size_t)xrows * Lds<T, NT>::X * sizeof(T) + 2 * (size_t)H * Lds<T, NT>::Y * sizeof(T) +
           smem_union_bytes<T, NT, H>();
}

// ---- small helpers -------------------------------------------------------------------
template <class T>
__device__ __forceinline__ void cp_async_elem(T *smem, const T *gmem)
{
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    if constexpr (sizeof(T) == 8)
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem));
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gmem));
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

// CPT consecutive elements from 16-byte aligned shared memory.
template <int CPT>
__device__ __forceinline__ void load_vec(double (&v)[CPT], const double *p)
{
#pragma unroll
    for (int j = 0; j < CPT; j += 2) {
        const double2 t = *reinterpret_cast<const double2 *>(p + j);
        v[j] = t.x;
        v[j + 1] = t.y;
    }
}
template <int CPT>
__device__ __forceinline__ void load_vec(float (&v)[CPT], const float *p)
{
#pragma unroll
    for (int j = 0; j < CPT; j += 4) {
        const float4 t = *reinterpret_cast<const float4 *>(p + j);
        v[j] = t.x;
        v[j + 1] = t.y;
        v[j + 2] = t.z;
        v[j + 3] = t.w;
    }
}
template <int CPT>
__device__ __forceinline__ void store_vec(double *p, const double (&v)[CPT])
{
#pragma unroll
    for (int j = 0; j < CPT; j += 2) *reinterpret_cast<double2 *>(p + j) = make_double2(v[j], v[j + 1]);
}
template <int CPT>
__device__ __forceinline__ void store_vec(float *p, const float (&v)[CPT])
{
#pragma unroll
    for (int j = 0; j < CPT; j += 4)
        *reinterpret_cast<float4 *>(p + j) = make_float4(v[j], v[j + 1], v[j + 2], v[j + 3]);
}

// Output rows [p0 + rl + 64 q] x columns [cg * CPT, +CPT) of acc += A B over K, where the A
// chunks (KC columns of the pass's rows, as As[k * ALD + row]) are staged by `issue` and
// B is row-major in shared memory (row k at Bs + k * bld).
template <class T, int CPT, int QN, class Issue>
__device__ __forceinline__ void gemm_pass(T *As, const T *Bs, int bld, int K, Issue &&issue, T (&acc)[QN][CPT],
                                          int rl, int cg)
{
    const int nch = (K + KC - 1) / KC;
    issue(As, 0);
    cp_commit();
    for (int c = 0; c < nch; c++) {
        if (c + 1 < nch) issue(As + ((c + 1) & 1) * KC * ALD, (c + 1) * KC);
        cp_commit();
        cp_wait<1>();
        __syncthreads();
        const T *a = As + (c & 1) * KC * ALD + rl;
        const T *b = Bs + (size_t)c * KC * bld + cg * CPT;
        const int kn = min(KC, K - c * KC);
#pragma unroll 4
        for (int kk = 0; kk < kn; kk++) {
            T av[QN], bv[CPT];
#pragma unroll
            for (int q = 0; q < QN; q++) av[q] = a[kk * ALD + 64 * q];
            load_vec<CPT>(bv, b + kk * bld);
#pragma unroll
            for (int q = 0; q < QN; q++)
#pragma unroll
                for (int j = 0; j < CPT; j++) acc[q][j] = fma(av[q], bv[j], acc[q][j]);
        }
        __syncthreads();
    }
}

// Shared per-column description of the current tile, and the columns that start an
// eigenvector and are active in the current row block (real ones, complex pairs).
template <class T, int NT>
struct TileCols {
    T coef[NT][4];
    int colk[NT];
    int out[NT];
    uint8_t kind[NT];
    int lreal[NT], lpair[NT];
    int nreal, npair;
};

template <class T>
__device__ __forceinline__ void scale_col(T *col, int ld, int a, int b, T s, int lane)
{
    for (int i = a + lane; i < b; i += 32) col[(size_t)i * ld] *= s;
}

// ---- prep unit -------------------------------------------------------------------------
template <class T, int NT>
__device__ void prep_unit(const Args<T> &a, int p, unsigned char *smem)
{
    const auto &d = a.pencils[p];
    const int n = d.n;
    Work<T> w;
    work_layout<T>(a.ws + a.woff[p], n, NT, &w);
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    T *red = reinterpret_cast<T *>(smem);                  // [2][WARPS]
    T *ai = red + 2 * WARPS;                                // [n] alphai
    uint8_t *start = reinterpret_cast<uint8_t *>(ai + n);   // [n] complex pair starts here
    uint8_t *sub = start + n;                               // [n] S[k+1, k] != 0
    uint8_t *kinds = sub + n;                               // [2][n]
    for (int k = tid; k < n; k += THREADS) ai[k] = d.alphai[k];
    // 1-norm of the quasi-triangle of S and of P: column sums over rows <= col + 1
    T ma = T(0), mb = T(0);
    for (int col = wid; col < n; col += WARPS) {
        const int last = min(col + 1, n - 1);
        T ss = T(0), sp = T(0);
        for (int r = lane; r <= last; r += 32) {
            ss += fabs(d.S[(size_t)r + (size_t)col * d.lds]);
            sp += fabs(d.P[(size_t)r + (size_t)col * d.ldp]);
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            ss += __shfl_xor_sync(0xffffffffu, ss, o);
            sp += __shfl_xor_sync(0xffffffffu, sp, o);
        }
        ma = fmax(ma, ss);
        mb = fmax(mb, sp);
    }
    if (lane == 0) {
        red[wid] = ma;
        red[WARPS + wid] = mb;
    }
    __syncthreads();
    // pair starts: k starts a pair iff alphai[k] != 0, k + 1 < n, and the run of nonzero
    // alphai ending just above k has even length (the upstream scan pairs greedily from 0)
    for (int k = tid; k < n; k += THREADS) {
        int run = 0;
        while (k - run - 1 >= 0 && ai[k - run - 1] != T(0)) run++;
        start[k] = (ai[k] != T(0) && k + 1 < n && (run & 1) == 0) ? 1 : 0;
        sub[k] = (k + 1 < n) && d.S[(size_t)(k + 1) + (size_t)k * d.lds] != T(0);
    }
    __syncthreads();
    if (tid == 0) {
        T x = red[0], y = red[WARPS];
        for (int q = 1; q < WARPS; q++) {
            x = fmax(x, red[q]);
            y = fmax(y, red[WARPS + q]);
        }
        red[0] = x;
        red[WARPS] = y;
        w.norms[0] = x;
        w.norms[1] = y;
    }
    // kinds and block-split flags of both orientations
    for (int c = tid; c < n; c += THREADS) {
        const uint8_t kr = start[c] ? kPairRe : (c > 0 && start[c - 1] ? kPairIm : kReal);
        const uint8_t kl = (c <= n - 2 && start[n - 2 - c]) ? kPairRe : (start[n - 1 - c] ? kPairIm : kReal);
        kinds[c] = kr;
        kinds[n + c] = kl;
        w.kind[c] = kr;
        w.kind[n + c] = kl;
    }
    for (int j = tid; j <= n; j += THREADS) {
        uint8_t fr = 0, fl = 0;
        if (j >= 1 && j < n) {
            fr = sub[j - 1] || start[j - 1];
            const int kq = n - 1 - j;
            fl = sub[kq] || start[kq];
        }
        w.splitf[j] = fr;
        w.splitf[(n + 1) + j] = fl;
    }
    __syncthreads();
    // shift coefficients (the single-pencil path's coef_real_kernel, both orientations)
    {
        const T safemin = limits<T>::safemin, eps = limits<T>::eps;
        const T anorm = red[0], bnorm = red[WARPS];
        const T ascale = T(1) / fmax(anorm, safemin), bscale = T(1) / fmax(bnorm, safemin);
        for (int q = tid; q < 2 * n; q += THREADS) {
            const int side = q / n, c = q % n;
            const uint8_t kd = kinds[q];
            int src;
            if (side == 0) src = kd == kPairIm ? c - 1 : c;
            else src = kd == kReal ? n - 1 - c : (kd == kPairRe ? n - 2 - c : n - 1 - c);
            T ar = d.alphar[src], ai = kd == kReal ? T(0) : d.alphai[src], b = d.beta[src];
            if (side == 1) ai = -ai;
            const T den = fmax(fmax(fabs(ar) * ascale + fabs(ai) * ascale, fabs(b) * bscale), safemin);
            const T t = T(1) / den;
            T ac = (t * b * bscale) * ascale;
            T br = (t * ar * ascale) * bscale;
            T bi = (t * ai * ascale) * bscale;
            if (fabs(b) <= safemin && (fabs(ar) + fabs(ai)) > safemin) {
                ac = T(0);
                br = T(1);
                bi = T(0);
            }
            T *cf = w.coef + 4 * (size_t)q;
            cf[0] = ac;
            cf[1] = br;
            cf[2] = bi;
            cf[3] = fmax(eps * (fabs(ac) * anorm + (fabs(br) + fabs(bi)) * bnorm), safemin);
        }
    }
    // column tiles: NT columns, one fewer when the last would be the Re column of a pair
    if (tid < 2) {
        const int side = tid, maxt = max_tiles(n, NT);
        int *tl = w.tiles + side * (maxt + 1);
        int c = 0, t = 0;
        while (c < n) {
            tl[t++] = c;
            int e = min(c + NT, n);
            if (e < n && kinds[side * n + e - 1] == kPairRe) e -= 1;
            c = e;
        }
        tl[t] = n;
        w.ntiles[side] = t;
    }
    __threadfence();
    __syncthreads();
    if (tid == 0) atomicExch(a.ctrl + 2 + p, 1);
}

// ---- one eigenvector item of a row block -------------------------------------------------
// The solve of diag_solve_real (kernels_diag.cuh) on a shared-memory tile column: X rows are
// Xc[i * XLD], the block's update operand goes to Ys rows i (-ac x) and jnb + i (b x).
template <class T, int NT, int H>
__device__ void solve_item(const TileCols<T, NT> &tc, int j, int r0, int r1, const T *Sd, const T *Pd,
                           uint64_t sec, T *Xs, T *Ys, bool left, T thr_rhs, T thr_upd, int lane)
{
    constexpr int XLD = Lds<T, NT>::X, YLD = Lds<T, NT>::Y, DLD = H + 1;
    const uint8_t kd = tc.kind[j];
    const int k = tc.colk[j];
    const int kl = k - r0;
    const bool diag = k < r1;
    const int jnb = r1 - r0;
    const T ac = tc.coef[j][0], br = tc.coef[j][1], bi = tc.coef[j][2], smin = tc.coef[j][3];
    T *colr = Xs + j;
    const int nrows = diag ? kl : jnb;
    if (kd == kReal) {
        const int top = k;
        auto W = [&](int i, int c) -> T { return ac * Sd[i + c * DLD] - br * Pd[i + c * DLD]; };
        T r[2];
        T seed = diag ? T(1) : T(0);
#pragma unroll
        for (int s = 0; s < 2; s++) {
            const int i = lane + 32 * s;
            T v = T(0);
            if (i < nrows) v = diag ? -W(i, kl) : colr[(size_t)(r0 + i) * XLD];
            r[s] = v;
        }
        if (nrows > 0) {
            const T mx = warp_max(fmax(fabs(r[0]), fabs(r[1])));
            if (mx > thr_rhs) {
                const T sc = thr_rhs / mx;
                r[0] *= sc; r[1] *= sc; seed *= sc;
                if (!diag) { scale_col(colr, XLD, 0, r0, sc, lane); scale_col(colr, XLD, r1, top + 1, sc, lane); }
            }
        }
        Factors<T> F;
        factor_rows(F, sec, nrows, lane, smin, W);
        // The substitution runs without the per-row cap (in the loop it costs this kernel its
        // second CTA per SM); a block in which a component passed the cap, or overflowed, is
        // solved again from its right-hand side with it.  Factors applied to the stored rows
        // in the first pass (acc) carry over; a non-finite maximum is left to the second.
        const T cap = limits<T>::big / T(4096);
        const T r_in[2] = {r[0], r[1]};
        T acc = T(1);
        auto rescale = [&](T (&rr)[2], T sc) {  // the whole column, by sc
            rr[0] *= sc; rr[1] *= sc; seed *= sc; acc *= sc;
            if (!diag) { scale_col(colr, XLD, 0, r0, sc, lane); scale_col(colr, XLD, r1, top + 1, sc, lane); }
        };
        auto mid = [&](T (&rr)[2], int jtop) {
            const T mx = warp_max(lane <= jtop ? fabs(rr[0]) : T(0));
            if (mx > thr_rhs && mx <= limits<T>::big) rescale(rr, thr_rhs / mx);
        };
        back_substitute_loop(r, F, sec, nrows, lane, W, 0, make_guard<false>(cap, thr_rhs, mid, rescale));
        if (__any_sync(0xffffffffu, !(fabs(r[0]) <= cap) || !(fabs(r[1]) <= cap))) {
            r[0] = acc * r_in[0];
            r[1] = acc * r_in[1];
            back_substitute_loop(r, F, sec, nrows, lane, W, 0, make_guard<true>(cap, thr_rhs, mid, rescale));
        }
        T x[2];
#pragma unroll
        for (int s = 0; s < 2; s++) {
            const int i = lane + 32 * s;
            x[s] = i < nrows ? r[s] : (diag && i == kl ? seed : T(0));
        }
        const T mx = warp_max(fmax(fmax(fabs(ac * x[0]), fabs(br * x[0])), fmax(fabs(ac * x[1]), fabs(br * x[1]))));
        if (mx > thr_upd) {
            const T sc = thr_upd / mx;
            x[0] *= sc; x[1] *= sc;
            if (!diag) { scale_col(colr, XLD, 0, r0, sc, lane); scale_col(colr, XLD, r1, top + 1, sc, lane); }
        }
#pragma unroll
        for (int s = 0; s < 2; s++) {
            const int i = lane + 32 * s;
            if (i < jnb) {
                colr[(size_t)(r0 + i) * XLD] = x[s];
                Ys[i * YLD + j] = -ac * x[s];
                Ys[(jnb + i) * YLD + j] = br * x[s];
            }
        }
    } else {
        using C = cplx<T>;
        T *coli = colr + 1;
        const int top = k + 1;
        const C b(br, bi);
        auto W = [&](int i, int c) -> C {
            const T s = Sd[i + c * DLD], p = Pd[i + c * DLD];
            return C(ac * s - br * p, -bi * p);
        };
        C seed0(0, 0), seed1(0, 0);
        if (diag) {
            if (!left) {  // (x_k, x_k+1) = (-w12, w11), src/dtgevc3.cpp:727-740
                seed0 = -W(kl, kl + 1);
                seed1 = W(kl, kl);
            } else {      // the left problem's seed, mirrored: (w22, -w21)
                seed0 = W(kl + 1, kl + 1);
                seed1 = -W(kl + 1, kl);
            }
        }
        C r[2];
#pragma unroll
        for (int s = 0; s < 2; s++) {
            const int i = lane + 32 * s;
            C v(0, 0);
            if (i < nrows) {
                if (diag) v = -(W(i, kl) * seed0 + W(i, kl + 1) * seed1);
                else v = C(colr[(size_t)(r0 + i) * XLD], coli[(size_t)(r0 + i) * XLD]);
            }
            r[s] = v;
        }
        if (nrows > 0) {
            const T mx = warp_max(fmax(fmax(fabs(r[0].x), fabs(r[0].y)), fmax(fabs(r[1].x), fabs(r[1].y))));
            if (mx > thr_rhs) {
                const T sc = thr_rhs / mx;
                r[0] = sc * r[0]; r[1] = sc * r[1]; seed0 = sc * seed0; seed1 = sc * seed1;
                if (!diag) {
                    scale_col(colr, XLD, 0, r0, sc, lane); scale_col(colr, XLD, r1, top + 1, sc, lane);
                    scale_col(coli, XLD, 0, r0, sc, lane); scale_col(coli, XLD, r1, top + 1, sc, lane);
                }
            }
        }
        Factors<C> F;
        factor_rows(F, sec, nrows, lane, smin, W);
        const T cap = limits<T>::big / T(4096);  // detect and redo, as for a real column
        const C r_in[2] = {r[0], r[1]};
        T acc = T(1);
        auto rescale = [&](C (&rr)[2], T sc) {  // the whole column pair, by sc
            rr[0] = sc * rr[0]; rr[1] = sc * rr[1]; seed0 = sc * seed0; seed1 = sc * seed1; acc *= sc;
            if (!diag) {
                scale_col(colr, XLD, 0, r0, sc, lane); scale_col(colr, XLD, r1, top + 1, sc, lane);
                scale_col(coli, XLD, 0, r0, sc, lane); scale_col(coli, XLD, r1, top + 1, sc, lane);
            }
        };
        auto mid = [&](C (&rr)[2], int jtop) {
            const T mx = warp_max(lane <= jtop ? fmax(fabs(rr[0].x), fabs(rr[0].y)) : T(0));
            if (mx > thr_rhs && mx <= limits<T>::big) rescale(rr, thr_rhs / mx);
        };
        back_substitute_loop(r, F, sec, nrows, lane, W, 0, make_guard<false>(cap, thr_rhs, mid, rescale));
        if (__any_sync(0xffffffffu, !(mag(r[0]) <= cap) || !(mag(r[1]) <= cap))) {
            r[0] = acc * r_in[0];
            r[1] = acc * r_in[1];
            back_substitute_loop(r, F, sec, nrows, lane, W, 0, make_guard<true>(cap, thr_rhs, mid, rescale));
        }
        C x[2];
#pragma unroll
        for (int s = 0; s < 2; s++) {
            const int i = lane + 32 * s;
            x[s] = i < nrows ? r[s] : (diag && i == kl ? seed0 : (diag && i == kl + 1 ? seed1 : C(0, 0)));
        }
        T mx = T(0);
#pragma unroll
        for (int s = 0; s < 2; s++) {
            const C ys = ac * x[s], yp = b * x[s];
            mx = fmax(mx, fmax(fmax(fabs(ys.x), fabs(ys.y)), fmax(fabs(yp.x), fabs(yp.y))));
        }
        mx = warp_max(mx);
        if (mx > thr_upd) {
            const T sc = thr_upd / mx;
            x[0] = sc * x[0]; x[1] = sc * x[1];
            if (!diag) {
                scale_col(colr, XLD, 0, r0, sc, lane); scale_col(colr, XLD, r1, top + 1, sc, lane);
                scale_col(coli, XLD, 0, r0, sc, lane); scale_col(coli, XLD, r1, top + 1, sc, lane);
            }
        }
#pragma unroll
        for (int s = 0; s < 2; s++) {
            const int i = lane + 32 * s;
            if (i < jnb) {
                colr[(size_t)(r0 + i) * XLD] = x[s].x;
                coli[(size_t)(r0 + i) * XLD] = x[s].y;
                const C yp = b * x[s];
                Ys[i * YLD + j] = -ac * x[s].x;
                Ys[i * YLD + j + 1] = -ac * x[s].y;
                Ys[(jnb + i) * YLD + j] = yp.x;
                Ys[(jnb + i) * YLD + j + 1] = yp.y;
            }
        }
    }
}

// ---- grouped solves: 32/G eigenvectors per warp ------------------------------------------
// The block solve of solve_item, with one eigenvector per group of G = H/4 lanes instead of
// per warp: lane gl of a group owns rows gl + G s (s < 4).  All groups of a warp step
// through the block's rows together (one shuffle latency per row serves 32/G
// eigenvectors); a group whose eigenvector has fewer rows in this block idles through the
// extra steps.  One pass handles real eigenvectors, another complex pairs, so the groups
// of a warp never take different arithmetic paths.
template <class E, int R>
__device__ __forceinline__ E sel_slot(const E (&v)[R], int s)
{
    E x = v[0];
#pragma unroll
    for (int q = 1; q < R; q++) x = (s == q) ? v[q] : x;
    return x;
}
template <class E, int R>
__device__ __forceinline__ void put_slot(E (&v)[R], int s, E x)
{
#pragma unroll
    for (int q = 0; q < R; q++)
        if (q == s) v[q] = x;
}
template <int G, class T>
__device__ __forceinline__ T group_max(T v)
{
#pragma unroll
    for (int o = G / 2; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}
template <class T> __device__ __forceinline__ T cmag(T v) { return fabs(v); }
template <class T> __device__ __forceinline__ T cmag(cplx<T> v) { return fmax(fabs(v.x), fabs(v.y)); }

template <class E, int R>
struct FactorsR {
    E inv1[R], fa[R], fb[R], fm[R], fu[R];
    bool sw[R];
};

template <class T, int NT, int H, bool PAIR>
__device__ void solve_group(const TileCols<T, NT> &tc, const int *list, int cnt, int r0, int r1, const T *Sd,
                            const T *Pd, uint64_t sec, T *Xs, T *Ys, bool left, T thr_rhs, T thr_upd)
{
    constexpr int XLD = Lds<T, NT>::X, YLD = Lds<T, NT>::Y, DLD = H + 1;
    constexpr int G = H / 4, R = 4, PER = 32 / G;
    using E = typename std::conditional<PAIR, cplx<T>, T>::type;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int gl = lane & (G - 1), gbase = lane & ~(G - 1), sg = lane / G;
    const int jnb = r1 - r0;
    for (int base = wid * PER; base < cnt; base += WARPS * PER) {
        const int it = base + sg;
        const bool has = it < cnt;  // groups past the list redo the first item and discard it
        const int j = list[has ? it : base];
        const int k = tc.colk[j], kl = k - r0;
        const bool diag = k < r1;
        const T ac = tc.coef[j][0], br = tc.coef[j][1], bi = tc.coef[j][2], smin = tc.coef[j][3];
        const int nrows = diag ? kl : jnb;
        int maxn = nrows;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) maxn = max(maxn, __shfl_xor_sync(0xffffffffu, maxn, o));
        T *colr = Xs + j;
        T *coli = colr + 1;
        const int top = PAIR ? k + 1 : k;
        auto W = [&](int i, int c) -> E {
            const T sv = Sd[i + c * DLD], pv = Pd[i + c * DLD];
            if constexpr (PAIR) return E(ac * sv - br * pv, -bi * pv);
            else return ac * sv - br * pv;
        };
        auto scale_outside = [&](T sc) {  // rows of the column outside the block
            if (diag || !has) return;
            for (int i = gl; i < r0; i += G) {
                colr[(size_t)i * XLD] *= sc;
                if (PAIR) coli[(size_t)i * XLD] *= sc;
            }
            for (int i = r1 + gl; i <= top; i += G) {
                colr[(size_t)i * XLD] *= sc;
                if (PAIR) coli[(size_t)i * XLD] *= sc;
            }
        };
        E seed0 = E(0), seed1 = E(0);
        if constexpr (PAIR) {
            if (diag) {
                if (!left) {  // (x_k, x_k+1) = (-w12, w11), src/dtgevc3.cpp:727-740
                    seed0 = -W(kl, kl + 1);
                    seed1 = W(kl, kl);
                } else {      // the left problem's seed, mirrored: (w22, -w21)
                    seed0 = W(kl + 1, kl + 1);
                    seed1 = -W(kl + 1, kl);
                }
            }
        } else {
            seed0 = diag ? T(1) : T(0);
        }
        E r[R];
#pragma unroll
        for (int q = 0; q < R; q++) {
            const int i = gl + G * q;
            E v = E(0);
            if (i < nrows) {
                if (diag) {
                    if constexpr (PAIR) v = -(W(i, kl) * seed0 + W(i, kl + 1) * seed1);
                    else v = -W(i, kl);
                } else {
                    if constexpr (PAIR) v = E(colr[(size_t)(r0 + i) * XLD], coli[(size_t)(r0 + i) * XLD]);
                    else v = colr[(size_t)(r0 + i) * XLD];
                }
            }
            r[q] = v;
        }
        {  // guard before the solve (bignum/10)
            T mx = T(0);
#pragma unroll
            for (int q = 0; q < R; q++) mx = fmax(mx, cmag(r[q]));
            mx = group_max<G>(mx);
            if (nrows > 0 && mx > thr_rhs) {
                const T sc = thr_rhs / mx;
#pragma unroll
                for (int q = 0; q < R; q++) r[q] = sc * r[q];
                seed0 = sc * seed0;
                seed1 = sc * seed1;
                scale_outside(sc);
            }
        }
        // factors of the owned rows: 1 / w_ii, and the pivoted LU of each 2x2 block
        FactorsR<E, R> F;
#pragma unroll
        for (int q = 0; q < R; q++) {
            const int i = gl + G * q;
            F.inv1[q] = E(0);
            F.fa[q] = F.fb[q] = F.fm[q] = F.fu[q] = E(0);
            F.sw[q] = false;
            if (i < nrows) {
                F.inv1[q] = rcp(floor_pivot(W(i, i), smin));
                if (i >= 1 && ((sec >> i) & 1ull)) {
                    const E w11 = W(i - 1, i - 1), w12 = W(i - 1, i), w21 = W(i, i - 1), w22 = W(i, i);
                    const bool swp = mag(w21) > mag(w11);
                    const E pa = swp ? w21 : w11, pb = swp ? w22 : w12, pc = swp ? w11 : w21, pd = swp ? w12 : w22;
                    const E ia = rcp(floor_pivot(pa, smin));
                    const E m = pc * ia;
                    F.fa[q] = ia;
                    F.fb[q] = pb;
                    F.fm[q] = m;
                    F.fu[q] = rcp(floor_pivot(pd - m * pb, smin));
                    F.sw[q] = swp;
                }
            }
        }
        // back substitution, warp-uniform row loop
        bool checked = H <= kMidRow || maxn <= kMidRow;  // blocks of H <= 32 rows need no check
        for (int jr = maxn - 1; jr >= 0;) {
            if (H > kMidRow && !checked && jr < kMidRow) {  // growth check of the block's upper rows
                checked = true;
                T mx = T(0);
#pragma unroll
                for (int q = 0; q < R; q++)
                    if (gl + G * q <= jr) mx = fmax(mx, cmag(r[q]));
                mx = group_max<G>(mx);
                if (nrows > kMidRow && mx > thr_rhs) {
                    const T sc = thr_rhs / mx;
#pragma unroll
                    for (int q = 0; q < R; q++) r[q] = sc * r[q];
                    seed0 = sc * seed0;
                    seed1 = sc * seed1;
                    scale_outside(sc);
                }
            }
            const bool act = jr < nrows;
            if (jr >= 1 && ((sec >> jr) & 1ull)) {
                const int pr = jr - 1, qr = jr;
                const int sp = pr / G, sq = qr / G, op = gbase + (pr & (G - 1)), oq = gbase + (qr & (G - 1));
                const E rp = shfl(sel_slot(r, sp), op);
                const E rq = sel_slot(r, sq);
                bool swp = F.sw[0];
                E ia = F.fa[0], b = F.fb[0], m = F.fm[0], iu = F.fu[0];
#pragma unroll
                for (int q = 1; q < R; q++)
                    if (q == sq) {
                        swp = F.sw[q];
                        ia = F.fa[q];
                        b = F.fb[q];
                        m = F.fm[q];
                        iu = F.fu[q];
                    }
                const E e1 = swp ? rq : rp, e2 = swp ? rp : rq;
                E xq = (e2 - m * e1) * iu;
                E xp = (e1 - b * xq) * ia;
                xq = shfl(xq, oq);
                xp = shfl(xp, oq);
                if (act) {
                    if (gl == (pr & (G - 1))) put_slot(r, sp, xp);
                    if (gl == (qr & (G - 1))) put_slot(r, sq, xq);
#pragma unroll
                    for (int q = 0; q < R; q++) {
                        const int i = gl + G * q;
                        if (i < pr) r[q] = r[q] - (W(i, pr) * xp + W(i, qr) * xq);
                    }
                }
                jr -= 2;
            } else {
                const int sj = jr / G, oj = gbase + (jr & (G - 1));
                const E x = shfl(sel_slot(r, sj) * sel_slot(F.inv1, sj), oj);
                if (act) {
                    if (gl == (jr & (G - 1))) put_slot(r, sj, x);
#pragma unroll
                    for (int q = 0; q < R; q++) {
                        const int i = gl + G * q;
                        if (i < jr) r[q] = r[q] - W(i, jr) * x;
                    }
                }
                jr -= 1;
            }
        }
        // the block column: solution rows, seed, zeros below it
        E x[R];
#pragma unroll
        for (int q = 0; q < R; q++) {
            const int i = gl + G * q;
            x[q] = i < nrows ? r[q] : (diag && i == kl ? seed0 : (PAIR && diag && i == kl + 1 ? seed1 : E(0)));
        }
        const E bc = [&] {
            if constexpr (PAIR) return E(br, bi);
            else return br;
        }();
        {  // guard before the update (bignum / block height)
            T mx = T(0);
#pragma unroll
            for (int q = 0; q < R; q++) mx = fmax(mx, fmax(cmag(ac * x[q]), cmag(bc * x[q])));
            mx = group_max<G>(mx);
            if (mx > thr_upd) {
                const T sc = thr_upd / mx;
#pragma unroll
                for (int q = 0; q < R; q++) x[q] = sc * x[q];
                scale_outside(sc);
            }
        }
        if (has) {
#pragma unroll
            for (int q = 0; q < R; q++) {
                const int i = gl + G * q;
                if (i < jnb) {
                    const E ys = -(ac * x[q]), yp = bc * x[q];
                    if constexpr (PAIR) {
                        colr[(size_t)(r0 + i) * XLD] = x[q].x;
                        coli[(size_t)(r0 + i) * XLD] = x[q].y;
                        Ys[i * YLD + j] = ys.x;
                        Ys[i * YLD + j + 1] = ys.y;
                        Ys[(jnb + i) * YLD + j] = yp.x;
                        Ys[(jnb + i) * YLD + j + 1] = yp.y;
                    } else {
                        colr[(size_t)(r0 + i) * XLD] = x[q];
                        Ys[i * YLD + j] = ys;
                        Ys[(jnb + i) * YLD + j] = yp;
                    }
                }
            }
        }
    }
}

// ---- compute unit ------------------------------------------------------------------------
template <class T, int NT, int H, int QN>
__device__ __forceinline__ void update_pass(const typename PencilOf<T>::type &d, bool left, int r0, int jnb, int p0,
                                            int rows, T *Xs, const T *Ys, T *As)
{
    constexpr int XLD = Lds<T, NT>::X, YLD = Lds<T, NT>::Y, CPT = NT / 4;
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    const int rl = (wid >> 2) * 32 + lane, cg = wid & 3;
    const int n = d.n, K = 2 * jnb;
    T acc[QN][CPT];
#pragma unroll
    for (int q = 0; q < QN; q++) {
        const int i = rl + 64 * q;
        if (i < rows) load_vec<CPT>(acc[q], Xs + (size_t)(p0 + i) * XLD + cg * CPT);
        else
#pragma unroll
            for (int j = 0; j < CPT; j++) acc[q][j] = T(0);
    }
    auto issue = [&](T *dst, int k0) {
        if (!left) {
            if (tid < rows) {
                const int row = p0 + tid;
#pragma unroll 4
                for (int kk = 0; kk < KC; kk++) {
                    const int k = k0 + kk;
                    if (k < K) {
                        const T *src = k < jnb ? d.S + (size_t)row + (size_t)(r0 + k) * d.lds
                                               : d.P + (size_t)row + (size_t)(r0 + k - jnb) * d.ldp;
                        cp_async_elem(dst + kk * ALD + tid, src);
                    }
                }
            }
        } else {
            const int kk = tid % KC, k = k0 + kk;
            if (k < K) {
                const int rs = k < jnb ? n - 1 - (r0 + k) : n - 1 - (r0 + k - jnb);
                const T *base = k < jnb ? d.S + rs : d.P + rs;
                const size_t ld = k < jnb ? (size_t)d.lds : (size_t)d.ldp;
                for (int r = tid / KC; r < rows; r += THREADS / KC)
                    cp_async_elem(dst + kk * ALD + r, base + (size_t)(n - 1 - (p0 + r)) * ld);
            }
        }
    };
    gemm_pass<T, CPT, QN>(As, Ys, YLD, K, issue, acc, rl, cg);
#pragma unroll
    for (int q = 0; q < QN; q++) {
        const int i = rl + 64 * q;
        if (i < rows) store_vec<CPT>(Xs + (size_t)(p0 + i) * XLD + cg * CPT, acc[q]);
    }
}

template <class T, int NT, int H, int QN>
__device__ __forceinline__ void back_pass(const typename PencilOf<T>::type &d, bool left, int khi, int p0, int rows,
                                          const T *Xs, T *As, const TileCols<T, NT> &tc, int ntc)
{
    constexpr int XLD = Lds<T, NT>::X, CPT = NT / 4;
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    const int rl = (wid >> 2) * 32 + lane, cg = wid & 3;
    const int n = d.n;
    T acc[QN][CPT];
#pragma unroll
    for (int q = 0; q < QN; q++)
#pragma unroll
        for (int j = 0; j < CPT; j++) acc[q][j] = T(0);
    const T *Zb = left ? d.Q : d.Z;
    const size_t ldz = left ? (size_t)d.ldq : (size_t)d.ldz;
    auto issue = [&](T *dst, int k0) {
        if (tid < rows) {
            const int row = p0 + tid;
#pragma unroll 4
            for (int kk = 0; kk < KC; kk++) {
                const int k = k0 + kk;
                if (k < khi) {
                    const int zc = left ? n - 1 - k : k;
                    cp_async_elem(dst + kk * ALD + tid, Zb + (size_t)row + (size_t)zc * ldz);
                }
            }
        }
    };
    gemm_pass<T, CPT, QN>(As, Xs, XLD, khi, issue, acc, rl, cg);
    T *V = left ? d.VL : d.VR;
    const size_t ldv = left ? (size_t)d.ldvl : (size_t)d.ldvr;
#pragma unroll
    for (int q = 0; q < QN; q++) {
        const int i = rl + 64 * q;
        if (i < rows)
#pragma unroll
            for (int j = 0; j < CPT; j++) {
                const int c = cg * CPT + j;
                if (c < ntc) V[(size_t)(p0 + i) + (size_t)tc.out[c] * ldv] = acc[q][j];
            }
    }
}

// ---- FP64 passes on the DMMA tensor path ---------------------------------------------------
// One warp per 32-row tile of the output (four m8 tiles) by NT columns (NT/8 n8 tiles) of
// mma.m8n8k4.f64.  The A fragments (lane (g, t): row g, K index t) are loaded from global
// memory: eight consecutive rows of one column (right problem) or four consecutive rows
// of eight columns (left problem, A = rows of S and P) -- 256 B in eight full sectors
// either way -- one 16-deep K chunk ahead of the MMAs.  B fragments come from shared
// memory.  Warps work on disjoint rows, so a pass needs no CTA-wide synchronisation.
template <int NT, class LoadA>
__device__ __forceinline__ void dmma_tile(LoadA &&loadA, const double *Bs, int bld, int K,
                                          double (&acc)[4][NT / 8][2], int lane)
{
    constexpr int NJ = NT / 8;
    const int g = lane >> 2, t = lane & 3;
    double cur[4][4], nxt[4][4];
    auto fetch = [&](double (&dst)[4][4], int kc) {
#pragma unroll
        for (int s = 0; s < 4; s++) {
            const int k = kc + 4 * s + t;
#pragma unroll
            for (int i = 0; i < 4; i++) dst[s][i] = k < K ? loadA(k, i) : 0.0;
        }
    };
    fetch(cur, 0);
    for (int kc = 0; kc < K; kc += 16) {
        if (kc + 16 < K) fetch(nxt, kc + 16);
#pragma unroll
        for (int s = 0; s < 4; s++) {
            const int k = kc + 4 * s + t;
            double b[NJ];
#pragma unroll
            for (int j = 0; j < NJ; j++) b[j] = k < K ? Bs[(size_t)k * bld + 8 * j + g] : 0.0;
#pragma unroll
            for (int i = 0; i < 4; i++)
#pragma unroll
                for (int j = 0; j < NJ; j++) dmma884(acc[i][j][0], acc[i][j][1], cur[s][i], b[j]);
        }
#pragma unroll
        for (int s = 0; s < 4; s++)
#pragma unroll
            for (int i = 0; i < 4; i++) cur[s][i] = nxt[s][i];
    }
}

// Xs[0:r0, tile] += [S | P][0:r0, I] Ys  (I = [r0, r0 + jnb), problem orientation)
template <int NT>
__device__ void update_dmma(const xtgevc3_dpencil &d, bool left, int r0, int jnb, double *Xs, const double *Ys)
{
    constexpr int XLD = Lds<double, NT>::X, YLD = Lds<double, NT>::Y, NJ = NT / 8;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, g = lane >> 2, t = lane & 3;
    const int n = d.n, K = 2 * jnb;
    for (int q = wid; q < (r0 + 31) / 32; q += WARPS) {
        const int rb = 32 * q;
        int rowc[4];
        double acc[4][NJ][2];
#pragma unroll
        for (int i = 0; i < 4; i++) {
            const int row = rb + 8 * i + g;
            rowc[i] = min(row, r0 - 1);
#pragma unroll
            for (int j = 0; j < NJ; j++)
#pragma unroll
                for (int h = 0; h < 2; h++)
                    acc[i][j][h] = row < r0 ? Xs[(size_t)row * XLD + 8 * j + 2 * t + h] : 0.0;
        }
        auto loadA = [&](int k, int i) -> double {
            const bool sp = k < jnb;
            const int kk = sp ? k : k - jnb;
            const double *M = sp ? d.S : d.P;
            const size_t ld = sp ? (size_t)d.lds : (size_t)d.ldp;
            if (!left) return __ldg(M + (size_t)rowc[i] + (size_t)(r0 + kk) * ld);
            return __ldg(M + (size_t)(n - 1 - (r0 + kk)) + (size_t)(n - 1 - rowc[i]) * ld);
        };
        dmma_tile<NT>(loadA, Ys, YLD, K, acc, lane);
#pragma unroll
        for (int i = 0; i < 4; i++) {
            const int row = rb + 8 * i + g;
            if (row < r0)
#pragma unroll
                for (int j = 0; j < NJ; j++)
#pragma unroll
                    for (int h = 0; h < 2; h++) Xs[(size_t)row * XLD + 8 * j + 2 * t + h] = acc[i][j][h];
        }
    }
}

// V[:, out(tile)] = Z[:, 0:khi] Xs[0:khi, tile]  (left: Q with reversed columns)
template <int NT>
__device__ void back_dmma(const xtgevc3_dpencil &d, bool left, int khi, const double *Xs,
                          const TileCols<double, NT> &tc, int ntc)
{
    constexpr int XLD = Lds<double, NT>::X, NJ = NT / 8;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, g = lane >> 2, t = lane & 3;
    const int n = d.n;
    const double *Zb = left ? d.Q : d.Z;
    const size_t ldz = left ? (size_t)d.ldq : (size_t)d.ldz;
    double *V = left ? d.VL : d.VR;
    const size_t ldv = left ? (size_t)d.ldvl : (size_t)d.ldvr;
    for (int q = wid; q < (n + 31) / 32; q += WARPS) {
        const int rb = 32 * q;
        int rowc[4];
        double acc[4][NJ][2];
#pragma unroll
        for (int i = 0; i < 4; i++) {
            rowc[i] = min(rb + 8 * i + g, n - 1);
#pragma unroll
            for (int j = 0; j < NJ; j++) acc[i][j][0] = acc[i][j][1] = 0.0;
        }
        auto loadA = [&](int k, int i) -> double {
            const int zc = left ? n - 1 - k : k;
            return __ldg(Zb + (size_t)rowc[i] + (size_t)zc * ldz);
        };
        dmma_tile<NT>(loadA, Xs, XLD, khi, acc, lane);
#pragma unroll
        for (int i = 0; i < 4; i++) {
            const int row = rb + 8 * i + g;
            if (row < n)
#pragma unroll
                for (int j = 0; j < NJ; j++)
#pragma unroll
                    for (int h = 0; h < 2; h++) {
                        const int c = 8 * j + 2 * t + h;
                        if (c < ntc) V[(size_t)row + (size_t)tc.out[c] * ldv] = acc[i][j][h];
                    }
        }
    }
}

template <class T, int NT, int H>
__device__ void compute_unit(const Args<T> &a, int p, int side, int t, unsigned char *smem, TileCols<T, NT> &tc,
                             uint64_t &s_sec)
{
    constexpr int XLD = Lds<T, NT>::X, YLD = Lds<T, NT>::Y, DLD = H + 1;
    const auto &d = a.pencils[p];
    const int n = d.n;
    const bool left = side == 1;
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    Work<T> w;
    work_layout<T>(a.ws + a.woff[p], n, NT, &w);
    const int maxt = max_tiles(n, NT);
    const int ntiles = __ldcg(w.ntiles + side);
    if (t >= ntiles) return;
    const int c_lo = __ldcg(w.tiles + side * (maxt + 1) + t), c_hi = __ldcg(w.tiles + side * (maxt + 1) + t + 1);
    const int ntc = c_hi - c_lo;

    T *Xs = reinterpret_cast<T *>(smem);
    T *Ys = Xs + (size_t)a.xrows * XLD;
    T *U = Ys + 2 * H * YLD;  // staged A chunks, or the diagonal blocks of S and P
    T *Sd = U, *Pd = U + H * DLD;

    if (tid < NT) {
        const int c = c_lo + tid;
        if (tid < ntc) {
            const uint8_t kd = __ldcg(w.kind + side * n + c);
            tc.kind[tid] = kd;
            tc.colk[tid] = kd == kPairIm ? c - 1 : c;
#pragma unroll
            for (int q = 0; q < 4; q++) tc.coef[tid][q] = __ldcg(w.coef + 4 * ((size_t)side * n + c) + q);
            tc.out[tid] = !left ? c : (kd == kReal ? n - 1 - c : (kd == kPairRe ? n - 2 - c : n - c));
        } else {
            tc.kind[tid] = kPairIm;  // never a solve item
            tc.colk[tid] = -1;
            tc.out[tid] = 0;
        }
    }
    for (int idx = tid; idx < c_hi * NT; idx += THREADS) Xs[(size_t)(idx / NT) * XLD + idx % NT] = T(0);
    __syncthreads();

    const T safemin = limits<T>::safemin, eps = limits<T>::eps;
    const T bignum = T(1) / (safemin / eps);
    const uint8_t *splitf = w.splitf + side * (n + 1);
    for (int cur = c_hi; cur > 0;) {
        const int r1 = cur;
        int r0 = max(0, cur - H);
        if (r0 > 0 && __ldcg(splitf + r0)) r0 += 1;
        const int jnb = r1 - r0;
        // diagonal blocks (problem orientation) and a zeroed update operand
        for (int idx = tid; idx < jnb * jnb; idx += THREADS) {
            int i, j;
            T sv = T(0), pv = T(0);
            if (!left) {
                i = idx % jnb;
                j = idx / jnb;
                if (i <= j + 1) {
                    sv = d.S[(size_t)(r0 + i) + (size_t)(r0 + j) * d.lds];
                    pv = d.P[(size_t)(r0 + i) + (size_t)(r0 + j) * d.ldp];
                }
            } else {
                i = idx / jnb;
                j = idx % jnb;
                if (i <= j + 1) {
                    sv = d.S[(size_t)(n - 1 - (r0 + j)) + (size_t)(n - 1 - (r0 + i)) * d.lds];
                    pv = d.P[(size_t)(n - 1 - (r0 + j)) + (size_t)(n - 1 - (r0 + i)) * d.ldp];
                }
            }
            Sd[i + j * DLD] = sv;
            Pd[i + j * DLD] = pv;
        }
        for (int idx = tid; idx < 2 * jnb * NT; idx += THREADS) Ys[(idx / NT) * YLD + idx % NT] = T(0);
        __syncthreads();
        if (tid == 32) {  // this block's active eigenvectors, real ones and complex pairs
            int nr = 0, np = 0;
            for (int j = 0; j < ntc; j++) {
                if (tc.kind[j] == kPairIm || tc.colk[j] < r0) continue;
                if (tc.kind[j] == kReal) tc.lreal[nr++] = j;
                else tc.lpair[np++] = j;
            }
            tc.nreal = nr;
            tc.npair = np;
        }
        if (tid < 32) {  // 2x2 diagonal blocks, paired greedily from the bottom
            const bool b0 = lane >= 1 && lane < jnb && Sd[lane + (lane - 1) * DLD] != T(0);
            const bool b1 = lane + 32 < jnb && Sd[(lane + 32) + (lane + 31) * DLD] != T(0);
            const uint64_t sub =
                (uint64_t)__ballot_sync(0xffffffffu, b0) | ((uint64_t)__ballot_sync(0xffffffffu, b1) << 32);
            if (lane == 0) {
                uint64_t sec = 0;
                for (int j = jnb - 1; j >= 1;) {
                    if ((sub >> j) & 1ull) {
                        sec |= 1ull << j;
                        j -= 2;
                    } else {
                        j -= 1;
                    }
                }
                s_sec = sec;
            }
        }
        __syncthreads();
        const uint64_t sec = s_sec;
        if constexpr (std::is_same<T, double>::value) {
            // FP64: several eigenvectors per warp (measured faster); FP32 keeps one per warp,
            // which keeps its register count low enough for two CTAs per SM
            solve_group<T, NT, H, false>(tc, tc.lreal, tc.nreal, r0, r1, Sd, Pd, sec, Xs, Ys, left,
                                         bignum / T(10), bignum / T(max(1, jnb)));
            solve_group<T, NT, H, true>(tc, tc.lpair, tc.npair, r0, r1, Sd, Pd, sec, Xs, Ys, left,
                                        bignum / T(10), bignum / T(max(1, jnb)));
        } else {
            for (int j = wid; j < ntc; j += WARPS) {
                if (tc.kind[j] == kPairIm || tc.colk[j] < r0) continue;
                solve_item<T, NT, H>(tc, j, r0, r1, Sd, Pd, sec, Xs, Ys, left, bignum / T(10),
                                     bignum / T(max(1, jnb)), lane);
            }
        }
        __syncthreads();
        if constexpr (std::is_same<T, double>::value) {
            if (r0 > 0) update_dmma<NT>(d, left, r0, jnb, Xs, Ys);
        } else {
            for (int p0 = 0; p0 < r0; p0 += PASS) {
                const int rows = min(PASS, r0 - p0);
                switch ((rows + 63) / 64) {
                case 1: update_pass<T, NT, H, 1>(d, left, r0, jnb, p0, rows, Xs, Ys, U); break;
                case 2: update_pass<T, NT, H, 2>(d, left, r0, jnb, p0, rows, Xs, Ys, U); break;
                case 3: update_pass<T, NT, H, 3>(d, left, r0, jnb, p0, rows, Xs, Ys, U); break;
                default: update_pass<T, NT, H, 4>(d, left, r0, jnb, p0, rows, Xs, Ys, U); break;
                }
            }
        }
        __syncthreads();
        cur = r0;
    }

    if (a.back && std::is_same<T, double>::value) {
        if constexpr (std::is_same<T, double>::value) back_dmma<NT>(d, left, c_hi, Xs, tc, ntc);
    } else if (a.back) {
        for (int p0 = 0; p0 < n; p0 += PASS) {
            const int rows = min(PASS, n - p0);
            switch ((rows + 63) / 64) {
            case 1: back_pass<T, NT, H, 1>(d, left, c_hi, p0, rows, Xs, U, tc, ntc); break;
            case 2: back_pass<T, NT, H, 2>(d, left, c_hi, p0, rows, Xs, U, tc, ntc); break;
            case 3: back_pass<T, NT, H, 3>(d, left, c_hi, p0, rows, Xs, U, tc, ntc); break;
            default: back_pass<T, NT, H, 4>(d, left, c_hi, p0, rows, Xs, U, tc, ntc); break;
            }
        }
    } else {
        T *V = left ? d.VL : d.VR;
        const size_t ldv = left ? (size_t)d.ldvl : (size_t)d.ldvr;
        for (int idx = tid; idx < n * ntc; idx += THREADS) {
            const int i = idx % n, j = idx / n;
            const int src = left ? n - 1 - i : i;
            V[(size_t)i + (size_t)tc.out[j] * ldv] = src < c_hi ? Xs[(size_t)src * XLD + j] : T(0);
        }
    }
}

// ---- the persistent kernel ---------------------------------------------------------------
// FP32 with 16-column tiles is held to the 128 registers that fit two CTAs per SM (its
// shared memory allows two; the rarely taken capped re-solve would otherwise set the count).
template <class T, int NT, int H>
__global__ void __launch_bounds__(THREADS, (std::is_same<T, float>::value && NT == 16) ? 2 : 1)
    batch_kernel(Args<T> a)
{
    extern __shared__ __align__(16) unsigned char smem_batch[];
    __shared__ TileCols<T, NT> tc;
    __shared__ uint64_t s_sec;
    __shared__ int s_unit, s_ok;
    for (;;) {
        if (threadIdx.x == 0) s_unit = atomicAdd(a.ctrl, 1);
        __syncthreads();
        const int u = s_unit;
        if (u >= a.nunits) break;
        const int4 wu = a.units[u];
        if (wu.x == 0) {
            prep_unit<T, NT>(a, wu.y, smem_batch);
        } else {
            if (threadIdx.x == 0) {
                int ok = 1;
                const volatile int *flag = a.ctrl + 2 + wu.y;
                long long it = 0;
                while (*flag == 0) {
                    if (++it > a.spin_limit) {
                        atomicOr(a.ctrl + 1, kErrWaitTimeout);
                        ok = 0;
                        break;
                    }
                    __nanosleep(128);
                }
                __threadfence();
                s_ok = ok;
            }
            __syncthreads();
            if (s_ok) compute_unit<T, NT, H>(a, wu.y, wu.z, wu.w, smem_batch, tc, s_sec);
        }
        __syncthreads();
    }
}

}  // namespace batch
}  // namespace xtg
