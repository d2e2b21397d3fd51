// GEMM kernels of the substitution: the trailing update of the accumulated right-hand
// sides and the back-transform by Z (or Q).
//
//   C[mlo:M, j] (+)= sum_kk A(m, kk) * B(kk, j)
//
// A is column-major and stacked from up to four segments along K (each a strip of S or P
// or of Z), which lets one launch apply every half of an update
//   X[0:r0, c] += S[0:r0, I] * (-ac x) + P[0:r0, I] * (b x)
// (upstream: the two dgemm_ calls at src/dtgevc3.cpp:1432-1433), also for two row blocks
// at once (K = 4 strips).  Segment s covers K rows [kb_s, kb_s + K_s) (K_s a multiple of
// 16), reads A_s columns [0, acols_s) (beyond them: zero) and B rows boff_s + (kk - kb_s).
// Rows [0, mlo) of the row window are computed but neither read nor written in C (they
// let a window start on an even row).  For the back-transform (src/dtgevc3.cpp:1446, 1638)
// A is Z (or Q with reversed columns), B is the upper triangular X, and `kext` gives per
// column the number of leading rows of B that can be nonzero so that a column tile only
// runs K up to its last nonzero row.  The optional column map scatters result columns
// into their output positions.
#pragma once
#include "common.cuh"

namespace xtg {

template <class E>
struct GemmSeg {
    const E *A;  // row 0 of the window, first column of the strip
    int lda, acols, K, boff;
};

template <class E>
struct GemmArgs {
    int M, N, K, mlo;
    int nseg;
    GemmSeg<E> seg[4];
    const E *B;
    int ldb, brows;      // rows of B that exist in memory
    E *C;
    int ldc;
    const int *ccol;     // output column of result column j (nullptr: j)
    const int *kext;     // nonzero leading rows of B per column (nullptr: K)
    int accumulate;
    // residue form only: B and its shape are those of the previous launch on the same
    // buffers (row panels of one back-transform), so its residues are reused
    int reuse_b = 0;
};

// Segment holding K row kk (segments are contiguous and cover [0, K)); kb = its first row.
template <class E>
__device__ __forceinline__ int find_seg(const GemmArgs<E> &g, int kk, int &kb)
{
    int base = 0;
#pragma unroll
    for (int s = 0; s < 4; s++) {
        if (s < g.nseg && kk < base + g.seg[s].K) {
            kb = base;
            return s;
        }
        if (s < g.nseg) base += g.seg[s].K;
    }
    kb = base;
    return -1;
}

template <class E>
__device__ __forceinline__ int tile_kmax(const GemmArgs<E> &g, int n0, int BN)
{
    int kmax = g.K;
    if (g.kext) {
        int last = min(n0 + BN, g.N) - 1;
        kmax = min(kmax, g.kext[last]);
    }
    return kmax;
}

// ------------------------------------------------------------------------------------
// SIMT kernel (any element type): 64 x 64 tile, 256 threads, 4 x 4 outputs per thread.
// ------------------------------------------------------------------------------------
template <class E>
__global__ void __launch_bounds__(256) gemm_simt(GemmArgs<E> g)
{
    constexpr int BM = 64, BN = 64, BK = 16;
    __shared__ E As[BK][BM + 1];
    __shared__ E Bs[BK][BN + 1];
    const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
    // with a per-column K extent (back-transform: triangular B, extent growing with the
    // column) the column tiles run last-first, so the longest tiles start first
    const int m0 = blockIdx.x * BM, n0 = (g.kext ? gridDim.y - 1 - blockIdx.y : blockIdx.y) * BN;
    const int kmax = tile_kmax(g, n0, BN);
    E acc[4][4];
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) acc[i][j] = E(0);

    for (int k0 = 0; k0 < kmax; k0 += BK) {
        int kb = 0;
        const int s = find_seg(g, k0, kb);
        const GemmSeg<E> sg = g.seg[s < 0 ? 0 : s];
#pragma unroll
        for (int q = 0; q < 4; q++) {
            int e = tid + 256 * q;
            int m = e % BM, kk = e / BM;
            int col = k0 - kb + kk, row = m0 + m;
            As[kk][m] = (s >= 0 && k0 + kk < kmax && col < sg.acols && row < g.M)
                            ? sg.A[(size_t)row + (size_t)col * sg.lda]
                            : E(0);
        }
#pragma unroll
        for (int q = 0; q < 4; q++) {
            int e = tid + 256 * q;
            int kk = e % BK, n = e / BK;
            int kr = sg.boff + k0 - kb + kk, col = n0 + n;
            Bs[kk][n] = (s >= 0 && k0 + kk < kmax && kr < g.brows && col < g.N) ? g.B[(size_t)kr + (size_t)col * g.ldb]
                                                                              : E(0);
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < BK; kk++) {
            E a[4], b[4];
#pragma unroll
            for (int i = 0; i < 4; i++) a[i] = As[kk][tx + 16 * i];
#pragma unroll
            for (int j = 0; j < 4; j++) b[j] = Bs[kk][ty + 16 * j];
#pragma unroll
            for (int i = 0; i < 4; i++)
#pragma unroll
                for (int j = 0; j < 4; j++) acc[i][j] = acc[i][j] + a[i] * b[j];
        }
        __syncthreads();
    }
#pragma unroll
    for (int j = 0; j < 4; j++) {
        int col = n0 + ty + 16 * j;
        if (col >= g.N) continue;
        int oc = g.ccol ? g.ccol[col] : col;
        E *cp = g.C + (size_t)oc * g.ldc;
#pragma unroll
        for (int i = 0; i < 4; i++) {
            int row = m0 + tx + 16 * i;
            if (row >= g.mlo && row < g.M) cp[row] = g.accumulate ? cp[row] + acc[i][j] : acc[i][j];
        }
    }
}

// ------------------------------------------------------------------------------------
// FP64 tensor-core kernel (DMMA, mma.sync m8n8k4 f64).
// CTA tile BM x 64 (BM = 128, or 64 for launches of at most 64 output rows, such as the
// update of a group's upper block), K step 16, BM/32 x 2 warps with 32 x 32 warp tiles,
// 3-stage cp.async pipeline into padded shared memory (conflict-free fragment loads).
// Requires 16-byte aligned segment bases and B, and even leading dimensions (checked by
// the launcher, which uses the SIMT kernel otherwise); B rows at an odd offset (a block
// boundary moved by a 2x2 block) take the BODD loader.
// ------------------------------------------------------------------------------------
namespace dmma {
constexpr int BN = 64, BK = 16, STAGES = 3;  // BK divides kKPad (segment K)
constexpr int BLD = BK + 4;                  // B tile stored [n][k]
constexpr int B_STAGE = BN * BLD;
template <int BM>
struct Tile {
    static constexpr int NT = 2 * BM;         // threads: BM/32 x 2 warps
    static constexpr int ALD = BM + 8;        // A tile stored [k][m]
    static constexpr int A_STAGE = BK * ALD;
    static constexpr int SMEM_BYTES = STAGES * (A_STAGE + B_STAGE) * 8;
};
}  // namespace dmma

__device__ __forceinline__ void cp_async16(void *smem, const void *gmem, int src_bytes)
{
    unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(src_bytes));
}
// 8 bytes (8-byte aligned addresses; the 16-byte form needs 16-byte alignment)
__device__ __forceinline__ void cp_async8(void *smem, const void *gmem, int src_bytes)
{
    unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(s), "l"(gmem), "r"(src_bytes));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

__device__ __forceinline__ void dmma884(double &d0, double &d1, double a, double b)
{
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                 : "+d"(d0), "+d"(d1)
                 : "d"(a), "d"(b));
}

// ACC = 1: trailing update (C += A B); ACC = 0: back-transform (C = A B, triangular B).
// BODD: some segment's B rows start at an odd offset (boff), so its row pairs are only
// 8-byte aligned and load as two 8-byte copies.
template <int ACC, int BM = 128, bool BODD = false>
__global__ void __launch_bounds__(2 * BM) gemm_dmma(GemmArgs<double> g)
{
    using namespace dmma;
    constexpr int NT = Tile<BM>::NT, ALD = Tile<BM>::ALD, A_STAGE = Tile<BM>::A_STAGE;
    constexpr int WM = BM / 32;  // warps along M
    static_assert((BK * BM) % (2 * NT) == 0 && (BN * BK) % (2 * NT) == 0, "loader chunks per thread");
    extern __shared__ __align__(16) unsigned char smem_gemm[];
    double *As = reinterpret_cast<double *>(smem_gemm);
    double *Bs = As + STAGES * A_STAGE;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int wm = warp % WM, wn = warp / WM;
    const int gq = lane >> 2, tq = lane & 3;
    // with a per-column K extent (back-transform: triangular B, extent growing with the
    // column) the column tiles run last-first, so the longest tiles start first
    const int m0 = blockIdx.x * BM, n0 = (g.kext ? gridDim.y - 1 - blockIdx.y : blockIdx.y) * BN;
    const int kmax = tile_kmax(g, n0, BN);
    const int ktiles = (kmax + BK - 1) / BK;

    double acc[4][4][2];
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) {
            acc[i][j][0] = 0.0;
            acc[i][j][1] = 0.0;
        }

    auto load_stage = [&](int kt, int st) {
        const int k0 = kt * BK;
        int kb = 0;
        const int s = find_seg(g, k0, kb);
        const GemmSeg<double> sg = g.seg[s < 0 ? 0 : s];
        double *as = As + st * A_STAGE;
        double *bs = Bs + st * B_STAGE;
#pragma unroll
        for (int q = 0; q < BK * BM / (2 * NT); q++) {  // A: BK columns x BM/2 chunks of 16 bytes
            int e = tid + NT * q;
            int kk = e / (BM / 2), ch = e % (BM / 2);
            int row = m0 + 2 * ch, col = k0 - kb + kk;
            int bytes = 0;
            if (s >= 0 && k0 + kk < kmax && col < sg.acols) bytes = row + 1 < g.M ? 16 : (row < g.M ? 8 : 0);
            const double *gp = bytes ? sg.A + (size_t)row + (size_t)col * sg.lda : g.B;
            cp_async16(as + kk * ALD + 2 * ch, gp, bytes);
        }
#pragma unroll
        for (int q = 0; q < BN * BK / (2 * NT); q++) {  // B: BN columns x BK/2 chunks
            int e = tid + NT * q;
            int nn = e / (BK / 2), ch = e % (BK / 2);
            int kr = sg.boff + k0 - kb + 2 * ch, col = n0 + nn;
            int lim = min(sg.boff + kmax - kb, g.brows);
            int bytes = 0;
            if (s >= 0 && col < g.N) bytes = kr + 1 < lim ? 16 : (kr < lim ? 8 : 0);
            const double *gp = bytes ? g.B + (size_t)kr + (size_t)col * g.ldb : g.B;
            if constexpr (BODD) {
                cp_async8(bs + nn * BLD + 2 * ch, gp, bytes ? 8 : 0);
                cp_async8(bs + nn * BLD + 2 * ch + 1, bytes == 16 ? gp + 1 : g.B, bytes == 16 ? 8 : 0);
            } else {
                cp_async16(bs + nn * BLD + 2 * ch, gp, bytes);
            }
        }
    };

#pragma unroll
    for (int s = 0; s < STAGES - 1; s++) {
        if (s < ktiles) load_stage(s, s);
        cp_async_commit();
    }
    // Accumulating launches start from C: its loads are issued here, behind the first
    // pipeline stages, so their latency overlaps the prologue instead of the epilogue.
    if (ACC) {
#pragma unroll
        for (int j = 0; j < 4; j++) {
#pragma unroll
            for (int h = 0; h < 2; h++) {
                const int col = n0 + wn * 32 + j * 8 + 2 * tq + h;
                if (col >= g.N) continue;
                const double *cp = g.C + (size_t)(g.ccol ? g.ccol[col] : col) * g.ldc;
#pragma unroll
                for (int i = 0; i < 4; i++) {
                    const int row = m0 + wm * 32 + i * 8 + gq;
                    if (row >= g.mlo && row < g.M) acc[i][j][h] = cp[row];
                }
            }
        }
    }
    for (int kt = 0; kt < ktiles; kt++) {
        cp_async_wait<STAGES - 2>();
        __syncthreads();
        int nk = kt + STAGES - 1;
        if (nk < ktiles) load_stage(nk, nk % STAGES);
        cp_async_commit();
        const double *as = As + (kt % STAGES) * A_STAGE;
        const double *bs = Bs + (kt % STAGES) * B_STAGE;
#pragma unroll
        for (int kk = 0; kk < BK; kk += 4) {
            double a[4], b[4];
#pragma unroll
            for (int i = 0; i < 4; i++) a[i] = as[(kk + tq) * ALD + wm * 32 + i * 8 + gq];
#pragma unroll
            for (int j = 0; j < 4; j++) b[j] = bs[(wn * 32 + j * 8 + gq) * BLD + kk + tq];
#pragma unroll
            for (int i = 0; i < 4; i++)
#pragma unroll
                for (int j = 0; j < 4; j++) dmma884(acc[i][j][0], acc[i][j][1], a[i], b[j]);
        }
    }
    cp_async_wait<0>();

    // epilogue: fragment (row gq, cols 2tq, 2tq+1) of each 8x8 tile
#pragma unroll
    for (int j = 0; j < 4; j++) {
#pragma unroll
        for (int h = 0; h < 2; h++) {
            int col = n0 + wn * 32 + j * 8 + 2 * tq + h;
            if (col >= g.N) continue;
            int oc = g.ccol ? g.ccol[col] : col;
            double *cp = g.C + (size_t)oc * g.ldc;
#pragma unroll
            for (int i = 0; i < 4; i++) {
                int row = m0 + wm * 32 + i * 8 + gq;
                if (row >= g.mlo && row < g.M) cp[row] = acc[i][j][h];
            }
        }
    }
}

// ------------------------------------------------------------------------------------
// Complex FP64 on the DMMA path (z): every complex product is four real m8n8k4 MMAs,
//   Cr += Ar Br - Ai Bi,   Ci += Ar Bi + Ai Br.
// CTA tile 64 x 64 complex, K step 8, 8 warps as 2 (M) x 4 (N) with 32 x 16 warp tiles,
// 3-stage cp.async pipeline of 16-byte complex elements (shared memory keeps the
// interleaved layout; fragments pick the real or imaginary half).  Segment, K-limit and
// column-map conventions as gemm_simt.  Needs 16-byte aligned operands (the launcher checks).
// ------------------------------------------------------------------------------------
namespace zmma {
constexpr int BM = 64, BN = 64, BK = 8, STAGES = 3;
constexpr int ALD = BM + 4;  // A tile [k][m], complex
constexpr int BLD = BK + 1;  // B tile [n][k], complex
constexpr int A_STAGE = BK * ALD;
constexpr int B_STAGE = BN * BLD;
constexpr int SMEM_BYTES = STAGES * (A_STAGE + B_STAGE) * 16;
}  // namespace zmma

template <int ACC>
__global__ void __launch_bounds__(256) gemm_dmma_cplx(GemmArgs<cplx<double>> g)
{
    using namespace zmma;
    using Z = cplx<double>;
    extern __shared__ __align__(16) unsigned char smem_gemm_z[];
    Z *As = reinterpret_cast<Z *>(smem_gemm_z);
    Z *Bs = As + STAGES * A_STAGE;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int wm = warp & 1, wn = warp >> 1;
    const int gq = lane >> 2, tq = lane & 3;
    // with a per-column K extent (back-transform: triangular B, extent growing with the
    // column) the column tiles run last-first, so the longest tiles start first
    const int m0 = blockIdx.x * BM, n0 = (g.kext ? gridDim.y - 1 - blockIdx.y : blockIdx.y) * BN;
    const int kmax = tile_kmax(g, n0, BN);
    const int ktiles = (kmax + BK - 1) / BK;

    double cr[4][2][2], ci[4][2][2];
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 2; j++)
#pragma unroll
            for (int h = 0; h < 2; h++) cr[i][j][h] = ci[i][j][h] = 0.0;

    auto load_stage = [&](int kt, int st) {
        const int k0 = kt * BK;
        int kb = 0;
        const int s = find_seg(g, k0, kb);
        const GemmSeg<Z> sg = g.seg[s < 0 ? 0 : s];
        Z *as = As + st * A_STAGE;
        Z *bs = Bs + st * B_STAGE;
#pragma unroll
        for (int q = 0; q < 2; q++) {  // A: 8 columns x 64 rows
            const int e = tid + 256 * q;
            const int kk = e >> 6, m = e & 63;
            const int row = m0 + m, col = k0 - kb + kk;
            const bool ok = s >= 0 && k0 + kk < kmax && col < sg.acols && row < g.M;
            const Z *gp = ok ? sg.A + (size_t)row + (size_t)col * sg.lda : reinterpret_cast<const Z *>(g.B);
            cp_async16(as + kk * ALD + m, gp, ok ? 16 : 0);
        }
        const int lim = min(sg.boff + kmax - kb, g.brows);
#pragma unroll
        for (int q = 0; q < 2; q++) {  // B: 64 columns x 8 rows
            const int e = tid + 256 * q;
            const int kk = e & 7, nn = e >> 3;
            const int kr = sg.boff + k0 - kb + kk, col = n0 + nn;
            const bool ok = s >= 0 && col < g.N && kr < lim;
            const Z *gp = ok ? g.B + (size_t)kr + (size_t)col * g.ldb : g.B;
            cp_async16(bs + nn * BLD + kk, gp, ok ? 16 : 0);
        }
    };

#pragma unroll
    for (int s = 0; s < STAGES - 1; s++) {
        if (s < ktiles) load_stage(s, s);
        cp_async_commit();
    }
    if (ACC) {
#pragma unroll
        for (int j = 0; j < 2; j++)
#pragma unroll
            for (int h = 0; h < 2; h++) {
                const int col = n0 + wn * 16 + j * 8 + 2 * tq + h;
                if (col >= g.N) continue;
                const Z *cp = g.C + (size_t)(g.ccol ? g.ccol[col] : col) * g.ldc;
#pragma unroll
                for (int i = 0; i < 4; i++) {
                    const int row = m0 + wm * 32 + i * 8 + gq;
                    if (row >= g.mlo && row < g.M) {
                        const Z v = cp[row];
                        cr[i][j][h] = v.x;
                        ci[i][j][h] = v.y;
                    }
                }
            }
    }
    for (int kt = 0; kt < ktiles; kt++) {
        cp_async_wait<STAGES - 2>();
        __syncthreads();
        const int nk = kt + STAGES - 1;
        if (nk < ktiles) load_stage(nk, nk % STAGES);
        cp_async_commit();
        const Z *as = As + (kt % STAGES) * A_STAGE;
        const Z *bs = Bs + (kt % STAGES) * B_STAGE;
#pragma unroll
        for (int kk = 0; kk < BK; kk += 4) {
            double ar[4], ai[4], br[2], bi[2], nbi[2];
#pragma unroll
            for (int i = 0; i < 4; i++) {
                const Z a = as[(kk + tq) * ALD + wm * 32 + i * 8 + gq];
                ar[i] = a.x;
                ai[i] = a.y;
            }
#pragma unroll
            for (int j = 0; j < 2; j++) {
                const Z b = bs[(wn * 16 + j * 8 + gq) * BLD + kk + tq];
                br[j] = b.x;
                bi[j] = b.y;
                nbi[j] = -b.y;
            }
#pragma unroll
            for (int i = 0; i < 4; i++)
#pragma unroll
                for (int j = 0; j < 2; j++) {
                    dmma884(cr[i][j][0], cr[i][j][1], ar[i], br[j]);
                    dmma884(cr[i][j][0], cr[i][j][1], ai[i], nbi[j]);
                    dmma884(ci[i][j][0], ci[i][j][1], ar[i], bi[j]);
                    dmma884(ci[i][j][0], ci[i][j][1], ai[i], br[j]);
                }
        }
    }
    cp_async_wait<0>();
#pragma unroll
    for (int j = 0; j < 2; j++)
#pragma unroll
        for (int h = 0; h < 2; h++) {
            const int col = n0 + wn * 16 + j * 8 + 2 * tq + h;
            if (col >= g.N) continue;
            Z *cp = g.C + (size_t)(g.ccol ? g.ccol[col] : col) * g.ldc;
#pragma unroll
            for (int i = 0; i < 4; i++) {
                const int row = m0 + wm * 32 + i * 8 + gq;
                if (row >= g.mlo && row < g.M) cp[row] = Z(cr[i][j][h], ci[i][j][h]);
            }
        }
}

}  // namespace xtg
