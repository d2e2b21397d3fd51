// Split-precision FP64 GEMM by residues (Chinese remainder theorem) on the INT8 tensor
// cores (tcgen05 kind::i8).
//
//   C[mlo:M, j] (+)= sum_k A(m, k) B(k, j)        A, B, C in FP64
//
// Integers.  Row m of A is scaled by a power of two and rounded to an integer of at most
// t bits, A'(m, k) = rint(A(m, k) 2^(t - ea_m)) with |A'| <= 2^t (ea_m: the exponent of the
// row's largest entry); columns of B likewise (eb_j).  Then A B = 2^(ea + eb - 2t) A' B' up to
// the rounding of the operands (2^-t relative to the row's / column's largest entry).
//
// Residues.  With L pairwise-coprime moduli p_l <= 256 (product P), the integer product
// C' = A' B' is recovered from its residues: c_l = (A' mod p_l)(B' mod p_l) is one INT8 GEMM
// per modulus (residues in [-128, 127], exact INT32 sums), and
//   C' = sum_l r_l W_l - k P,   r_l = c_l mod p_l,   W_l = M_l (M_l^-1 mod p_l) mod P,  M_l = P / p_l,
// with k = round(sum / P), exact when |C'| < P / 4, i.e. 2t + log2(K) + 2 <= log2(P): t is
// chosen from L and K on the host.  The number of tensor-core products is L (14 for ~47-bit
// operands), against s(s+1)/2 = 28 digit products of 7-bit slices for 49 bits.
//
// Kernels (one GEMM = six launches):
//   row_absmax_kernel / col_absmax_kernel, residue_rows_kernel / residue_cols_kernel: the
//       exponents ea / eb, then A' and B' residues stored K-major as out[l][row][k] (INT8,
//       row pitch Kp);
//   gemm_crt_kernel: persistent; work item (l, column tile, row tile), modulus outermost
//       so that one modulus' operands stay in L2; tile 256 rows x 128 columns of C, computed
//       transposed (MMA M = the tile's columns, N = its rows), one CTA per SM.
//       warp 0: TMA producer (64-byte K rows, 64-byte swizzle, STAGES-deep ring, no
//               multicast); warp 1: TMEM allocation and MMA issue (one thread; two
//               128 x 256 x 32 MMAs per stage into one of two TMEM accumulators of 256
//               columns, so a tile's epilogue overlaps the next tile's MMAs); warps 2-9:
//               epilogue, one TMEM lane (a column of C) per thread, 128 rows per warp in
//               chunks of 32: r_l = c_l mod p_l (integer Barrett reduction) stored as 32
//               contiguous bytes of U[l][col][row];
//   crt_kernel: per element, the exact sums H = sum r_l W1_l, Mid = sum r_l W2_l (W_l ~
//       W1_l 2^hi + W2_l 2^lo, each product and partial sum an exact FP64 integer), k, and
//       C' = (H - k P1) 2^hi + (Mid - k P2) 2^lo, scaled by 2^(ea + eb - 2t) into C.
// Every mbarrier wait is bounded (abort flag, global error word, in-flight copies and MMAs
// drained, TMEM released).
#pragma once
#include "kernels_split.cuh"

namespace xtg {
namespace crt {

// Tile: TM = 256 rows x TN = 128 columns of C, computed as its transpose on the tensor core:
// the MMA's M dimension (128, one TMEM lane each) runs over C's columns (B residues) and its
// N dimension (256) over C's rows (A residues), so that an epilogue thread (one TMEM lane =
// one column of C) holds 32 consecutive rows per TMEM load and stores them as 32
// contiguous bytes of U[l][col][row].
constexpr int TM = 256;        // rows of C per tile  (MMA N)
constexpr int TN = 128;        // columns of C per tile (MMA M, TMEM lanes)
constexpr int BK = 64;         // K bytes per stage (one 64-byte swizzle row)
constexpr int STAGES = 8;
constexpr int THREADS = 320;   // warp 0 TMA, warp 1 MMA, warps 2-9 epilogue
constexpr int EPI_WARPS = 8;
constexpr int MAXL = 16;
constexpr int ROW_TILE = TM * BK;               // 16 KB of A residues per stage
constexpr int COL_TILE = TN * BK;               // 8 KB of B residues per stage
constexpr int SMEM_BYTES = STAGES * (ROW_TILE + COL_TILE) + 1024;
// S8 x S8 -> S32, K-major operands, MMA M = 128, N = 256
constexpr uint32_t IDESC = (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(TM >> 3) << 17) |
                           ((uint32_t)(TN >> 4) << 24);
// Moduli and reconstruction constants of one modulus count L (built on the host).
//   C' = sum_l r_l W_l - k P,  r_l = c_l mod p_l,  W_l = (P / p_l) ((P / p_l)^-1 mod p_l) mod P,
// the CRT weights with the inverse folded in (so the epilogue only reduces c_l mod p_l).
struct Moduli {
    int L;
    int p[MAXL];              // moduli, largest first
    unsigned int barrett[MAXL];  // floor(2^32 / p_l)
    double invp[MAXL];
    double pd[MAXL];          // p_l as a double
    // W_l ~ w1_l 2^hi + w2_l 2^lo with w1_l, w2_l < 2^41 (bits below 2^lo dropped), so that
    // every r_l w_l (r_l < 256) and every partial sum of L <= 16 of them is an exact FP64 integer
    double w1[MAXL], w2[MAXL];
    double P1, P2;            // the same split of P
    double c1, c2;            // 2^hi / P, 2^lo / P
    int hi, lo;
    double log2P;
};

struct Params {
    int M, N, Kp;        // Kp: padded K (multiple of BK)
    int Mp, Np;          // rows of each modulus' A residues (multiple of TM) / columns of B's (of TN)
    int L, mtiles, ntiles, items;
    const int *kext;     // per output column: K extent (nullptr: Kp)
    unsigned char *U;    // r_l, [l][col][row], pitch Mp, Np columns per modulus
    int *err;            // global error word (kErrWaitTimeout on a bounded-wait expiry)
    int p[MAXL];
    unsigned int barrett[MAXL];
};

// ---- operand residues -------------------------------------------------------------------
// v in (-1, 1): a = rint(v 2^t) (exact integer, |a| <= 2^t < 2^51), residue a mod p_l in
// [-128, 127] (symmetric; 128 mod 256 stored as -128).  All rounding goes through the FP64
// adder against R = 1.5 2^52 (where the spacing of doubles is 1 and the low word of x + R is
// the two's complement of the integer x), so no conversion-unit instruction is needed:
//   aR = fma(v, 2^t, R) = a + R  (rint, ties to even: R is even), a = aR - R,
//   qR = fma(a, 1/p, R) = q + R  (q the integer nearest a / p, |a / p| < 2^43),
//   fma(-q, p, aR) = a - q p + R (exact), whose low word is r = a - q p, |r| <= p/2 + 1.
constexpr double kRoundMagic = 6755399441055744.0;  // R = 1.5 * 2^52
// With q the integer nearest a fl(1/p) (|a| <= 2^50: within 2^-3 / p of a / p), |r| <= p / 2,
// so for odd p the low byte of r is a residue in [-127, 127], for p = 256 one in [-128, 128]
// (128 and -128 share the byte 0x80): the byte is taken as it is.
__device__ __forceinline__ uint32_t residue_word(double a, double aR, double invp, double pd)
{
    const double q = __dsub_rn(fma(a, invp, kRoundMagic), kRoundMagic);
    return (uint32_t)__double2loint(fma(-q, pd, aR));
}

// The low bytes of four words, packed (w0 in byte 0).
__device__ __forceinline__ uint32_t pack4(uint32_t w0, uint32_t w1, uint32_t w2, uint32_t w3)
{
    return __byte_perm(__byte_perm(w0, w1, 0x0040), __byte_perm(w2, w3, 0x0040), 0x5410);
}

// Residues of eight entries (a, a + R) for every modulus, 8 bytes per modulus at o + l stride.
// NLC > 0: the modulus count as a compile-time constant (the moduli read at fixed offsets).
template <int NLC>
__device__ __forceinline__ void store_residues8(const double (&a)[8], const double (&aR)[8], const Moduli &md,
                                                int8_t *o, size_t stride)
{
    auto one = [&](int l) {
        const double invp = md.invp[l], pd = md.pd[l];
        uint32_t w[8];
#pragma unroll
        for (int q = 0; q < 8; q++) w[q] = residue_word(a[q], aR[q], invp, pd);
        *reinterpret_cast<uint2 *>(o + (size_t)l * stride) =
            make_uint2(pack4(w[0], w[1], w[2], w[3]), pack4(w[4], w[5], w[6], w[7]));
    };
    if constexpr (NLC > 0) {
#pragma unroll
        for (int l = 0; l < NLC; l++) one(l);
    } else {
#pragma unroll 1
        for (int l = 0; l < md.L; l++) one(l);
    }
}

// a = rint(v 2^s) and a + R: one fma with the power of two when 2^s is a normal double,
// else ldexp and rint.
__device__ __forceinline__ void scaled_int(double v, int s, double &a, double &aR)
{
    if (s > -1000 && s < 1000) {
        aR = fma(v, __longlong_as_double((long long)(s + 1023) << 52), kRoundMagic);
        a = __dsub_rn(aR, kRoundMagic);
    } else {
        a = rint(ldexp(v, s));
        aR = __dadd_rn(a, kRoundMagic);
    }
}

// Largest |A(m, k)| of each row (through the segment description of a GEMM launch), as the
// bit pattern of a non-negative double (ordered like the values), max-reduced into
// rmax[row] (zeroed by the caller).  Grid: (Mp / 32, K chunks of 256); 256 threads, rows
// along lanes (coalesced column-major reads).
__global__ void __launch_bounds__(256) row_absmax_kernel(GemmArgs<double> g, unsigned long long *rmax)
{
    __shared__ double part[8][32];
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    const int row = blockIdx.x * 32 + tx;
    const int k0 = blockIdx.y * 256, k1 = min(g.K, k0 + 256);
    double mx = 0.0;
    for (int k = k0 + ty; k < k1; k += 8) {
        int kb = 0;
        const int sg = find_seg(g, k, kb);
        const int col = k - kb;
        if (sg >= 0 && row < g.M && col < g.seg[sg].acols)
            mx = fmax(mx, fabs(g.seg[sg].A[(size_t)row + (size_t)col * g.seg[sg].lda]));
    }
    part[ty][tx] = mx;
    __syncthreads();
    if (ty == 0) {
        for (int q = 1; q < 8; q++) mx = fmax(mx, part[q][tx]);
        if (mx > 0.0) atomicMax(&rmax[blockIdx.x * 32 + tx], (unsigned long long)__double_as_longlong(mx));
    }
}

// Rows of A -> residues out[l][row][k] (row pitch Kp, l-th block of Mp rows), ea[row].
// Grid: (Mp / 32, Kp / 64): one CTA per 32 rows x 64 K; thread t takes row t / 8 and the 8
// consecutive K from 8 (t % 8) (K segments are multiples of 16 long: one segment), loaded
// straight from A (a warp's load covers 4 consecutive rows of 8 columns: whole 32-byte
// sectors), and stores 8 bytes per modulus.
template <int NLC>
__global__ void __launch_bounds__(256) residue_rows_kernel(GemmArgs<double> g, int Kp, int Mp, int t, Moduli md,
                                                           const unsigned long long *rmax, int8_t *out, int *ea)
{
    const int row = blockIdx.x * 32 + (threadIdx.x >> 3);
    const int k0 = blockIdx.y * 64 + (threadIdx.x & 7) * 8;
    double v[8];
#pragma unroll
    for (int q = 0; q < 8; q++) v[q] = 0.0;
    if (row < g.M && k0 < g.K) {
        int kb = 0;
        const int sg = find_seg(g, k0, kb);
        if (sg >= 0) {
            const int col = k0 - kb, acols = g.seg[sg].acols;
            const double *A = g.seg[sg].A + row + (size_t)col * g.seg[sg].lda;
#pragma unroll
            for (int q = 0; q < 8; q++)
                if (col + q < acols) v[q] = A[(size_t)q * g.seg[sg].lda];
        }
    }
    const int e = split::scale_exp(__longlong_as_double((long long)rmax[row]));
    if (blockIdx.y == 0 && (threadIdx.x & 7) == 0) ea[row] = e;
    double a[8], aR[8];
#pragma unroll
    for (int q = 0; q < 8; q++) scaled_int(v[q], t - e, a[q], aR[q]);
    store_residues8<NLC>(a, aR, md, out + (size_t)row * Kp + k0, (size_t)Mp * Kp);
}

// Eight consecutive K of column `col` of B (rows through the segment offsets; K segments are
// multiples of 16 long, so k0 % 8 == 0 keeps the eight in one segment); zero outside B.
__device__ __forceinline__ void b_values8(const GemmArgs<double> &g, int col, int k0, double (&v)[8])
{
#pragma unroll
    for (int q = 0; q < 8; q++) v[q] = 0.0;
    if (col >= g.N || k0 >= g.K) return;
    int kb = 0;
    const int sg = find_seg(g, k0, kb);
    if (sg < 0) return;
    const int off = k0 - kb;
    const double *b = g.B + (size_t)g.seg[sg].boff + off + (size_t)col * g.ldb;
#pragma unroll
    for (int q = 0; q < 8; q++)
        if (off + q < g.seg[sg].acols && g.seg[sg].boff + off + q < g.brows) v[q] = b[q];
}

// Largest |B(k, j)| of each column, as the bit pattern of a non-negative double, max-reduced
// into cmax[col] (zeroed by the caller).  Grid: (Np / 32, Kp / 64); thread = (column t / 8,
// K 8 (t % 8) .. +7 of the block's 64).
__global__ void __launch_bounds__(256) col_absmax_kernel(GemmArgs<double> g, unsigned long long *cmax)
{
    // with a per-column K extent (nondecreasing), B is zero from kext[col] on
    if (g.kext && (int)blockIdx.y * 64 >= g.kext[min((int)blockIdx.x * 32 + 31, g.N - 1)]) return;
    const int col = blockIdx.x * 32 + (threadIdx.x >> 3);
    const int k0 = blockIdx.y * 64 + (threadIdx.x & 7) * 8;
    double v[8];
    b_values8(g, col, k0, v);
    double mx = 0.0;
#pragma unroll
    for (int q = 0; q < 8; q++) mx = fmax(mx, fabs(v[q]));
#pragma unroll
    for (int o = 1; o < 8; o <<= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    if ((threadIdx.x & 7) == 0 && mx > 0.0) atomicMax(&cmax[col], (unsigned long long)__double_as_longlong(mx));
}

// Columns of B -> residues out[l][col][k] (column pitch Kp, l-th block of Np columns),
// eb[col].  Grid: (Np / 32, Kp / 64), the thread layout of col_absmax_kernel; a thread
// stores 8 bytes per modulus.  With a per-column K extent the GEMM reads a tile of `tnw`
// columns up to the extent of its last column: K blocks beyond it are not written.
template <int NLC>
__global__ void __launch_bounds__(256) residue_cols_kernel(GemmArgs<double> g, int Kp, int Np, int tnw, int t,
                                                           Moduli md, const unsigned long long *cmax, int8_t *out,
                                                           int *eb)
{
    if (g.kext) {
        const int last = min(((int)blockIdx.x * 32 / tnw + 1) * tnw, g.N) - 1;
        if ((int)blockIdx.y * 64 >= g.kext[last]) return;
    }
    const int col = blockIdx.x * 32 + (threadIdx.x >> 3);
    const int k0 = blockIdx.y * 64 + (threadIdx.x & 7) * 8;
    const int e = split::scale_exp(__longlong_as_double((long long)cmax[col]));
    if (blockIdx.y == 0 && (threadIdx.x & 7) == 0) eb[col] = e;
    double v[8];
    b_values8(g, col, k0, v);
    double a[8], aR[8];
#pragma unroll
    for (int q = 0; q < 8; q++) scaled_int(v[q], t - e, a[q], aR[q]);
    store_residues8<NLC>(a, aR, md, out + (size_t)col * Kp + k0, (size_t)Np * Kp);
}

// ---- the residue GEMM ---------------------------------------------------------------------
// c mod p in [0, p) for |c| < 2^27 (K <= 2^13 terms of |a b| <= 2^14; the host keeps K below
// 2^16, |c| < 2^30): c + p 2^23 >= 0 is reduced by Barrett's method with floor(2^32 / p)
// (a quotient at most one short), integer operations only.
__device__ __forceinline__ unsigned int mod_p(int c, unsigned int p, unsigned int barrett)
{
    const unsigned int x = (unsigned int)c + (p << 23);  // the true sum is in [0, 2^32)
    const unsigned int q = __umulhi(x, barrett);
    unsigned int r = x - q * p;                          // in [0, 2p)
    return r >= p ? r - p : r;
}

__device__ __forceinline__ void item_tile(const Params &p, int item, int &l, int &m0, int &n0, int &ksteps)
{
    const int per = p.mtiles * p.ntiles;
    l = item / per;
    const int r = item - l * per;
    const int nt = r / p.mtiles;
    m0 = (r - nt * p.mtiles) * TM;
    // with a per-column K extent (back-transform) the longest column tiles come first
    n0 = (p.kext ? p.ntiles - 1 - nt : nt) * TN;
    int kmax = p.Kp;
    if (p.kext) kmax = min(kmax, p.kext[min(n0 + TN, p.N) - 1]);
    ksteps = max(1, (kmax + BK - 1) / BK);
}

// tmR: A residues (rows l Mp + m, K bytes), box TM rows; tmC: B residues (rows l Np + n), box TN.
__global__ void __launch_bounds__(THREADS, 1)
gemm_crt_kernel(const __grid_constant__ CUtensorMap tmR, const __grid_constant__ CUtensorMap tmC, Params p)
{
    extern __shared__ __align__(16) unsigned char smem_crt[];
    unsigned char *base = reinterpret_cast<unsigned char *>(((uintptr_t)smem_crt + 1023) & ~(uintptr_t)1023);
    unsigned char *sR = base;                        // [STAGES][ROW_TILE]
    unsigned char *sC = base + STAGES * ROW_TILE;    // [STAGES][COL_TILE]
    __shared__ __align__(8) uint64_t full[STAGES], empty[STAGES], acc_full[2], acc_empty[2], mma_done;
    __shared__ uint32_t tmem_base;
    __shared__ volatile int abort_flag;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (threadIdx.x == 0) {
        abort_flag = 0;
        for (int q = 0; q < STAGES; q++) {
            split::mbar_init(&full[q], 1);
            split::mbar_init(&empty[q], 1);
        }
        for (int q = 0; q < 2; q++) {
            split::mbar_init(&acc_full[q], 1);
            split::mbar_init(&acc_empty[q], EPI_WARPS);
        }
        split::mbar_init(&mma_done, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1) {  // TMEM: two accumulators of 256 columns
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         split::smem_u32(&tmem_base)),
                     "r"(512));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    split::tc_fence_before();
    __syncthreads();
    split::tc_fence_after();
    const uint32_t tmem = tmem_base;

    if (warp == 0) {
        // ---------------- TMA producer ----------------
        if (lane == 0) {
            long long use = 0;  // stage fills issued
            for (int item = blockIdx.x; item < p.items && !abort_flag; item += gridDim.x) {
                int l, m0, n0, ks;
                item_tile(p, item, l, m0, n0, ks);
                bool ok = true;
                for (int k = 0; k < ks; k++, use++) {
                    const int s = (int)(use % STAGES);
                    if (use >= STAGES &&
                        !split::mbar_wait(&empty[s], (uint32_t)(((use / STAGES) - 1) & 1), &abort_flag, p.err)) {
                        ok = false;
                        break;
                    }
                    split::mbar_expect_tx(&full[s], (uint32_t)(ROW_TILE + COL_TILE));
                    split::tma_load_2d(sR + s * ROW_TILE, &tmR, k * BK, l * p.Mp + m0, &full[s]);
                    split::tma_load_2d(sC + s * COL_TILE, &tmC, k * BK, l * p.Np + n0, &full[s]);
                }
                if (!ok) break;
            }
            if (abort_flag) {
                // let every issued load land before the CTA can exit: the latest fill of
                // stage s is its n-th with n = fills of s; it completes phase n - 1
                for (int s = 0; s < STAGES; s++) {
                    const long long fills = use / STAGES + (s < use % STAGES ? 1 : 0);
                    if (fills) split::mbar_drain(&full[s], (uint32_t)((fills - 1) & 1));
                }
            }
        }
    } else if (warp == 1) {
        // ---------------- MMA issue ----------------
        if (lane == 0) {
            long long use = 0;
            int tcount = 0;
            bool ok = true;
            for (int item = blockIdx.x; item < p.items && ok; item += gridDim.x, tcount++) {
                int l, m0, n0, ks;
                item_tile(p, item, l, m0, n0, ks);
                const int buf = tcount & 1;
                if (tcount >= 2) {
                    if (!split::mbar_wait(&acc_empty[buf], (uint32_t)(((tcount >> 1) - 1) & 1), &abort_flag, p.err))
                        break;
                    split::tc_fence_after();
                }
                const uint32_t dcol = tmem + (uint32_t)(buf * TM);
                for (int k = 0; k < ks; k++, use++) {
                    const int s = (int)(use % STAGES);
                    if (!split::mbar_wait(&full[s], (uint32_t)((use / STAGES) & 1), &abort_flag, p.err)) {
                        ok = false;
                        break;
                    }
                    split::tc_fence_after();
#pragma unroll
                    for (int kk = 0; kk < 2; kk++)  // two 32-byte-deep MMAs per 64-byte K step
                        split::umma_i8(dcol, split::smem_desc(sC + s * COL_TILE, kk * 32),
                                       split::smem_desc(sR + s * ROW_TILE, kk * 32), IDESC, (k | kk) ? 1u : 0u);
                    split::umma_commit(&empty[s]);
                }
                if (ok) split::umma_commit(&acc_full[buf]);
            }
            // every MMA issued so far completes before TMEM can be released
            split::umma_commit(&mma_done);
            split::mbar_drain(&mma_done, 0);
        }
    } else {
        // ---------------- epilogue: warps 2..9 ----------------
        // TMEM lane = column of C (quadrant of the warp), TMEM column = row of C; the warp
        // takes 128 of the tile's 256 rows in chunks of 32
        const int quad = warp & 3, half = (warp - 2) >> 2;
        int tcount = 0;
        for (int item = blockIdx.x; item < p.items; item += gridDim.x, tcount++) {
            int l, m0, n0, ks;
            item_tile(p, item, l, m0, n0, ks);
            const int buf = tcount & 1;
            if (!split::mbar_wait(&acc_full[buf], (uint32_t)((tcount >> 1) & 1), &abort_flag, p.err)) break;
            split::tc_fence_after();
            const unsigned int pl = (unsigned int)p.p[l], bl = p.barrett[l];
            const int col = n0 + quad * 32 + lane;
            unsigned char *Ucol = p.U + ((size_t)l * p.Np + col) * p.Mp + m0 + half * 128;
            const uint32_t tb = tmem + ((uint32_t)(quad * 32) << 16) + (uint32_t)(buf * TM + half * 128);
#pragma unroll 1
            for (int h = 0; h < 128; h += 32) {
                uint32_t v[32];
                split::tmem_ld32(tb + (uint32_t)h, v);
                split::tmem_wait_ld();
                uint32_t w[8];
#pragma unroll
                for (int g = 0; g < 8; g++)
                    w[g] = mod_p((int)v[4 * g], pl, bl) | (mod_p((int)v[4 * g + 1], pl, bl) << 8) |
                           (mod_p((int)v[4 * g + 2], pl, bl) << 16) | (mod_p((int)v[4 * g + 3], pl, bl) << 24);
                uint4 *dst = reinterpret_cast<uint4 *>(Ucol + h);  // 32 rows: 32 contiguous bytes
                dst[0] = make_uint4(w[0], w[1], w[2], w[3]);
                dst[1] = make_uint4(w[4], w[5], w[6], w[7]);
            }
            split::tc_fence_before();
            __syncwarp();
            if (lane == 0) split::mbar_arrive(&acc_empty[buf]);
        }
    }

    split::tc_fence_before();
    __syncthreads();
    if (warp == 1) {
        split::tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(512));
    }
}

// ---- reconstruction ---------------------------------------------------------------------
// One thread per 4 consecutive rows of one column (grid: (Mp / 1024, N), 256 threads): the
// 4 residues of each modulus come in one 32-bit load (a warp reads 128 contiguous bytes per
// modulus), all L loads in flight before the arithmetic; C' of each element from its
// residues, scaled into C.  A residue byte u becomes a double as (2^52 + u) - 2^52, the
// byte placed in the low word of 2^52 (an FP64 add instead of a conversion instruction).
// NLC > 0: the modulus count as a compile-time constant.
template <int NLC>
__global__ void __launch_bounds__(256) crt_kernel(const unsigned char *U, int Mp, int Np, Moduli md, int t,
                                                  const int *ea, const int *eb, int M, int N, int mlo, double *C,
                                                  int ldc, const int *ccol, int accumulate)
{
    constexpr int LMAX = NLC > 0 ? NLC : MAXL;
    const int L = NLC > 0 ? NLC : md.L;
    const int row0 = (blockIdx.x * blockDim.x + threadIdx.x) * 4;
    const int col = blockIdx.y;
    if (row0 >= M || col >= N) return;
    const size_t plane = (size_t)Np * Mp;
    const uint32_t *u = reinterpret_cast<const uint32_t *>(U + (size_t)col * Mp + row0);  // Mp % 128 == 0
    uint32_t w[LMAX];
#pragma unroll
    for (int l = 0; l < LMAX; l++) w[l] = l < L ? u[(size_t)l * plane / 4] : 0u;
    const double two_hi = ldexp(1.0, md.hi), two_lo = ldexp(1.0, md.lo);
    constexpr double two52 = 4503599627370496.0;
    const int ecol = eb[col] - 2 * t;
    double *ccolp = C + (size_t)(ccol ? ccol[col] : col) * ldc;
#pragma unroll
    for (int q = 0; q < 4; q++) {
        const int row = row0 + q;
        if (row < mlo || row >= M) continue;
        double H = 0.0, Mid = 0.0;
#pragma unroll
        for (int l = 0; l < LMAX; l++) {
            const double ul = __dsub_rn(__hiloint2double(0x43300000, (int)__byte_perm(w[l], 0u, 0x4440 + q)), two52);
            H = fma(ul, md.w1[l], H);
            Mid = fma(ul, md.w2[l], Mid);
        }
        const double k = rint(fma(H, md.c1, Mid * md.c2));
        const double d1 = fma(-k, md.P1, H);  // exact integers
        const double d2 = fma(-k, md.P2, Mid);
        const double cp = fma(d1, two_hi, d2 * two_lo);  // both products exact (powers of two)
        const double v = ldexp(cp, ea[row] + ecol);
        double *cptr = ccolp + row;
        *cptr = accumulate ? *cptr + v : v;
    }
}

}  // namespace crt
}  // namespace xtg
