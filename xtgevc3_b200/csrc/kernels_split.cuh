// Split-precision FP64 GEMM on the 5th-generation tensor cores (tcgen05, BF16 -> FP32).
//
//   C[mlo:M, j] (+)= sum_k A(m, k) B(k, j)       A, B, C in FP64
//
// Slicing (Ozaki-style, integer slices): row m of A is scaled by 2^-ea_m so that |v| < 1,
// then t_0 = 256 v, a_i = rint(t_i), t_(i+1) = 256 (t_i - a_i), so that
//   256 v = sum_i a_i 256^-i      (s slices; error below 256^-(s-1) / 2)
// with |a_0| <= 256 and |a_i| <= 128 for i >= 1: integers with at most 8 significant bits.
// Slice i is stored pre-scaled, a_i 256^-i, which is still exact in BF16.  Columns of B
// likewise (exponent eb_j).  Then
//   (A B)(m, j) = 2^(ea_m + eb_j - 16) sum_{i + i' <= s-1} (a_i 256^-i) . (b_i' 256^-i')
// (pairs below the anti-diagonal are dropped: they are below the slicing error).
//
// Accumulation.  Every pair product of anti-diagonal g = i + i' is an integer sum times
// 256^-g.  Over a K-chunk of 128 the partial sums of the diagonals g = 0 .. 3 stay below
// 2^24 in units of 256^-g (per K index at most 2^16, 2^16, 2^16 + 2^14 and 3 x 2^15), so
// each of these four is accumulated EXACTLY in its own FP32 TMEM accumulator.  All
// diagonals g >= 4 together are below 2^-32 of the leading terms and share a fifth FP32
// accumulator, where FP32 rounding stays below 2^-50 of them.  After each chunk the five
// accumulators are added into FP64 registers; FP64 summation across chunks.
//
// Kernel (one CTA per 128 x 96 output tile, 10 warps, one CTA per SM):
//   warp 0: TMA producer.  Per 32-deep K step: the s slices of the B tile (BSTAGES
//           buffered), then the s slices of the A tile through an 8-stage ring.
//   warp 1: TMEM allocation (512 columns; 5 accumulators x 96) and MMA issue (one
//           thread): for A slice i, MMAs with B slices i' <= s-1-i into accumulator
//           min(i + i', 4); commits release the smem buffers and, per chunk, the
//           accumulators.
//   warps 2-9: epilogue.  Warp w reads TMEM lanes 32 (w % 4) .. +31 and columns
//           48 ((w - 2) / 4) .. +47: per chunk it adds the accumulators into 48 FP64
//           registers per thread; at the end it scales by 2^(ea + eb - 16), adds C for
//           accumulating launches and stores.
// Shared-memory tiles are K-major with 64-byte swizzle (TMA SWIZZLE_64B), described to the
// MMA by matrix descriptors; no TMA multicast anywhere.
//
// Every mbarrier wait is bounded: on expiry the waiting thread sets the CTA's abort flag
// and the global error word, every role leaves its loop, loads and MMAs already in flight
// are drained (bounded), and TMEM is released.
#pragma once
#include <cuda.h>
#include <cuda_bf16.h>

#include "common.cuh"
#include "kernels_gemm.cuh"

namespace xtg {
namespace split {

constexpr int BM = 128;                      // output rows per CTA (one TMEM lane each)
constexpr int THREADS = 320;
constexpr int EPI_WARPS = 8;
constexpr long long kSpinLimit = 1ll << 22;  // bounded mbarrier polls (legitimate waits are microseconds)

// Slice kinds.  Both move 64-byte K rows (one 64-byte swizzle span) per TMA box and issue
// two 32-byte-deep MMAs per K step.
//   kBF16: BF16 slices (8-bit digits) on kind::f16 with FP32 accumulators; diagonals
//          0..3 exact per 128-deep K chunk, diagonals >= 4 shared (see above).
//   kI8:   INT8 slices (7-bit digits) on kind::i8 with INT32 accumulators, one per
//          diagonal, exact over any K up to 2^15 (|digit| <= 64, at most 7 products per
//          diagonal: 7 * 2^12 * 2^15 < 2^31), so K is never chunked.
enum SliceKind : int { kBF16 = 0, kI8 = 1 };

template <int KIND> struct Cfg;
template <> struct Cfg<kBF16> {
    using Elem = __nv_bfloat16;
    static constexpr int BN = 96, BK = 32, CHUNK = 128, MAXS = 6, NACC = 5, ASTAGES = 8, BSTAGES = 2;
    // BF16 x BF16 -> FP32, K-major A and B, M = BM, N = BN
    static constexpr uint32_t IDESC =
        (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(BN >> 3) << 17) | ((uint32_t)(BM >> 4) << 24);
};
template <> struct Cfg<kI8> {
    using Elem = int8_t;
    static constexpr int BN = 64, BK = 64, CHUNK = 32768, MAXS = 7, NACC = 7, ASTAGES = 12, BSTAGES = 2;
    // S8 x S8 -> S32, K-major A and B, M = BM, N = BN
    static constexpr uint32_t IDESC =
        (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(BN >> 3) << 17) | ((uint32_t)(BM >> 4) << 24);
};

template <int KIND> struct Layout {
    using C = Cfg<KIND>;
    static constexpr int A_TILE = BM * 64;        // bytes per A slice tile (64-byte K rows)
    static constexpr int B_TILE = C::BN * 64;     // bytes per B slice tile (a multiple of the 512-B atom)
    static constexpr int EPI_COLS = C::BN / 2;    // columns per epilogue thread
    // dynamic shared memory: [B buffers: BSTAGES x MAXS tiles][A ring: ASTAGES tiles], 1024-aligned
    static constexpr int SMEM_B = C::BSTAGES * C::MAXS * B_TILE;
    static constexpr int SMEM_A = C::ASTAGES * A_TILE;
    static constexpr int SMEM_BYTES = SMEM_B + SMEM_A + 1024;  // + alignment slack
    static_assert(C::NACC * C::BN <= 512, "accumulators exceed TMEM");
};

struct Params {
    int M, N, Kp, s;          // Kp: padded K (multiple of BK) of the slice buffers
    int Mp, Np;               // padded rows of A slices / columns of B slices
    int mlo, accumulate;
    const int *ea, *eb;       // exponents of rows of A / columns of B
    const int *kext;          // per output column: K extent (nullptr: Kp)
    double *C;
    int ldc;
    const int *ccol;
    int *err;                 // global error word (kErrWaitTimeout on a bounded-wait expiry)
};

// ---- PTX helpers --------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t *b, int count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(b)), "r"(count));
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t *b, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(b)), "r"(bytes));
}
__device__ __forceinline__ void mbar_arrive(uint64_t *b)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(b)));
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *b, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(b)), "r"(parity));
    return ok != 0;
}
// Bounded wait; returns false (and raises the abort flags) on expiry or when another role
// has already aborted.
__device__ __forceinline__ bool mbar_wait(uint64_t *b, uint32_t parity, volatile int *abort, int *err)
{
    for (long long it = 0; it < kSpinLimit; it++) {
        if (mbar_try_wait(b, parity)) return true;
        if ((it & 1023) == 1023 && *abort) return false;
    }
    *abort = 1;
    atomicOr(err, kErrWaitTimeout);
    return false;
}
// Bounded wait that ignores the abort flag (used to drain work already in flight).
__device__ __forceinline__ void mbar_drain(uint64_t *b, uint32_t parity)
{
    for (long long it = 0; it < kSpinLimit; it++)
        if (mbar_try_wait(b, parity)) return;
}

__device__ __forceinline__ void tma_load_2d(void *dst, const CUtensorMap *map, int x, int y, uint64_t *bar)
{
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];"
        ::"r"(smem_u32(dst)), "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(smem_u32(bar))
        : "memory");
}

// K-major, 64-byte swizzled operand: rows of 64 B (32 BF16), 8-row atoms 512 B apart.
__device__ __forceinline__ uint64_t smem_desc(const void *tile, int kbyte_off)
{
    const uint32_t addr = smem_u32(tile) + kbyte_off;
    uint64_t d = 0;
    d |= (uint64_t)((addr >> 4) & 0x3FFF);        // start address
    d |= (uint64_t)1 << 16;                       // leading byte offset (unused for swizzled K-major)
    d |= (uint64_t)(512 >> 4) << 32;              // stride byte offset: 8 rows x 64 B
    d |= (uint64_t)1 << 46;                       // descriptor version (sm100)
    d |= (uint64_t)4 << 61;                       // SWIZZLE_64B
    return d;
}

template <int KIND>
__device__ __forceinline__ void umma(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t accumulate)
{
    if constexpr (KIND == kBF16)
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "setp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
            ::"r"(tmem_d), "l"(adesc), "l"(bdesc), "r"(Cfg<KIND>::IDESC), "r"(accumulate), "r"(0), "r"(0), "r"(0),
            "r"(0));
    else
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "setp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
            ::"r"(tmem_d), "l"(adesc), "l"(bdesc), "r"(Cfg<KIND>::IDESC), "r"(accumulate), "r"(0), "r"(0), "r"(0),
            "r"(0));
}
// INT8 MMA with a runtime instruction descriptor (any M / N the descriptor encodes)
__device__ __forceinline__ void umma_i8(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                        uint32_t accumulate)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}"
        ::"r"(tmem_d), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate));
}
__device__ __forceinline__ void umma_commit(uint64_t *bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&r)[16])
{
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
}
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&r)[32])
{
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// ---- the MMA kernel ---------------------------------------------------------------------
template <int KIND>
__global__ void __launch_bounds__(THREADS, 1)
gemm_split_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB, Params p)
{
    using C = Cfg<KIND>;
    using L = Layout<KIND>;
    constexpr int BN = C::BN, BK = C::BK, CHUNK = C::CHUNK, MAXS = C::MAXS, NACC = C::NACC, ASTAGES = C::ASTAGES;
    constexpr int BSTAGES = C::BSTAGES;
    constexpr int A_TILE = L::A_TILE, B_TILE = L::B_TILE, EPI_COLS = L::EPI_COLS, SMEM_B = L::SMEM_B;
    extern __shared__ __align__(16) unsigned char smem_split[];
    // tiles need 512-byte alignment (64-byte swizzle atoms); SMEM_BYTES includes the slack
    unsigned char *base = reinterpret_cast<unsigned char *>(((uintptr_t)smem_split + 1023) & ~(uintptr_t)1023);
    unsigned char *sB = base;               // [BSTAGES][MAXS][B_TILE]
    unsigned char *sA = base + SMEM_B;      // [ASTAGES][A_TILE]
    __shared__ __align__(8) uint64_t a_full[ASTAGES], a_empty[ASTAGES], b_full[BSTAGES], b_empty[BSTAGES], acc_full, acc_empty,
        mma_done;
    __shared__ uint32_t tmem_base;
    __shared__ volatile int abort_flag;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    // with a per-column K extent (back-transform) the column tiles run last-first, so the
    // longest tiles start first
    const int m0 = blockIdx.x * BM, n0 = (p.kext ? gridDim.y - 1 - blockIdx.y : blockIdx.y) * BN;
    const int s = p.s;
    const int nacc = s < NACC ? s : NACC;
    int kmax = p.Kp;
    if (p.kext) {
        const int last = min(n0 + BN, p.N) - 1;
        kmax = min(kmax, p.kext[last]);
    }
    const int ksteps = (kmax + BK - 1) / BK;
    constexpr int kPerChunk = CHUNK / BK;
    const int nchunks = (ksteps + kPerChunk - 1) / kPerChunk;

    if (threadIdx.x == 0) {
        abort_flag = 0;
        for (int q = 0; q < ASTAGES; q++) {
            mbar_init(&a_full[q], 1);
            mbar_init(&a_empty[q], 1);
        }
        for (int q = 0; q < BSTAGES; q++) {
            mbar_init(&b_full[q], 1);
            mbar_init(&b_empty[q], 1);
        }
        mbar_init(&acc_full, 1);
        mbar_init(&acc_empty, EPI_WARPS);
        mbar_init(&mma_done, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1) {  // TMEM: 512 columns (4 accumulators of 128 columns)
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base)),
                     "r"(512));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tmem_base;

    if (warp == 0) {
        // ---------------- TMA producer ----------------
        if (lane == 0) {
            int astage = 0, ause = 0;
            uint32_t aph = 0;      // phase bits of the A stages, one bit per stage
            uint32_t bph = 0;      // phase bits of the B buffers, one bit per buffer
            uint32_t afill = 0;    // stages holding a load not yet observed complete (for the drain)
            int bfills[BSTAGES] = {};
            for (int t = 0; t < ksteps && !abort_flag; t++) {
                const int bb = t % BSTAGES;
                if (t >= BSTAGES) {
                    if (!mbar_wait(&b_empty[bb], (bph >> bb) & 1u, &abort_flag, p.err)) break;
                    bph ^= 1u << bb;
                }
                mbar_expect_tx(&b_full[bb], (uint32_t)(s * B_TILE));
                for (int j = 0; j < s; j++)
                    tma_load_2d(sB + (bb * MAXS + j) * B_TILE, &tmB, t * BK, j * p.Np + n0, &b_full[bb]);
                bfills[bb]++;
                bool ok = true;
                for (int i = 0; i < s; i++, ause++) {
                    if (ause >= ASTAGES) {
                        if (!mbar_wait(&a_empty[astage], (aph >> astage) & 1u, &abort_flag, p.err)) {
                            ok = false;
                            break;
                        }
                        aph ^= 1u << astage;
                    }
                    mbar_expect_tx(&a_full[astage], (uint32_t)A_TILE);
                    tma_load_2d(sA + astage * A_TILE, &tmA, t * BK, i * p.Mp + m0, &a_full[astage]);
                    afill |= 1u << astage;
                    astage = (astage + 1) % ASTAGES;
                }
                if (!ok) break;
            }
            if (abort_flag) {  // let every load already issued land before the CTA can exit
                // a stage's latest fill is its n-th with n = (uses of the stage); parity (n-1) & 1
                for (int q = 0; q < ASTAGES; q++) {
                    if (!((afill >> q) & 1u)) continue;
                    const int uses = ause / ASTAGES + (q < ause % ASTAGES ? 1 : 0);
                    if (uses) mbar_drain(&a_full[q], (uint32_t)((uses - 1) & 1));
                }
                for (int q = 0; q < BSTAGES; q++)
                    if (bfills[q]) mbar_drain(&b_full[q], (uint32_t)((bfills[q] - 1) & 1));
            }
        }
    } else if (warp == 1) {
        // ---------------- MMA issue ----------------
        if (lane == 0) {
            int astage = 0;
            uint32_t aph = 0, bph = 0, eph = 0;
            bool ok = true;
            for (int c = 0; c < nchunks && ok; c++) {
                if (c > 0) {
                    if (!mbar_wait(&acc_empty, eph, &abort_flag, p.err)) break;
                    eph ^= 1;
                    tc_fence_after();
                }
                for (int tt = 0; tt < kPerChunk && ok; tt++) {
                    const int t = c * kPerChunk + tt;
                    if (t >= ksteps) break;
                    const int bb = t % BSTAGES;
                    if (!mbar_wait(&b_full[bb], (bph >> bb) & 1u, &abort_flag, p.err)) { ok = false; break; }
                    bph ^= 1u << bb;
                    tc_fence_after();
                    for (int i = 0; i < s; i++) {
                        if (!mbar_wait(&a_full[astage], (aph >> astage) & 1u, &abort_flag, p.err)) { ok = false; break; }
                        aph ^= 1u << astage;
                        tc_fence_after();
                        const unsigned char *at = sA + astage * A_TILE;
                        for (int j = 0; i + j < s; j++) {  // pair (i, j), anti-diagonal i + j
                            const unsigned char *bt = sB + (bb * MAXS + j) * B_TILE;
                            const int g = (i + j) < NACC - 1 ? (i + j) : NACC - 1;
                            const uint32_t dcol = tmem + (uint32_t)(g * BN);
                            // the first product into each accumulator of a chunk overwrites it
                            const bool first = tt == 0 && i == 0 && j <= NACC - 1;
#pragma unroll
                            for (int kk = 0; kk < 2; kk++)  // two 32-byte-deep MMAs per 64-byte K step
                                umma<KIND>(dcol, smem_desc(at, kk * 32), smem_desc(bt, kk * 32),
                                           (first && kk == 0) ? 0u : 1u);
                        }
                        umma_commit(&a_empty[astage]);
                        astage = (astage + 1) % ASTAGES;
                    }
                    if (ok) umma_commit(&b_empty[bb]);
                }
                if (ok) umma_commit(&acc_full);
            }
            // every MMA issued so far completes before TMEM can be released
            umma_commit(&mma_done);
            mbar_drain(&mma_done, 0);
        }
    } else {
        // ---------------- epilogue: warps 2..9 ----------------
        const int quad = warp & 3, half = (warp - 2) >> 2;
        const int row = m0 + quad * 32 + lane;
        const uint32_t tbase = tmem + ((uint32_t)(quad * 32) << 16) + (uint32_t)(half * EPI_COLS);
        double acc[EPI_COLS];
#pragma unroll
        for (int q = 0; q < EPI_COLS; q++) acc[q] = 0.0;
        uint32_t fph = 0;
        for (int c = 0; c < nchunks; c++) {
            if (!mbar_wait(&acc_full, fph, &abort_flag, p.err)) break;
            fph ^= 1;
            tc_fence_after();
            for (int g = 0; g < nacc; g++) {
                // BF16 slices carry their scale 256^-i; INT8 digits are integers: 2^-7g here
                const double w = KIND == kI8 ? ldexp(1.0, -7 * g) : 1.0;
#pragma unroll
                for (int h = 0; h < EPI_COLS / 16; h++) {
                    uint32_t v[16];
                    tmem_ld16(tbase + (uint32_t)(g * BN + h * 16), v);
                    tmem_wait_ld();
#pragma unroll
                    for (int q = 0; q < 16; q++) {
                        if constexpr (KIND == kI8) acc[h * 16 + q] += w * (double)(int)v[q];
                        else acc[h * 16 + q] += (double)__uint_as_float(v[q]);
                    }
                }
            }
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(&acc_empty);
        }
        if (!abort_flag && row >= p.mlo && row < p.M) {
            const int er = p.ea[row] - (KIND == kI8 ? 12 : 16);
#pragma unroll
            for (int q = 0; q < EPI_COLS; q++) {
                const int col = n0 + half * EPI_COLS + q;
                if (col < p.N) {
                    double *cp = p.C + (size_t)(p.ccol ? p.ccol[col] : col) * p.ldc + row;
                    const double v = ldexp(acc[q], er + p.eb[col]);
                    *cp = p.accumulate ? *cp + v : v;
                }
            }
        }
    }

    tc_fence_before();
    __syncthreads();
    if (warp == 1) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(512));
    }
}

// ---- slicing kernels ----------------------------------------------------------------------
// exponent e with 2^-e max in [0.5, 1) (0 for a zero vector)
__device__ __forceinline__ int scale_exp(double mx) { return mx > 0.0 ? ilogb(mx) + 1 : 0; }

// v in (-1, 1) -> s slices.  BF16: pre-scaled a_i 256^-i with t_0 = 256 v (see the header
// comment).  INT8: integer digits a_i with t_0 = 64 v, t_(i+1) = 128 (t_i - a_i), so that
// v = sum_i a_i 2^(-6-7i) + O(2^(-7s)) and |a_i| <= 64.
template <int KIND>
__device__ __forceinline__ void slice_value(double v, int s, typename Cfg<KIND>::Elem *out, size_t stride)
{
    if constexpr (KIND == kBF16) {
        double t = v * 256.0;
        for (int i = 0; i < s; i++) {
            const double a = rint(t);
            t = (t - a) * 256.0;
            out[(size_t)i * stride] = __double2bfloat16(ldexp(a, -8 * i));
        }
    } else {
        double t = v * 64.0;
        for (int i = 0; i < s; i++) {
            const double a = rint(t);
            t = (t - a) * 128.0;
            out[(size_t)i * stride] = (int8_t)(int)a;
        }
    }
}

// Rows of A (through the segment description of a GEMM launch) -> slices
// out[i][row][k] (row pitch Kp, i-th block of Mp rows), ea[row].  One CTA = 32 rows.
template <int KIND>
__global__ void __launch_bounds__(256) slice_rows_kernel(GemmArgs<double> g, int Kp, int Mp, int s,
                                                         typename Cfg<KIND>::Elem *out, int *ea)
{
    __shared__ double tile[64][33];
    __shared__ double rmax[8][32];
    const int r0 = blockIdx.x * 32;
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    // pass 1: row maxima (rows along lanes: coalesced column-major reads)
    double mx = 0.0;
    const int row = r0 + tx;
    for (int k = ty; k < g.K; k += 8) {
        int kb = 0;
        const int sg = find_seg(g, k, kb);
        const int col = k - kb;
        if (sg >= 0 && row < g.M && col < g.seg[sg].acols)
            mx = fmax(mx, fabs(g.seg[sg].A[(size_t)row + (size_t)col * g.seg[sg].lda]));
    }
    rmax[ty][tx] = mx;
    __syncthreads();
    if (ty == 0) {
        double m = rmax[0][tx];
        for (int q = 1; q < 8; q++) m = fmax(m, rmax[q][tx]);
        rmax[0][tx] = m;
        if (row < Mp) ea[row] = scale_exp(m);
    }
    __syncthreads();
    const int e = scale_exp(rmax[0][tx]);
    // pass 2: 64-wide K tiles through shared memory, written K-contiguous
    for (int k0 = 0; k0 < Kp; k0 += 64) {
        for (int kk = ty; kk < 64; kk += 8) {
            const int k = k0 + kk;
            double v = 0.0;
            if (k < g.K) {
                int kb = 0;
                const int sg = find_seg(g, k, kb);
                const int col = k - kb;
                if (sg >= 0 && row < g.M && col < g.seg[sg].acols)
                    v = g.seg[sg].A[(size_t)row + (size_t)col * g.seg[sg].lda];
            }
            tile[kk][tx] = ldexp(v, -e);
        }
        __syncthreads();
        // thread (ty, tx): rows ty*4 .. +3, k = tx and tx + 32 (Kp is a multiple of 32)
        for (int rr = ty * 4; rr < ty * 4 + 4; rr++) {
            const int gr = r0 + rr;
            if (gr >= Mp) continue;
            for (int h = 0; h < 2; h++) {
                const int kk = tx + 32 * h;
                if (k0 + kk >= Kp) continue;
                slice_value<KIND>(tile[kk][rr], s, out + (size_t)gr * Kp + k0 + kk, (size_t)Mp * Kp);
            }
        }
        __syncthreads();
    }
}

// Columns of B (rows through the segment offsets) -> slices out[j][col][k], eb[col].
// One warp per column, lanes along K.
template <int KIND>
__global__ void __launch_bounds__(256) slice_cols_kernel(GemmArgs<double> g, int Kp, int Np, int s,
                                                         typename Cfg<KIND>::Elem *out, int *eb)
{
    const int col = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (col >= Np) return;
    auto bval = [&](int k) -> double {
        if (col >= g.N || k >= g.K) return 0.0;
        int kb = 0;
        const int sg = find_seg(g, k, kb);
        if (sg < 0) return 0.0;
        const int r = g.seg[sg].boff + k - kb;
        if (r >= g.brows || k - kb >= g.seg[sg].acols) return 0.0;  // B rows past a segment's columns pair with zeros
        return g.B[(size_t)r + (size_t)col * g.ldb];
    };
    double mx = 0.0;
    for (int k = lane; k < g.K; k += 32) mx = fmax(mx, fabs(bval(k)));
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    const int e = scale_exp(mx);
    if (lane == 0) eb[col] = e;
    for (int k = lane; k < Kp; k += 32)
        slice_value<KIND>(ldexp(bval(k), -e), s, out + (size_t)col * Kp + k, (size_t)Np * Kp);
}

}  // namespace split
}  // namespace xtg
