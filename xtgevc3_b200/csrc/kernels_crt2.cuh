// Residue GEMM on SM pairs (tcgen05 cta_group::2): the kernel of kernels_crt.cuh with a
// pair tile of 256 rows x 256 columns of C computed by a cluster of two CTAs.
//
// The MMA (M = 256, N = 256, issued by the pair's leader CTA) runs M over C's columns and N
// over C's rows.  CTA r of the pair holds, at the same shared-memory offsets, its 128
// columns of C's operand (the MMA's M half) and 128 of the tile's 256 rows (its N half); the
// MMA reads both CTAs' halves, and CTA r's TMEM receives its 128 columns of C for all 256
// rows.  Per SM and per 64-byte K step that is 16 KB of operands for 128 x 256 x 64
// products, against 24 KB in the one-CTA tile: the loads from L2, which bound the one-CTA
// kernel, shrink by a third.
//
// Synchronisation (barriers at the same offsets in both CTAs; "leader" = rank 0):
//   full[s]     leader only: the leader's producer arms it with both CTAs' bytes; both
//               producers' TMA loads (cta_group::2 form, no multicast) complete on it;
//   empty[s]    both: the MMA's commit arrives on both CTAs' copies (multicast commit);
//   acc_full[b] both: the MMA's commit at the end of a tile, to both epilogues;
//   acc_empty[b] leader only: 8 epilogue warps of each CTA arrive (the peer's remotely);
//   mma_done    leader: every MMA complete before TMEM is released.
// A cluster barrier follows barrier initialisation (before any cross-CTA use) and precedes
// TMEM release and exit (the leader's MMAs read the peer's shared memory and write its
// TMEM; the peer's epilogue arrives on the leader's barriers).  Every wait is bounded.
#pragma once
#include "kernels_crt.cuh"

namespace xtg {
namespace crt2 {

using crt::BK;
using crt::EPI_WARPS;
using crt::MAXL;
using crt::Params;
using crt::THREADS;
constexpr int TM = 256;                   // rows of C per pair tile (MMA N)
constexpr int TNP = 256;                  // columns of C per pair tile (MMA M; 128 per CTA)
constexpr int HALF = 128;                 // rows / columns held per CTA
constexpr int STAGES = 12;
constexpr int ROW_TILE = HALF * BK;       // 8 KB: this CTA's 128 of the tile's rows
constexpr int COL_TILE = HALF * BK;       // 8 KB: this CTA's 128 columns
constexpr int STAGE_BYTES = ROW_TILE + COL_TILE;
constexpr int SMEM_BYTES = STAGES * STAGE_BYTES + 1024;
// S8 x S8 -> S32, K-major, M = 256 (pair), N = 256
constexpr uint32_t IDESC = (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(TM >> 3) << 17) |
                           ((uint32_t)(TNP >> 4) << 24);

__device__ __forceinline__ uint32_t cluster_rank()
{
    uint32_t r;
    asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
    return r;
}
// shared::cluster address of the same shared-memory offset in CTA `rank` of the cluster
__device__ __forceinline__ uint32_t map_to_rank(const void *p, uint32_t rank)
{
    uint32_t r;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(split::smem_u32(p)), "r"(rank));
    return r;
}
__device__ __forceinline__ void cluster_sync()
{
    asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}
// arrive on the barrier at cluster address `a` (possibly in the peer CTA)
__device__ __forceinline__ void mbar_arrive_cluster(uint32_t a)
{
    asm volatile("mbarrier.arrive.shared::cluster.b64 _, [%0];" ::"r"(a) : "memory");
}
// TMA 2-D load into this CTA's shared memory, completing on the barrier at cluster address
// `bar` (the leader's)
__device__ __forceinline__ void tma_load_2d_pair(void *dst, const CUtensorMap *map, int x, int y, uint32_t bar)
{
    asm volatile(
        "cp.async.bulk.tensor.2d.cta_group::2.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], "
        "[%4];" ::"r"(split::smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(bar)
        : "memory");
}
__device__ __forceinline__ void umma_pair_i8(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t accumulate)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::2.kind::i8 [%0], %1, %2, %3, p;\n\t}"
        ::"r"(tmem_d), "l"(adesc), "l"(bdesc), "r"(IDESC), "r"(accumulate));
}
// arrive (once the MMAs issued so far complete) on the barrier at this offset in both CTAs
__device__ __forceinline__ void umma_commit_pair(uint64_t *bar)
{
    asm volatile(
        "tcgen05.commit.cta_group::2.mbarrier::arrive::one.shared::cluster.multicast::cluster.b64 [%0], %1;" ::"r"(
            split::smem_u32(bar)),
        "h"((uint16_t)3)
        : "memory");
}

__device__ __forceinline__ void pair_item_tile(const Params &p, int item, int &l, int &m0, int &n0, int &ksteps)
{
    const int per = p.mtiles * p.ntiles;
    l = item / per;
    const int r = item - l * per;
    const int nt = r / p.mtiles;
    m0 = (r - nt * p.mtiles) * TM;
    n0 = (p.kext ? p.ntiles - 1 - nt : nt) * TNP;  // longest column tiles first (back-transform)
    int kmax = p.Kp;
    if (p.kext) kmax = min(kmax, p.kext[min(n0 + TNP, p.N) - 1]);
    ksteps = max(1, (kmax + BK - 1) / BK);
}

// Grid: pairs of CTAs (cluster dims 2), persistent over items; p.mtiles = Mp / 256,
// p.ntiles = Np / 256.  tmR: A residues (rows l Mp + m), tmC: B residues (rows l Np + n), boxes
// of 128 rows.
__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(THREADS, 1)
    gemm_crt2_kernel(const __grid_constant__ CUtensorMap tmR, const __grid_constant__ CUtensorMap tmC, Params p)
{
    extern __shared__ __align__(16) unsigned char smem_crt2[];
    unsigned char *base = reinterpret_cast<unsigned char *>(((uintptr_t)smem_crt2 + 1023) & ~(uintptr_t)1023);
    unsigned char *sR = base;                      // [STAGES][ROW_TILE]
    unsigned char *sC = base + STAGES * ROW_TILE;  // [STAGES][COL_TILE]
    __shared__ __align__(8) uint64_t full[STAGES], empty[STAGES], acc_full[2], acc_empty[2], mma_done;
    __shared__ uint32_t tmem_base;
    __shared__ volatile int abort_flag;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t rank = cluster_rank();
    const bool leader = rank == 0;
    const int pair = blockIdx.x >> 1, npairs = gridDim.x >> 1;
    if (threadIdx.x == 0) {
        abort_flag = 0;
        for (int q = 0; q < STAGES; q++) {
            split::mbar_init(&full[q], 1);
            split::mbar_init(&empty[q], 1);
        }
        for (int q = 0; q < 2; q++) {
            split::mbar_init(&acc_full[q], 1);
            split::mbar_init(&acc_empty[q], 2 * EPI_WARPS);
        }
        split::mbar_init(&mma_done, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1) {  // TMEM of the pair: two accumulators of 256 columns in each CTA
        asm volatile("tcgen05.alloc.cta_group::2.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         split::smem_u32(&tmem_base)),
                     "r"(512));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::2.sync.aligned;");
    }
    split::tc_fence_before();
    __syncthreads();
    cluster_sync();  // both CTAs' barriers initialised before any cross-CTA arrive or load
    split::tc_fence_after();
    const uint32_t tmem = tmem_base;

    if (warp == 0) {
        // ---------------- TMA producer (both CTAs) ----------------
        if (lane == 0) {
            long long use = 0;
            for (int item = pair; item < p.items && !abort_flag; item += npairs) {
                int l, m0, n0, ks;
                pair_item_tile(p, item, l, m0, n0, ks);
                bool ok = true;
                for (int k = 0; k < ks; k++, use++) {
                    const int s = (int)(use % STAGES);
                    if (use >= STAGES &&
                        !split::mbar_wait(&empty[s], (uint32_t)(((use / STAGES) - 1) & 1), &abort_flag, p.err)) {
                        ok = false;
                        break;
                    }
                    if (leader) split::mbar_expect_tx(&full[s], (uint32_t)(2 * STAGE_BYTES));
                    const uint32_t bar = map_to_rank(&full[s], 0);
                    tma_load_2d_pair(sR + s * ROW_TILE, &tmR, k * BK, l * p.Mp + m0 + (int)rank * HALF, bar);
                    tma_load_2d_pair(sC + s * COL_TILE, &tmC, k * BK, l * p.Np + n0 + (int)rank * HALF, bar);
                }
                if (!ok) break;
            }
            if (abort_flag) {
                if (leader) {
                    // the loads of both CTAs complete on the leader's barriers: wait (bounded)
                    // for the latest phase of every stage filled
                    for (int s = 0; s < STAGES; s++) {
                        const long long fills = use / STAGES + (s < use % STAGES ? 1 : 0);
                        if (fills) split::mbar_drain(&full[s], (uint32_t)((fills - 1) & 1));
                    }
                } else {
                    // the peer cannot observe its loads (they complete on the leader's
                    // barriers): give those in flight ~200 us to land
                    for (int q = 0; q < 2000; q++) __nanosleep(100);
                }
            }
        }
    } else if (warp == 1) {
        // ---------------- MMA issue (leader) ----------------
        if (leader && lane == 0) {
            long long use = 0;
            int tcount = 0;
            bool ok = true;
            for (int item = pair; item < p.items && ok; item += npairs, tcount++) {
                int l, m0, n0, ks;
                pair_item_tile(p, item, l, m0, n0, ks);
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
                    for (int kk = 0; kk < 2; kk++)
                        umma_pair_i8(dcol, split::smem_desc(sC + s * COL_TILE, kk * 32),
                                     split::smem_desc(sR + s * ROW_TILE, kk * 32), (k | kk) ? 1u : 0u);
                    umma_commit_pair(&empty[s]);
                }
                if (ok) umma_commit_pair(&acc_full[buf]);
            }
            asm volatile("tcgen05.commit.cta_group::2.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                             split::smem_u32(&mma_done))
                         : "memory");
            split::mbar_drain(&mma_done, 0);
        }
    } else {
        // ---------------- epilogue: warps 2..9 of both CTAs ----------------
        const int quad = warp & 3, half = (warp - 2) >> 2;
        int tcount = 0;
        for (int item = pair; item < p.items; item += npairs, tcount++) {
            int l, m0, n0, ks;
            pair_item_tile(p, item, l, m0, n0, ks);
            const int buf = tcount & 1;
            if (!split::mbar_wait(&acc_full[buf], (uint32_t)((tcount >> 1) & 1), &abort_flag, p.err)) break;
            split::tc_fence_after();
            const unsigned int pl = (unsigned int)p.p[l], bl = p.barrett[l];
            const int col = n0 + (int)rank * HALF + quad * 32 + lane;
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
                    w[g] = crt::mod_p((int)v[4 * g], pl, bl) | (crt::mod_p((int)v[4 * g + 1], pl, bl) << 8) |
                           (crt::mod_p((int)v[4 * g + 2], pl, bl) << 16) |
                           (crt::mod_p((int)v[4 * g + 3], pl, bl) << 24);
                uint4 *dst = reinterpret_cast<uint4 *>(Ucol + h);
                dst[0] = make_uint4(w[0], w[1], w[2], w[3]);
                dst[1] = make_uint4(w[4], w[5], w[6], w[7]);
            }
            split::tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive_cluster(map_to_rank(&acc_empty[buf], 0));
        }
    }

    split::tc_fence_before();
    __syncthreads();
    cluster_sync();  // the pair's MMAs, loads and remote arrivals are over
    if (warp == 1) {
        split::tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::2.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(512));
    }
}

}  // namespace crt2
}  // namespace xtg
