// Device algorithm of the blocked generalized-eigenvector back-substitution (xTGEVC3).
//
// Right eigenvectors of the upper quasi-triangular pencil (S, P) are computed for all
// selected eigenvalues at once with a right-looking blocked substitution over row blocks
// of kBlock rows, bottom to top:
//     for each row block I = [r0, r1):
//         diag_solve:  X[I, c] = (ac_c S_II - b_c P_II)^-1 X[I, c]  for active columns c
//         update:      X[0:r0, c] += S[0:r0, I] (-ac_c X[I, c]) + P[0:r0, I] (b_c X[I, c])
// (the upstream driver does the same per 32-column panel, src/dtgevc3.cpp:1281-1470;
// panels are independent, so all of them advance together here and every update is one
// large GEMM instead of nb_sel <= 33 columns at a time).
//
// Left eigenvectors y (y^H (b S - a P) = 0) are the right eigenvectors of the reversed
// (conjugate-)transposed pencil (F S^H F, F P^H F), F the reversal permutation, with the
// columns and rows of the result reversed back; the same code therefore serves both sides
// (upstream: src/dtgevc3.cpp:1476-1663).
//
// HOWMNY = 'B' multiplies by Z (Q) with a triangular-aware GEMM; otherwise the triangle is
// written back with zeros elsewhere.
#include "engine.cuh"
#include "kernels_diag.cuh"
#include "kernels_diag_tc.cuh"
#include "kernels_gemm.cuh"
#include "kernels_misc.cuh"
#include "kernels_split.cuh"
#include "kernels_crt.cuh"
#include "kernels_crt2.cuh"
#include "kernels_refine.cuh"
#include "host_common.cuh"

#include <cudaTypedefs.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <type_traits>
#include <vector>

namespace xtg {

static thread_local std::string g_err;
// eigenvector columns the last split-form call of this thread solved again in FP64
static thread_local int g_refined = 0;
int refined_columns() { return g_refined; }
const char *last_error() { return g_err.c_str(); }
void set_last_error(const std::string &s) { g_err = s; }


// ---- kernel trace ----------------------------------------------------------------------
namespace {
struct TraceTotals {
    long long launches = 0;
    double ms = 0, flops = 0, bytes = 0;
};
std::atomic<long long> g_launches{0};
std::atomic<int> g_trace_on{0};
std::mutex g_trace_mu;
TraceTotals g_tot[kTCount];
const char *g_trace_names[kTCount] = {"prep", "diag_solve", "gemm_update", "gemm_backtransform", "writeback",
                                      "normalize", "split_slices", "split_gemm", "split_reconstruct"};

// Brackets each kernel launch of one call with events when tracing is on; totals are
// folded in after the call's stream synchronisation.
struct Tracer {
    struct Ev {
        int cat;
        cudaEvent_t a, b;
        double flops, bytes;
    };
    std::vector<Ev> pend;
    bool on = g_trace_on.load() != 0;
    template <class F>
    void run(int cat, double flops, double bytes, cudaStream_t st, F &&launch)
    {
        g_launches.fetch_add(1);
        if (!on) {
            launch();
            return;
        }
        Ev e{cat, nullptr, nullptr, flops, bytes};
        cudaEventCreate(&e.a);
        cudaEventCreate(&e.b);
        cudaEventRecord(e.a, st);
        launch();
        cudaEventRecord(e.b, st);
        pend.push_back(e);
    }
    void flush()
    {
        std::lock_guard<std::mutex> lk(g_trace_mu);
        for (Ev &e : pend) {
            float ms = 0;
            if (cudaEventElapsedTime(&ms, e.a, e.b) == cudaSuccess) {
                TraceTotals &t = g_tot[e.cat];
                t.launches += 1;
                t.ms += ms;
                t.flops += e.flops;
                t.bytes += e.bytes;
            }
            cudaEventDestroy(e.a);
            cudaEventDestroy(e.b);
        }
        pend.clear();
    }
    ~Tracer()
    {
        for (Ev &e : pend) {
            cudaEventDestroy(e.a);
            cudaEventDestroy(e.b);
        }
    }
};
}  // namespace

const char *trace_name(int cat) { return (cat >= 0 && cat < kTCount) ? g_trace_names[cat] : ""; }
void trace_enable(int on) { g_trace_on.store(on ? 1 : 0); }
void trace_reset()
{
    std::lock_guard<std::mutex> lk(g_trace_mu);
    for (auto &t : g_tot) t = TraceTotals{};
}
int trace_get(int cat, long long *launches, double *ms, double *flops, double *bytes)
{
    if (cat < 0 || cat >= kTCount) return -1;
    std::lock_guard<std::mutex> lk(g_trace_mu);
    if (launches) *launches = g_tot[cat].launches;
    if (ms) *ms = g_tot[cat].ms;
    if (flops) *flops = g_tot[cat].flops;
    if (bytes) *bytes = g_tot[cat].bytes;
    return 0;
}
long long launch_count() { return g_launches.load(); }
void count_launches(long long k) { g_launches.fetch_add(k); }

size_t arena_bytes_needed(int n, int m, bool right, bool left, bool back, bool normalize, bool cplx, size_t rsz)
{
    auto r256 = [](size_t b) { return (std::max<size_t>(b, 1) + 255) & ~size_t(255); };
    const size_t esz = cplx ? 2 * rsz : rsz, ld = (size_t)round_up(n, 32);
    const size_t nn = (size_t)n, mm = (size_t)m;
    // eigenvalues, column sums, norms; then each side's column lists (uploaded before either
    // side starts, so they stay allocated for the whole call)
    const size_t cols = r256(sizeof(int) * 5 * mm) + r256(mm);
    const size_t shared = r256(rsz * (cplx ? 4 : 3) * nn) + r256(rsz * 2 * nn) + r256(rsz * 2) +
                          (right ? cols : 0) + (left ? cols : 0);
    auto side = [&](bool lft) {
        size_t b = 0;
        if (lft) b += 2 * r256(esz * ld * nn);
        b += r256(esz * ld * mm) + r256(esz * 4 * kBlock * mm) + r256(rsz * (cplx ? 6 : 4) * mm);
        if (back) b += r256(esz * ld * nn);
        if (normalize && !cplx) b += r256(mm);
        return b;
    };
    size_t s = 0;
    if (right) s = side(false);
    if (left) s = std::max(s, side(true));
    return shared + s;
}

static std::once_flag g_pool_once[64];
void configure_device(int dev)
{
    if (dev < 0 || dev >= 64) return;
    std::call_once(g_pool_once[dev], [dev]() {
        cudaMemPool_t pool;
        if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
            uint64_t thr = UINT64_MAX;
            cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
        }
        cudaFuncSetAttribute(diag_solve_real<double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             2 * kBlock * kSmLd * (int)sizeof(double));
        cudaFuncSetAttribute(diag_solve_real<float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             2 * kBlock * kSmLd * (int)sizeof(float));
        cudaFuncSetAttribute(diag_solve_cplx<double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             2 * kBlock * kSmLd * (int)sizeof(cplx<double>));
        cudaFuncSetAttribute(dtc::diag_solve_real_tc, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)dtc::kSmemBytes);
        cudaFuncSetAttribute(diag_solve_cplx<float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             2 * kBlock * kSmLd * (int)sizeof(cplx<float>));
        cudaFuncSetAttribute(gemm_dmma<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, dmma::Tile<128>::SMEM_BYTES);
        cudaFuncSetAttribute(gemm_dmma<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, dmma::Tile<128>::SMEM_BYTES);
        cudaFuncSetAttribute(gemm_dmma<0, 64>, cudaFuncAttributeMaxDynamicSharedMemorySize, dmma::Tile<64>::SMEM_BYTES);
        cudaFuncSetAttribute(gemm_dmma<1, 64>, cudaFuncAttributeMaxDynamicSharedMemorySize, dmma::Tile<64>::SMEM_BYTES);
        cudaFuncSetAttribute(gemm_dmma<0, 128, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, dmma::Tile<128>::SMEM_BYTES);
        cudaFuncSetAttribute(gemm_dmma<1, 128, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, dmma::Tile<128>::SMEM_BYTES);
        cudaFuncSetAttribute(gemm_dmma<0, 64, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, dmma::Tile<64>::SMEM_BYTES);
        cudaFuncSetAttribute(gemm_dmma<1, 64, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, dmma::Tile<64>::SMEM_BYTES);
        cudaFuncSetAttribute(gemm_dmma_cplx<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, zmma::SMEM_BYTES);
        cudaFuncSetAttribute(gemm_dmma_cplx<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, zmma::SMEM_BYTES);
        cudaFuncSetAttribute(split::gemm_split_kernel<split::kBF16>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             split::Layout<split::kBF16>::SMEM_BYTES);
        cudaFuncSetAttribute(split::gemm_split_kernel<split::kI8>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             split::Layout<split::kI8>::SMEM_BYTES);
        cudaFuncSetAttribute(crt::gemm_crt_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, crt::SMEM_BYTES);
        cudaFuncSetAttribute(crt2::gemm_crt2_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, crt2::SMEM_BYTES);
    });
}

// ---- reusable per-call resources -------------------------------------------------------
// A call with both sides runs the left one on a second stream, and a call on a real pencil
// in device memory copies one status word back to pinned host memory.  Creating and
// destroying a stream, its events and a pinned word per call costs tens of microseconds
// (noticeable for small pencils), so they come from a per-device pool: a call leases one
// set and returns it when it ends; sets are created on demand and kept for the process.
namespace {
struct CallRes {
    cudaStream_t side = nullptr;
    cudaEvent_t fork = nullptr, join = nullptr, check = nullptr;
    int *status = nullptr;  // pinned host word written by the structure check's copy
    uint8_t *hflags = nullptr;  // pinned refinement flags of the split form (grown on demand)
    size_t hflags_cap = 0;
    // per side: the stream and fork / join events of the refinement sketch of S and P
    // (created on first use)
    cudaStream_t sk_stream[2] = {nullptr, nullptr};
    cudaEvent_t sk_ev[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};
    cudaError_t reserve_sketch()
    {
        cudaError_t e = cudaSuccess;
        for (int s = 0; s < 2 && e == cudaSuccess; s++) {
            if (!sk_stream[s]) e = cudaStreamCreateWithFlags(&sk_stream[s], cudaStreamNonBlocking);
            for (int k = 0; k < 2 && e == cudaSuccess; k++)
                if (!sk_ev[s][k]) e = cudaEventCreateWithFlags(&sk_ev[s][k], cudaEventDisableTiming);
        }
        return e;
    }
    cudaError_t reserve_flags(size_t bytes)
    {
        if (bytes <= hflags_cap) return cudaSuccess;
        if (hflags) cudaFreeHost(hflags);
        hflags = nullptr;
        hflags_cap = 0;
        const cudaError_t e = cudaHostAlloc(reinterpret_cast<void **>(&hflags), bytes, cudaHostAllocDefault);
        if (e == cudaSuccess) hflags_cap = bytes;
        return e;
    }
};
std::mutex g_res_mu;
std::vector<CallRes *> g_res_free[64];

class ResLease {
public:
    explicit ResLease(int dev) : dev_(dev) {}
    ~ResLease()
    {
        if (r_) {
            std::lock_guard<std::mutex> lk(g_res_mu);
            g_res_free[dev_].push_back(r_);
        }
    }
    // The set of this call (created on first use, on the current device); nullptr and a
    // CUDA error code on failure.
    CallRes *get(cudaError_t *err)
    {
        *err = cudaSuccess;
        if (r_) return r_;
        if (dev_ < 0 || dev_ >= 64) {
            *err = cudaErrorInvalidDevice;
            return nullptr;
        }
        {
            std::lock_guard<std::mutex> lk(g_res_mu);
            if (!g_res_free[dev_].empty()) {
                r_ = g_res_free[dev_].back();
                g_res_free[dev_].pop_back();
                return r_;
            }
        }
        CallRes *r = new CallRes;
        cudaError_t e = cudaStreamCreateWithFlags(&r->side, cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&r->fork, cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&r->join, cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&r->check, cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaHostAlloc(reinterpret_cast<void **>(&r->status), sizeof(int), cudaHostAllocDefault);
        if (e != cudaSuccess) {
            if (r->status) cudaFreeHost(r->status);
            if (r->check) cudaEventDestroy(r->check);
            if (r->join) cudaEventDestroy(r->join);
            if (r->fork) cudaEventDestroy(r->fork);
            if (r->side) cudaStreamDestroy(r->side);
            delete r;
            *err = e;
            return nullptr;
        }
        r_ = r;
        return r_;
    }

private:
    int dev_;
    CallRes *r_ = nullptr;
};
}  // namespace

// Selected eigenvalues in ascending order; a complex-conjugate pair (real arithmetic) is
// one item of two columns.  Selection rule of src/dtgevc3.cpp:1193-1207 / 1295-1324.
struct Item {
    int k;
    bool pair;
    int out;  // first output column
};

// Per-column description of one side's computation (problem orientation).
struct ColList {
    int m = 0;
    std::vector<int> colk, src, kext, outcol;
    std::vector<uint8_t> kind;
};

// ---- split-precision GEMM launcher ---------------------------------------------------------
static PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder()
{
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, []() {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    });
    return fn;
}

// 2-D tensor map over a row-major [rows][cols] slice buffer: 64-byte swizzled boxes of one
// 64-byte K row (32 BF16 or 64 INT8 elements) by box_rows rows.
static bool slice_tensor_map(CUtensorMap *m, const void *base, int kind, int cols, int rows, int box_rows)
{
    auto enc = tensor_map_encoder();
    if (!enc) return false;
    const int esz = kind == split::kI8 ? 1 : 2;
    cuuint64_t dims[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
    cuuint64_t strides[1] = {(cuuint64_t)cols * esz};
    cuuint32_t box[2] = {(cuuint32_t)(64 / esz), (cuuint32_t)box_rows};
    cuuint32_t es[2] = {1, 1};
    return enc(m, kind == split::kI8 ? CU_TENSOR_MAP_DATA_TYPE_UINT8 : CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2,
               const_cast<void *>(base), dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
               CU_TENSOR_MAP_SWIZZLE_64B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// Reusable slice buffers of one side (grown on demand from the call's scratch).
struct SplitBufs {
    unsigned char *A = nullptr, *B = nullptr;
    int *ea = nullptr, *eb = nullptr;
    size_t acap = 0, bcap = 0, ecap_a = 0, ecap_b = 0;
};

// C (+)= A B for a GemmArgs<double> launch, through s slices of kind KIND on the tensor
// cores (see kernels_split.cuh).  Returns a CUDA error code (cudaSuccess on success).
template <int KIND>
static cudaError_t launch_split(const GemmArgs<double> &g, int s, SplitBufs &sb, Scratch &scr, int *d_err,
                                cudaStream_t st)
{
    using namespace split;
    using Elem = typename Cfg<KIND>::Elem;
    constexpr int KBK = Cfg<KIND>::BK, KBN = Cfg<KIND>::BN;
    const int Kp = round_up(g.K, KBK), Mp = round_up(g.M, BM), Np = round_up(g.N, KBN);
    const size_t an = (size_t)s * Mp * Kp * sizeof(Elem), bn = (size_t)s * Np * Kp * sizeof(Elem);
    if (an > sb.acap) { sb.A = scr.get<unsigned char>(an); sb.acap = an; }
    if (bn > sb.bcap) { sb.B = scr.get<unsigned char>(bn); sb.bcap = bn; }
    if ((size_t)Mp > sb.ecap_a) { sb.ea = scr.get<int>(Mp); sb.ecap_a = Mp; }
    if ((size_t)Np > sb.ecap_b) { sb.eb = scr.get<int>(Np); sb.ecap_b = Np; }
    if (scr.err) return scr.err;
    slice_rows_kernel<KIND><<<Mp / 32, 256, 0, st>>>(g, Kp, Mp, s, reinterpret_cast<Elem *>(sb.A), sb.ea);
    slice_cols_kernel<KIND><<<Np / 8, 256, 0, st>>>(g, Kp, Np, s, reinterpret_cast<Elem *>(sb.B), sb.eb);
    CUtensorMap tmA, tmB;
    if (!slice_tensor_map(&tmA, sb.A, KIND, Kp, s * Mp, BM) || !slice_tensor_map(&tmB, sb.B, KIND, Kp, s * Np, KBN))
        return cudaErrorInvalidValue;
    Params p;
    p.M = g.M;
    p.N = g.N;
    p.Kp = Kp;
    p.s = s;
    p.Mp = Mp;
    p.Np = Np;
    p.mlo = g.mlo;
    p.accumulate = g.accumulate;
    p.ea = sb.ea;
    p.eb = sb.eb;
    p.kext = g.kext;
    p.C = g.C;
    p.ldc = g.ldc;
    p.ccol = g.ccol;
    p.err = d_err;
    gemm_split_kernel<KIND><<<dim3(Mp / BM, Np / KBN), THREADS, Layout<KIND>::SMEM_BYTES, st>>>(tmA, tmB, p);
    return cudaGetLastError();
}

// ---- residue (CRT) split GEMM launcher ------------------------------------------------------
// Moduli of the residue form: pairwise coprime, largest first (256 = 2^8, 255 = 3 5 17,
// 253 = 11 23, 247 = 13 19, 217 = 7 31, the rest prime); the first L are used.
static const int kModuli[crt::MAXL] = {256, 255, 253, 251, 247, 241, 239, 233, 229, 227, 223, 217, 211, 199, 197, 193};

static void build_moduli(crt::Moduli &md, int L)
{
    typedef unsigned __int128 u128;
    md = crt::Moduli{};
    md.L = L;
    u128 P = 1;
    for (int l = 0; l < L; l++) P *= (u128)kModuli[l];
    int bits = 0;  // bits of P (every weight W_l < P)
    for (u128 v = P; v; v >>= 1) bits++;
    md.hi = std::max(0, bits - 41);
    md.lo = std::max(0, md.hi - 41);
    const u128 mask_mid = (((u128)1) << (md.hi - md.lo)) - 1;  // bits [lo, hi) of W_l and P
    for (int l = 0; l < L; l++) {
        const int p = kModuli[l];
        const u128 Ml = P / (u128)p;
        const int r = (int)(Ml % (u128)p);
        int y = 1;
        while ((r * y) % p != 1) y++;  // the inverse exists: the moduli are pairwise coprime
        const u128 W = Ml * (u128)y;  // < Ml p = P (y < p): the weight is already reduced mod P
        md.p[l] = p;
        md.barrett[l] = (unsigned int)((((unsigned long long)1) << 32) / (unsigned long long)p);
        md.invp[l] = 1.0 / (double)p;
        md.pd[l] = (double)p;
        md.w1[l] = (double)(W >> md.hi);
        md.w2[l] = (double)((W >> md.lo) & mask_mid);
    }
    md.P1 = (double)(P >> md.hi);
    md.P2 = (double)((P >> md.lo) & mask_mid);
    const double Pd = (double)P;
    md.c1 = std::ldexp(1.0, md.hi) / Pd;
    md.c2 = std::ldexp(1.0, md.lo) / Pd;
    md.log2P = std::log2(Pd);
}

static const crt::Moduli &crt_moduli(int L)
{
    static crt::Moduli tab[crt::MAXL + 1];
    static std::once_flag once;
    std::call_once(once, [] {
        for (int l = 1; l <= crt::MAXL; l++) build_moduli(tab[l], l);
    });
    return tab[std::max(1, std::min(L, crt::MAXL))];
}

// Operand bits t of a residue GEMM with L moduli and K terms: 2t + ceil(log2 K) + 2 <= log2 P,
// so that |C'| < P / 4 and the rounded quotient of the reconstruction is exact.
static int crt_bits(int L, int K)
{
    int kb = 0;
    while ((1 << kb) < std::max(K, 2)) kb++;
    // at most 50: the residue kernels round v 2^t against 1.5 2^52, exact for |a| < 2^51
    return std::min(50, (int)std::floor((crt_moduli(L).log2P - kb - 2) / 2));
}

// Reusable residue buffers of one side (grown on demand from the call's scratch).
struct CrtBufs {
    int8_t *A = nullptr, *B = nullptr;
    unsigned char *U = nullptr;
    int *ea = nullptr, *eb = nullptr;
    unsigned long long *rmax = nullptr;
    size_t acap = 0, bcap = 0, ucap = 0, eacap = 0, ebcap = 0, rcap = 0;
    // what B and eb hold: the operand and shape of the launch that wrote them
    const void *b_src = nullptr;
    int b_Kp = 0, b_Np = 0, b_L = 0, b_t = 0;
};

static int sm_count()
{
    int dev = 0, nsm = 148;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    return std::max(1, nsm);
}

// C (+)= A B for a GemmArgs<double> launch by L residues on the INT8 tensor cores (see
// kernels_crt.cuh).  K must stay below 2^16 (exact INT32 sums; the caller checks).
// The residue GEMM runs on one CTA per SM (kernels_crt.cuh); XTGEVC3_CRT_PAIR=1 selects the
// SM-pair kernel (kernels_crt2.cuh: a third less operand traffic per SM, measured slower on
// this solver's shapes).  Pairs resident at once come from the occupancy API (cached per device).
// Row blocks per group of the split forms' blocked substitution (one trailing GEMM per
// group, K = 2 x the group's rows); XTGEVC3_SPLIT_GROUP (1..32) overrides the default for
// tuning, read once per process.
static int split_group_blocks()
{
    static const int g = [] {
        const char *v = std::getenv("XTGEVC3_SPLIT_GROUP");
        const int x = v ? std::atoi(v) : 0;
        return (x >= 1 && x <= 32) ? x : kGroupBlocksSplit;
    }();
    return g;
}

static bool crt_pairs()
{
    static const bool on = [] {
        const char *v = std::getenv("XTGEVC3_CRT_PAIR");
        return v && v[0] == '1';
    }();
    return on;
}
static int crt_pair_grid()
{
    static int cached[64] = {};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 2 * (sm_count() / 2);
    if (!cached[dev]) {
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(2 * (sm_count() / 2));
        cfg.blockDim = dim3(crt::THREADS);
        cfg.dynamicSmemBytes = crt2::SMEM_BYTES;
        int clusters = 0;
        if (cudaOccupancyMaxActiveClusters(&clusters, crt2::gemm_crt2_kernel, &cfg) != cudaSuccess || clusters <= 0) {
            cudaGetLastError();
            clusters = sm_count() / 2;
        }
        cached[dev] = 2 * clusters;
    }
    return cached[dev];
}

static cudaError_t launch_crt(const GemmArgs<double> &g, int L, CrtBufs &cb, Scratch &scr, int *d_err,
                              cudaStream_t st, Tracer *tr = nullptr, double flops = 0)
{
    auto run = [&](int cat, double fl, double by, auto &&f) {
        if (tr) tr->run(cat, fl, by, st, f);
        else f();
    };
    using namespace crt;
    const Moduli &md = crt_moduli(L);
    const bool pairs = crt_pairs();
    const int Kp = round_up(g.K, BK), Mp = round_up(g.M, TM), Np = round_up(g.N, pairs ? crt2::TNP : TN);
    const int t = crt_bits(L, g.K);
    const size_t an = (size_t)L * Mp * Kp, bn = (size_t)L * Np * Kp, un = (size_t)L * Np * Mp;
    if (an > cb.acap) { cb.A = scr.get<int8_t>(an); cb.acap = an; }
    if (bn > cb.bcap) { cb.B = scr.get<int8_t>(bn); cb.bcap = bn; cb.b_src = nullptr; }
    if (un > cb.ucap) { cb.U = scr.get<unsigned char>(un); cb.ucap = un; }
    if ((size_t)Mp > cb.eacap) { cb.ea = scr.get<int>(Mp); cb.eacap = Mp; }
    if ((size_t)Np > cb.ebcap) { cb.eb = scr.get<int>(Np); cb.ebcap = Np; cb.b_src = nullptr; }
    if ((size_t)(Mp + Np) > cb.rcap) { cb.rmax = scr.get<unsigned long long>(Mp + Np); cb.rcap = Mp + Np; }
    if (scr.err) return scr.err;
    unsigned long long *cmax = cb.rmax + Mp;
    cudaError_t e = cudaMemsetAsync(cb.rmax, 0, (size_t)(Mp + Np) * sizeof(unsigned long long), st);
    if (e != cudaSuccess) return e;
    // operand bytes: A and B read twice (maximum, residues), L residue bytes written per entry
    const double slice_bytes = ((double)g.M + g.N) * g.K * (2.0 * 8 + L);
    // B's residues stay valid across the row panels of one back-transform (same B, shape and
    // bits): only the first panel computes them
    const bool keep_b = g.reuse_b && cb.b_src == (const void *)g.B && cb.b_Kp == Kp && cb.b_Np == Np &&
                        cb.b_L == L && cb.b_t == t;
    run(kTSplitPrep, 0, slice_bytes, [&] {
        row_absmax_kernel<<<dim3(Mp / 32, (g.K + 255) / 256), 256, 0, st>>>(g, cb.rmax);
        if (!keep_b) col_absmax_kernel<<<dim3(Np / 32, Kp / 64), 256, 0, st>>>(g, cmax);
        const dim3 gr(Mp / 32, Kp / 64), gc(Np / 32, Kp / 64);
        const int tnw = pairs ? crt2::TNP : TN;
        if (L == 14) {  // the default modulus count: moduli at fixed offsets
            residue_rows_kernel<14><<<gr, 256, 0, st>>>(g, Kp, Mp, t, md, cb.rmax, cb.A, cb.ea);
            if (!keep_b) residue_cols_kernel<14><<<gc, 256, 0, st>>>(g, Kp, Np, tnw, t, md, cmax, cb.B, cb.eb);
        } else {
            residue_rows_kernel<0><<<gr, 256, 0, st>>>(g, Kp, Mp, t, md, cb.rmax, cb.A, cb.ea);
            if (!keep_b) residue_cols_kernel<0><<<gc, 256, 0, st>>>(g, Kp, Np, tnw, t, md, cmax, cb.B, cb.eb);
        }
    });
    cb.b_src = g.B;
    cb.b_Kp = Kp;
    cb.b_Np = Np;
    cb.b_L = L;
    cb.b_t = t;
    CUtensorMap tmA, tmB;
    if (!slice_tensor_map(&tmA, cb.A, split::kI8, Kp, L * Mp, pairs ? crt2::HALF : TM) ||
        !slice_tensor_map(&tmB, cb.B, split::kI8, Kp, L * Np, pairs ? crt2::HALF : TN))
        return cudaErrorInvalidValue;
    Params p;
    p.M = g.M;
    p.N = g.N;
    p.Kp = Kp;
    p.Mp = Mp;
    p.Np = Np;
    p.L = L;
    p.mtiles = Mp / TM;
    p.ntiles = Np / (pairs ? crt2::TNP : TN);
    p.items = L * p.mtiles * p.ntiles;
    p.kext = g.kext;
    p.U = cb.U;
    p.err = d_err;
    for (int l = 0; l < MAXL; l++) {
        p.p[l] = md.p[l];
        p.barrett[l] = md.barrett[l];
    }
    // residue bytes: both operands read once, one byte per output entry and modulus written
    const double gemm_bytes = (double)L * ((double)Mp * Kp + (double)Np * Kp + (double)Mp * Np);
    if (pairs) {
        const int grid = std::min(crt_pair_grid(), 2 * p.items);  // persistent pairs of CTAs
        run(kTSplitGemm, flops, gemm_bytes,
            [&] { crt2::gemm_crt2_kernel<<<grid, THREADS, crt2::SMEM_BYTES, st>>>(tmA, tmB, p); });
    } else {
        const int grid = std::min(sm_count(), p.items);  // persistent: one CTA per SM
        run(kTSplitGemm, flops, gemm_bytes,
            [&] { gemm_crt_kernel<<<grid, THREADS, SMEM_BYTES, st>>>(tmA, tmB, p); });
    }
    // residues in, C (read when accumulating) and out
    const double crt_bytes = (double)(g.M - g.mlo) * g.N * (L + 8.0 * (1 + g.accumulate));
    run(kTSplitCrt, 0, crt_bytes, [&] {
        const dim3 grid((g.M + 1023) / 1024, g.N);
        if (L == 14)
            crt_kernel<14><<<grid, 256, 0, st>>>(cb.U, Mp, Np, md, t, cb.ea, cb.eb, g.M, g.N, g.mlo, g.C, g.ldc, g.ccol,
                                                 g.accumulate);
        else
            crt_kernel<0><<<grid, 256, 0, st>>>(cb.U, Mp, Np, md, t, cb.ea, cb.eb, g.M, g.N, g.mlo, g.C, g.ldc, g.ccol,
                                                g.accumulate);
    });
    return cudaGetLastError();
}

int split_gemm_device(int kind, int slices, int M, int N, int K, const double *A, int lda, const double *B, int ldb,
                      double *C, int ldc, int accumulate, cudaStream_t st)
{
    if (M <= 0 || N <= 0 || K <= 0) return 0;
    if (K >= (1 << 16)) {
        set_last_error("split GEMM: K must be below 65536");
        return -1;
    }
    int dev = 0;
    XTG_CK(cudaGetDevice(&dev));
    configure_device(dev);
    Scratch scr(st);
    int *d_err = scr.get<int>(1);
    if (scr.err) { set_last_error(cudaGetErrorString(scr.err)); return 1; }
    XTG_CK(cudaMemsetAsync(d_err, 0, sizeof(int), st));
    GemmArgs<double> g{};
    g.M = M;
    g.N = N;
    g.mlo = 0;
    g.nseg = 1;
    g.seg[0].A = A;
    g.seg[0].lda = lda;
    g.seg[0].acols = K;
    g.seg[0].K = round_up(K, kKPad);
    g.seg[0].boff = 0;
    g.K = g.seg[0].K;
    g.B = B;
    g.ldb = ldb;
    g.brows = K;
    g.C = C;
    g.ldc = ldc;
    g.ccol = nullptr;
    g.kext = nullptr;
    g.accumulate = accumulate;
    cudaError_t e;
    if (kind == 2) {
        CrtBufs cb;
        e = launch_crt(g, std::max(2, std::min(slices, crt::MAXL)), cb, scr, d_err, st);
    } else {
        SplitBufs sb;
        e = kind == 1 ? launch_split<split::kI8>(g, std::max(1, std::min(slices, 7)), sb, scr, d_err, st)
                      : launch_split<split::kBF16>(g, std::max(1, std::min(slices, 6)), sb, scr, d_err, st);
    }
    if (e != cudaSuccess) {
        set_last_error(std::string("split GEMM launch: ") + cudaGetErrorString(e));
        return 1;
    }
    XTG_CK(cudaStreamSynchronize(st));
    int h_err = 0;
    XTG_CK(cudaMemcpy(&h_err, d_err, sizeof(int), cudaMemcpyDeviceToHost));
    if (h_err) {
        set_last_error("split GEMM: a bounded wait in the tensor-core pipeline expired");
        return 1;
    }
    return 0;
}

template <class R, bool CPLX>
int solve_device(char side, char howmny, const int *select, int n, const void *S_, int lds, const void *P_,
                 int ldp, const void *alpha_, const void *alphai_, const void *beta_, void *VL_, int ldvl,
                 void *VR_, int ldvr, int m_total, const Options &opt, cudaStream_t st)
{
    using E = typename std::conditional<CPLX, cplx<R>, R>::type;
    const E *S = static_cast<const E *>(S_);
    const E *P = static_cast<const E *>(P_);
    E *VL = static_cast<E *>(VL_);
    E *VR = static_cast<E *>(VR_);
    const bool want_r = (side == 'R' || side == 'B') && VR;
    const bool want_l = (side == 'L' || side == 'B') && VL;
    const bool do_back = howmny == 'B';
    const bool do_all = howmny == 'A' || howmny == 'B';
    if (n <= 0 || m_total <= 0 || (!want_r && !want_l)) return 0;

    int dev = 0;
    XTG_CK(cudaGetDevice(&dev));
    configure_device(dev);
    XTG_CK(cudaGetLastError());

    // ---- host-side structure: selection items, 2x2 blocks --------------------------------
    const R *alphai = static_cast<const R *>(alphai_);
    std::vector<Item> items;
    std::vector<char> pairstart(n + 1, 0);
    {
        int out = 0;
        for (int k = 0; k < n;) {
            bool pair = !CPLX && alphai[k] != R(0) && k + 1 < n;
            bool sel = do_all;
            if (!do_all && select) {
                sel = select[k] != 0;
                if (pair) sel = sel || select[k + 1] != 0;
            }
            if (pair) pairstart[k] = 1;
            if (sel) {
                items.push_back({k, pair, out});
                out += pair ? 2 : 1;
            }
            k += pair ? 2 : 1;
        }
        if (out != m_total) {
            set_last_error("internal: selection count mismatch");
            return 1;
        }
    }
    ResLease res(dev);
    std::vector<char> sub(n, 0);  // sub[k] = S[k+1, k] != 0
    // device check of a plan made from alphai alone (see Options::read_sub)
    bool check_sub = false;
    if constexpr (!CPLX) {
        if (n > 1 && opt.host_S) {  // the caller's copy (the device one may still be in flight)
            const E *hs = static_cast<const E *>(opt.host_S);
            for (int k = 0; k + 1 < n; k++) sub[k] = hs[(size_t)(k + 1) + (size_t)k * opt.host_lds] != E(0);
        } else if (n > 1 && (opt.read_sub || opt.arena)) {
            std::vector<E> d(n - 1);
            XTG_CK(cudaMemcpy2DAsync(d.data(), sizeof(E), S + 1, (size_t)(lds + 1) * sizeof(E), sizeof(E), n - 1,
                                     cudaMemcpyDeviceToHost, st));
            XTG_CK(cudaStreamSynchronize(st));
            for (int k = 0; k + 1 < n; k++) sub[k] = d[k] != E(0);
        } else if (n > 1) {
            check_sub = true;
        }
    }

    Scratch scr = opt.arena ? Scratch(st, opt.arena, opt.arena_bytes) : Scratch(st);
    Tracer tr;
    const double esz = sizeof(E), cfl = CPLX ? 4.0 : 1.0;
    // eigenvalue data on the device (for the coefficient kernels)
    const int ncoef = CPLX ? 6 : 4;
    R *d_eig = scr.get<R>(CPLX ? 4 * (size_t)n : 3 * (size_t)n);
    R *d_sums = scr.get<R>(2 * (size_t)n);
    R *d_norms = scr.get<R>(2);
    // split-precision GEMMs: real double only; their bounded waits report through d_err
    const int split_max = opt.split_kind == 2 ? crt::MAXL
                          : opt.split_kind == split::kI8 ? split::Cfg<split::kI8>::MAXS
                                                          : split::Cfg<split::kBF16>::MAXS;
    const int nsplit = (!CPLX && std::is_same<R, double>::value && opt.split > 0) ? std::min(opt.split, split_max)
                                                                                 : 0;
    int *d_err = nsplit ? scr.get<int>(1) : nullptr;
    if (scr.err) { set_last_error(cudaGetErrorString(scr.err)); return 1; }
    if (d_err) XTG_CK(cudaMemsetAsync(d_err, 0, sizeof(int), st));
    // standard problem (xTREVC3): P = I, built here; the solves and the norms read it
    if (opt.p_identity) {
        const int ldi = round_up(n, 32);
        E *Pid = scr.get<E>((size_t)ldi * n);
        if (scr.err) { set_last_error(cudaGetErrorString(scr.err)); return 1; }
        XTG_CK(cudaMemsetAsync(Pid, 0, (size_t)ldi * n * sizeof(E), st));
        identity_diag_kernel<E><<<(n + 255) / 256, 256, 0, st>>>(Pid, ldi, n);
        XTG_CK(cudaGetLastError());
        P = Pid;
        ldp = ldi;
    }
    if (CPLX) {
        XTG_CK(cudaMemcpyAsync(d_eig, alpha_, 2 * n * sizeof(R), cudaMemcpyHostToDevice, st));
        XTG_CK(cudaMemcpyAsync(d_eig + 2 * n, beta_, 2 * n * sizeof(R), cudaMemcpyHostToDevice, st));
    } else {
        XTG_CK(cudaMemcpyAsync(d_eig, alpha_, n * sizeof(R), cudaMemcpyHostToDevice, st));
        XTG_CK(cudaMemcpyAsync(d_eig + n, alphai_, n * sizeof(R), cudaMemcpyHostToDevice, st));
        XTG_CK(cudaMemcpyAsync(d_eig + 2 * n, beta_, n * sizeof(R), cudaMemcpyHostToDevice, st));
    }
    // The row blocks below are planned from alphai (pairstart); S's subdiagonal is checked
    // against that plan on the device, and the result reaches the host through the leased
    // pinned word.  `gate` (before anything is written to VL / VR) waits for it: a mismatch
    // abandons the call, which then runs again with the subdiagonal read back.
    CallRes *cres = nullptr;
    int gate_state = check_sub ? 0 : 1;  // 0 pending, 1 plan confirmed, 2 plan rejected
    if (check_sub) {
        cudaError_t e = cudaSuccess;
        cres = res.get(&e);
        XTG_CK(e);
        uint8_t *d_ps = scr.get<uint8_t>((size_t)n);
        int *d_flag = scr.get<int>(1);
        if (scr.err) { set_last_error(cudaGetErrorString(scr.err)); return 1; }
        std::vector<uint8_t> ps(pairstart.begin(), pairstart.begin() + n);
        XTG_CK(cudaMemcpyAsync(d_ps, ps.data(), n, cudaMemcpyHostToDevice, st));
        XTG_CK(cudaMemsetAsync(d_flag, 0, sizeof(int), st));
        subdiag_check_kernel<R><<<(n + 255) / 256, 256, 0, st>>>(reinterpret_cast<const R *>(S), lds, n, d_ps, d_flag);
        XTG_CK(cudaGetLastError());
        XTG_CK(cudaMemcpyAsync(cres->status, d_flag, sizeof(int), cudaMemcpyDeviceToHost, st));
        XTG_CK(cudaEventRecord(cres->check, st));
    }
    auto gate = [&]() -> int {  // 0: go on, 1: CUDA error, 2: plan rejected
        if (gate_state == 0) {
            XTG_CK(cudaEventSynchronize(cres->check));
            gate_state = *cres->status ? 2 : 1;
        }
        return gate_state == 1 ? 0 : 2;
    };

    // anorm / bnorm (src/dtgevc3.cpp:1254-1270; complex: rows <= col only); with host_norms
    // they come from the caller after `staged` (below)
    if (!opt.host_norms) {
        tr.run(kTPrep, 0, (double)n * (n + 1) * esz, st, [&] {
            colsum_kernel<E, R><<<(n + 7) / 8, 256, 0, st>>>(S, lds, P, ldp, n, CPLX ? 0 : 1, d_sums);
        });
        tr.run(kTPrep, 0, 2.0 * n * sizeof(R), st, [&] { colmax_kernel<R><<<1, 1024, 0, st>>>(d_sums, n, d_norms); });
        XTG_CK(cudaGetLastError());
    }

    // diagonal-solve launches: one warp per eigenvector, as many CTAs as stay resident
    const int diag_threads = CPLX ? kDiagThreadsCplx : 256, diag_warps = diag_threads / 32;
    int diag_ctas = 2 * 148;
    {
        int nsm = 0, occ = 0;
        const size_t dsm = 2 * kBlock * kSmLd * sizeof(E);
        cudaError_t e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
        if (e == cudaSuccess) {
            if constexpr (CPLX) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, diag_solve_cplx<R>, diag_threads, dsm);
            else e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, diag_solve_real<R>, diag_threads, dsm);
        }
        if (e == cudaSuccess && nsm > 0 && occ > 0) diag_ctas = nsm * occ;
        XTG_CK(cudaGetLastError());
    }
    const R safemin = limits<R>::safemin, eps = limits<R>::eps;
    const R bignum = R(1) / (safemin / eps);
    const int ld_n = round_up(n, 32);

    // Real double solves with their in-block updates on the FP64 tensor cores
    // (kernels_diag_tc.cuh) with XTGEVC3_DIAG_TC=1, outside arena mode (fixed scratch).  Off
    // by default: the solves are bound by each launch's latency (one eigenvector's chain of
    // 64 dependent row steps), and the eight-column form's per-warp chain is longer (n = 8192
    // B/B: 14.4 ms per call against 9.5 ms for the one-eigenvector-per-warp kernel).
    bool diag_tc = false;
    if constexpr (!CPLX && std::is_same<R, double>::value) {
        const char *v = std::getenv("XTGEVC3_DIAG_TC");
        diag_tc = !opt.arena && v && v[0] == '1';
    }

    // ---- column lists of each side (problem orientation) and their device copies ------------
    // Both sides' lists go to the device on the call's stream before either side starts, so
    // that every host-to-device copy of the call's own is queued before `opt.staged` runs.
    struct SideCols {
        ColList L;
        std::vector<int> starts;  // columns that start an eigenvector (diagonal-solve items)
        const int *d_ints = nullptr;  // colk, src, kext, outcol, starts: m ints each
        const uint8_t *d_kind = nullptr;
        // slots of the tensor-core diagonal solves: a pair's two columns, or up to two
        // consecutive real columns; slot_k: eigenvalue index of each slot's last column
        std::vector<int> slot_k;
        const int2 *d_slots = nullptr;
        int nslots = 0;
    };
    // keep_k (optional): only the eigenvalues k with keep_k[k] set (their output columns kept)
    auto build_cols = [&](bool left, SideCols &sc, const std::vector<char> *keep_k = nullptr) -> int {
        ColList &L = sc.L;
        int m = m_total;
        if (keep_k) {
            m = 0;
            for (const Item &it : items)
                if ((*keep_k)[it.k]) m += it.pair ? 2 : 1;
        }
        L.m = m;
        L.colk.resize(m);
        L.src.resize(m);
        L.kext.resize(m);
        L.outcol.resize(m);
        L.kind.resize(m);
        int c = 0;
        auto emit = [&](const Item &it) {
            if (keep_k && !(*keep_k)[it.k]) return;
            int kk = left ? (it.pair ? n - 2 - it.k : n - 1 - it.k) : it.k;
            int w = it.pair ? 2 : 1;
            for (int q = 0; q < w; q++) {
                L.colk[c] = kk;
                L.src[c] = it.k;
                L.kext[c] = kk + w;
                L.outcol[c] = it.out + q;
                L.kind[c] = it.pair ? (q == 0 ? kPairRe : kPairIm) : kReal;
                c++;
            }
        };
        if (!left) for (const Item &it : items) emit(it);
        else for (auto it = items.rbegin(); it != items.rend(); ++it) emit(*it);
        sc.starts.reserve(m);
        for (int q = 0; q < m; q++)
            if (L.kind[q] != kPairIm) sc.starts.push_back(q);
        std::vector<int2> slots;
        for (int q = 0; q < m;) {
            if (L.kind[q] == kPairRe) {
                slots.push_back(make_int2(q, q + 1));
                sc.slot_k.push_back(L.colk[q + 1]);
                q += 2;
            } else if (q + 1 < m && L.kind[q + 1] == kReal) {
                slots.push_back(make_int2(q, q + 1));
                sc.slot_k.push_back(L.colk[q + 1]);
                q += 2;
            } else {
                slots.push_back(make_int2(q, -1));
                sc.slot_k.push_back(L.colk[q]);
                q += 1;
            }
        }
        sc.nslots = (int)slots.size();
        int *d_ints = scr.get<int>(5 * (size_t)m);
        uint8_t *d_kind = scr.get<uint8_t>((size_t)m);
        int2 *d_slots = diag_tc ? scr.get<int2>(std::max<size_t>(1, slots.size())) : nullptr;
        if (scr.err) { set_last_error(cudaGetErrorString(scr.err)); return 1; }
        if (d_slots && !slots.empty())
            XTG_CK(cudaMemcpyAsync(d_slots, slots.data(), slots.size() * sizeof(int2), cudaMemcpyHostToDevice, st));
        sc.d_slots = d_slots;
        std::vector<int> ints(5 * (size_t)m, 0);
        std::copy(L.colk.begin(), L.colk.end(), ints.begin());
        std::copy(L.src.begin(), L.src.end(), ints.begin() + m);
        std::copy(L.kext.begin(), L.kext.end(), ints.begin() + 2 * m);
        std::copy(L.outcol.begin(), L.outcol.end(), ints.begin() + 3 * m);
        std::copy(sc.starts.begin(), sc.starts.end(), ints.begin() + 4 * m);
        XTG_CK(cudaMemcpyAsync(d_ints, ints.data(), ints.size() * sizeof(int), cudaMemcpyHostToDevice, st));
        XTG_CK(cudaMemcpyAsync(d_kind, L.kind.data(), m, cudaMemcpyHostToDevice, st));
        sc.d_ints = d_ints;
        sc.d_kind = d_kind;
        return 0;
    };
    SideCols side_cols[2];
    if (want_r && build_cols(false, side_cols[0])) return 1;
    if (want_l && build_cols(true, side_cols[1])) return 1;
    if (opt.staged) opt.staged(st);
    if (opt.host_norms) {
        // kernel arguments, not a copy: a host-to-device copy could wait behind the panels
        double hn[2] = {0, 0};
        opt.host_norms(hn);
        set_norms_kernel<R><<<1, 1, 0, st>>>(d_norms, R(hn[0]), R(hn[1]));
        XTG_CK(cudaGetLastError());
    }

    // One side on stream `st` with scratch from `scr` (both shadow the call's own).
    // ---- refinement of the split form (real double) --------------------------------------------
    // Each side's split pass flags the columns whose sketched residual exceeds the bound
    // (d_flags, copied to pinned host memory before the call's final synchronisation); the
    // flagged eigenvectors are then solved again with FP64 GEMMs and written over their
    // output columns (the back-transform reuses the split pass's copy of Z / Q).
    const bool refine_on = nsplit > 0 && opt.refine && !CPLX && std::is_same<R, double>::value;
    uint8_t *d_flags = nullptr, *h_flags = nullptr;
    if (refine_on) {
        cudaError_t e = cudaSuccess;
        CallRes *cr = res.get(&e);
        XTG_CK(e);
        XTG_CK(cr->reserve_flags(2 * (size_t)m_total));
        h_flags = cr->hflags;
        d_flags = scr.get<uint8_t>(2 * (size_t)m_total);
        if (scr.err) { set_last_error(cudaGetErrorString(scr.err)); return 1; }
    }
    // Flags of one side's columns from the sketch T = [GS; GP] X and ||x||^2 (see
    // kernels_refine.cuh), copied to the pinned host flags.
    auto refine_side = [&](const SideCols &sc, const R *coef, const E *T, const E *x2, uint8_t *flags,
                           cudaStream_t st, Scratch &scr) -> int {
        if constexpr (!CPLX && std::is_same<R, double>::value) {
            using namespace refine;
            const int m = sc.L.m, nitems = (int)sc.starts.size();
            int *cnt = scr.get<int>(1);
            if (scr.err) { set_last_error(cudaGetErrorString(scr.err)); return 1; }
            XTG_CK(cudaMemsetAsync(cnt, 0, sizeof(int), st));
            tr.run(kTPrep, 0, 0, st, [&] {
                refine_flags_kernel<<<(nitems + 7) / 8, 256, 0, st>>>(
                    T, x2, sketch_chunks(n), m, sc.d_ints + 4 * m, nitems, sc.d_kind, coef, d_norms,
                    opt.refine_bound, flags, cnt);
            });
            XTG_CK(cudaGetLastError());
            const size_t off = (size_t)(flags - d_flags);
            XTG_CK(cudaMemcpyAsync(h_flags + off, flags, (size_t)m, cudaMemcpyDeviceToHost, st));
        }
        return 0;
    };

    // `o`: the options of this pass; `sc`: its column list; `plain`: FP64 GEMMs whatever the
    // call's split form; `zc_in`: the back-transform's copy of Z / reversed Q made by an
    // earlier pass (else made here), returned through `zc_keep`; `flags`: when set, the split
    // pass writes one refinement flag per column of sc before anything goes to VL / VR.
    auto run_side = [&](bool left, cudaStream_t st, Scratch &scr, const Options &o, const SideCols &sc, bool plain,
                        E *zc_in, E **zc_keep, uint8_t *flags) -> int {
        const int nsplit_side = plain ? 0 : nsplit;
        const ColList &L = sc.L;
        SplitBufs sbuf;
        CrtBufs cbuf;
        cudaError_t split_err = cudaSuccess;
        // C (+)= A B of one update or back-transform launch, FP64 DMMA/SIMT or BF16 slices
        // traced as class `cat` (flops / bytes: the product's algorithmic counts), the residue
        // form by parts (kTSplitPrep / kTSplitGemm / kTSplitCrt)
        auto gemm = [&](const GemmArgs<E> &g, cudaStream_t gs, int cat, double flops, double bytes) {
            if constexpr (std::is_same<E, double>::value) {
                // launches with few output rows (the update of the upper block of a pair) do
                // too little work per tile to amortise slicing and the tensor-core pipeline;
                // they never use the slice buffers, so the buffers have one user stream
                if (nsplit_side && g.M - g.mlo >= 512 && (o.split_kind != 2 || g.K < (1 << 16))) {
                    cudaError_t e = cudaSuccess;
                    if (o.split_kind == 2) {
                        e = launch_crt(g, nsplit_side, cbuf, scr, d_err, gs, &tr, flops);
                    } else {
                        tr.run(cat, flops, bytes, gs, [&] {
                            e = o.split_kind == split::kI8
                                    ? launch_split<split::kI8>(g, nsplit_side, sbuf, scr, d_err, gs)
                                    : launch_split<split::kBF16>(g, nsplit_side, sbuf, scr, d_err, gs);
                        });
                    }
                    if (e != cudaSuccess) split_err = e;
                    return;
                }
            }
            tr.run(cat, flops, bytes, gs, [&] { launch_gemm<E>(g, o.simt != 0, gs); });
        };
        // row blocks (problem orientation), bottom to top; a 2x2 block is never split
        auto split = [&](int j) -> bool {  // rows j-1, j form a 2x2 diagonal block
            if (CPLX || j <= 0 || j >= n) return false;
            int kq = left ? n - 1 - j : j - 1;  // original index of the block's first row
            return sub[kq] || pairstart[kq];
        };
        std::vector<std::pair<int, int>> blocks;
        for (int cur = n; cur > 0;) {
            int j = std::max(0, cur - kBlock);
            if (j > 0 && split(j)) j += 1;
            blocks.push_back({j, cur});
            cur = j;
        }

        // ---- device buffers -------------------------------------------------------------
        const int m = L.m;
        const E *Sp = S, *Pp = P;
        int lsp = lds, lpp = ldp;
        // Left problem: (F S^H F, F P^H F).  Rows [0, t) of S and P become columns [n - t, n) of
        // the transposed copies; t_done rows are done.  With o.rows_ready (S and P still on
        // their way up) each group transposes the rows it needs once they have arrived,
        // otherwise all rows are transposed here.
        E *St = nullptr, *Pt = nullptr;
        int t_done = 0;
        auto transpose_rows = [&](int t1) {
            if (t1 <= t_done) return;
            const int c0 = n - t1, c1 = n - t_done;
            dim3 g((n + 31) / 32, (c1 - c0 + 31) / 32), b(32, 8);
            tr.run(kTPrep, 0, 2.0 * n * (c1 - c0) * esz, st,
                   [&] { rev_transpose_kernel<E><<<g, b, 0, st>>>(S, lds, St, ld_n, n, 1, c0, c1); });
            if (Pt)
                tr.run(kTPrep, 0, 2.0 * n * (c1 - c0) * esz, st,
                       [&] { rev_transpose_kernel<E><<<g, b, 0, st>>>(P, ldp, Pt, ld_n, n, 1, c0, c1); });
            t_done = t1;
        };
        auto left_rows = [&](int need) {  // rows [0, need) of S, P on the device and transposed
            if (!left || need <= t_done) return;
            const int got = o.rows_ready ? std::min(n, std::max(need, o.rows_ready(need, st))) : n;
            transpose_rows(got);
        };
        if (left) {
            St = scr.get<E>((size_t)ld_n * n);
            Pt = o.p_identity ? nullptr : scr.get<E>((size_t)ld_n * n);  // F I^H F = I
            if (scr.err) { set_last_error(cudaGetErrorString(scr.err)); return 1; }
            if (!o.rows_ready) transpose_rows(n);
            if (Pt) {
                Pp = Pt;
                lpp = ld_n;
            }
            Sp = St;
            lsp = ld_n;
        }
        // work items of the diagonal solves: every column that starts an eigenvector
        const std::vector<int> &items = sc.starts;
        const int nitems = (int)items.size();
        // look-ahead (XTGEVC3_LOOKAHEAD): the trailing update of a block pair runs on a second
        // stream while the next pair is solved (see the loop below); off while tracing
        // (clean per-kernel times) and in arena mode (fixed scratch)
        const bool ahead = o.lookahead && !tr.on && !o.arena && !o.p_identity && blocks.size() >= 3 &&
                           !(nsplit_side && o.split_kind == 2);
        // Without look-ahead, row blocks are taken in groups of `group` (one trailing GEMM
        // with K = 2 x the group's rows); arena mode keeps groups of two, so that its fixed
        // scratch holds the update operand.  Look-ahead takes pairs with padded blocks.
        const int group = o.arena ? 2 : (nsplit_side ? split_group_blocks() : kGroupBlocks);
        const int ldx = ld_n;
        const int ldy = ahead ? 4 * kBlock : 2 * round_up(group * kBlock, kKPad);  // both halves
        E *X = scr.get<E>((size_t)ldx * m);
        E *Ybuf[2];
        Ybuf[0] = scr.get<E>((size_t)ldy * m);
        Ybuf[1] = ahead ? scr.get<E>((size_t)ldy * m) : Ybuf[0];
        E *Y = Ybuf[0];
        R *pending = ahead ? scr.get<R>((size_t)m) : nullptr;
        R *coef = scr.get<R>((size_t)ncoef * m);
        if (scr.err) { set_last_error(cudaGetErrorString(scr.err)); return 1; }
        const int *d_ints = sc.d_ints;
        const uint8_t *d_kind = sc.d_kind;
        const int *d_colk = d_ints, *d_src = d_ints + m, *d_kext = d_ints + 2 * m, *d_outcol = d_ints + 3 * m;
        const int *d_items = d_ints + 4 * m;
        XTG_CK(cudaMemsetAsync(X, 0, (size_t)ldx * m * sizeof(E), st));
        if (pending) fill_one_kernel<R><<<(m + 255) / 256, 256, 0, st>>>(pending, m);

        tr.run(kTPrep, 0, (double)m * ncoef * sizeof(R), st, [&] {
            if constexpr (CPLX) {
                coef_cplx_kernel<R><<<(m + 127) / 128, 128, 0, st>>>(
                    reinterpret_cast<const cplx<R> *>(d_eig), reinterpret_cast<const cplx<R> *>(d_eig + 2 * n), d_src,
                    m, left ? 1 : 0, d_norms, coef);
            } else {
                coef_real_kernel<R><<<(m + 127) / 128, 128, 0, st>>>(d_eig, d_eig + n, d_eig + 2 * n, d_src, d_kind,
                                                                     m, left ? 1 : 0, d_norms, coef);
            }
        });
        XTG_CK(cudaGetLastError());

        // ---- residual sketch of the refinement check (split form) ------------------------------
        // [GS; GP] = G [S P] and T = [GS; GP] X with ||x_c||^2, after the substitution.
        E *sk_G2 = nullptr, *sk_G2p = nullptr, *sk_T = nullptr, *sk_x2 = nullptr;
        const int sk_nch = refine::sketch_chunks(n);
        if (flags) {
            sk_G2 = scr.get<E>((size_t)n * 2 * refine::K);
            sk_G2p = scr.get<E>((size_t)sk_nch * n * 2 * refine::K);
            sk_T = scr.get<E>((size_t)sk_nch * m * 2 * refine::K);
            sk_x2 = scr.get<E>((size_t)sk_nch * m);
            if (scr.err) { set_last_error(cudaGetErrorString(scr.err)); return 1; }
        }
        // [GS; GP] depends on S and P only: when all of them are on the device at this point it
        // is computed on a second stream while the substitution runs (joined before T is
        // formed), otherwise after the substitution.  An early return joins it before the
        // stream-ordered scratch is released.
        // the stream and events are the call's pooled ones (one set per side)
        cudaStream_t sk_st = nullptr;
        cudaEvent_t sk_ev[2] = {nullptr, nullptr};
        bool sk_pending = false;
        struct SketchGuard {
            cudaEvent_t *ev;
            bool &pending;
            cudaStream_t main;
            ~SketchGuard()
            {
                if (pending) cudaStreamWaitEvent(main, ev[1], 0);
            }
        } sk_guard{sk_ev, sk_pending, st};
        auto matrix_sketch = [&](cudaStream_t s) -> int {
            if constexpr (!CPLX && std::is_same<R, double>::value) {
                using namespace refine;
                XTG_CK(cudaMemsetAsync(sk_G2p, 0, (size_t)sk_nch * n * 2 * K * sizeof(E), s));
                tr.run(kTPrep, 0, (double)n * n * esz, s, [&] {
                    sketch_matrix_kernel<<<dim3((n + SK_COLS - 1) / SK_COLS, sk_nch), 256, 0, s>>>(Sp, lsp, Pp, lpp,
                                                                                                   n, sk_G2p);
                    sum_chunks_kernel<<<4 * sm_count(), 256, 0, s>>>(sk_G2p, sk_nch, (size_t)n * 2 * K, sk_G2);
                });
                XTG_CK(cudaGetLastError());
            }
            return 0;
        };
        if (flags && !o.arena && !tr.on && !o.cols_ready && !o.rows_ready) {
            cudaError_t e = cudaSuccess;
            CallRes *cr = res.get(&e);
            XTG_CK(e);
            XTG_CK(cr->reserve_sketch());
            sk_st = cr->sk_stream[left ? 1 : 0];
            sk_ev[0] = cr->sk_ev[left ? 1 : 0][0];
            sk_ev[1] = cr->sk_ev[left ? 1 : 0][1];
            XTG_CK(cudaEventRecord(sk_ev[0], st));
            XTG_CK(cudaStreamWaitEvent(sk_st, sk_ev[0], 0));
            if (matrix_sketch(sk_st)) return 1;
            XTG_CK(cudaEventRecord(sk_ev[1], sk_st));
            sk_pending = true;
        }
        // ---- blocked substitution ----------------------------------------------------------
        // Row blocks are taken in groups of `group` adjacent blocks, rows [q0, q1), bottom to
        // top: each block is solved, then the rows of the group's blocks above it are updated
        // with its solution (small GEMM); after the top block one GEMM updates every row above
        // the group with the whole group, K = 2 (q1 - q0) (256 rows: K = 512).  The update
        // operand Y of a group holds the -ac x rows of its blocks in row order, rows [0, q1 -
        // q0), zero padded to Kq = round_up(q1 - q0, kKPad), then the b x rows at Kq; the
        // GEMMs read it as one S strip and one P strip.  A guard that fires in a block rescales
        // the rows of Y below it (zl window of the solve), which the group's GEMMs consume
        // together with the block's own.  (Look-ahead: pairs, each block padded to kKPad.)
        const size_t diag_smem = 2 * kBlock * kSmLd * sizeof(E);
        auto first_col = [&](int r) {
            return int(std::lower_bound(L.colk.begin(), L.colk.end(), r) - L.colk.begin());
        };
        auto strip = [&](const E *A, int lda, int w0, int col, int jnb, int boff) {
            GemmSeg<E> sg;
            sg.A = A + (size_t)w0 + (size_t)col * lda;
            sg.lda = lda;
            sg.acols = jnb;
            sg.K = round_up(jnb, kKPad);
            sg.boff = boff;
            return sg;
        };
        // X[w0 + mlo : w0 + M, c0:m] += sum over segments
        auto update = [&](int w0, int mlo, int M, int c0, int nseg, const GemmSeg<E> *segs, double kflops,
                          cudaStream_t us) {
            GemmArgs<E> g;
            g.M = M;
            g.N = m - c0;
            g.mlo = mlo;
            g.nseg = nseg;
            g.K = 0;
            for (int s = 0; s < nseg; s++) {
                g.seg[s] = segs[s];
                g.K += segs[s].K;
            }
            g.B = Y + (size_t)c0 * ldy;
            g.ldb = ldy;
            g.brows = ldy;
            g.C = X + (size_t)w0 + (size_t)c0 * ldx;
            g.ldc = ldx;
            g.ccol = nullptr;
            g.kext = nullptr;
            g.accumulate = 1;
            const double rows = M - mlo;
            const double uf = 2.0 * rows * g.N * kflops * cfl;
            const double ub = (2.0 * rows * g.N + rows * kflops + kflops * g.N) * esz;
            gemm(g, us, kTUpdate, uf, ub);
        };
        // safe_lo >= 0: deferred guard scaling of the rows above safe_lo (look-ahead)
        // ypad < 0: the block's rows padded to kKPad
        auto diag_solve = [&](int r0, int r1, int ys_off, int yhalf, int zl_off, int zl_len, int safe_lo,
                              int ypad = -1) {
            const int jnb = r1 - r0;
            const int c0 = first_col(r0);
            if (c0 >= m) return;
            const int bpad = ypad >= 0 ? ypad : round_up(jnb, kKPad);
            DiagArgs<R> da{};
            da.S = reinterpret_cast<const R *>(Sp);
            da.P = reinterpret_cast<const R *>(Pp);
            da.lds = lsp;
            da.ldp = lpp;
            da.n = n;
            da.r0 = r0;
            da.r1 = r1;
            da.ys_off = ys_off;
            da.yhalf = yhalf;
            da.ypad = bpad;
            da.zl_off = zl_off;
            da.zl_len = zl_len;
            da.items = d_items;
            da.it0 = int(std::lower_bound(items.begin(), items.end(), c0) - items.begin());
            da.nitems = nitems;
            da.colk = d_colk;
            da.kind = d_kind;
            da.coef = coef;
            da.X = reinterpret_cast<R *>(X);
            da.ldx = ldx;
            da.Y = reinterpret_cast<R *>(Y);
            da.ldy = ldy;
            da.thr_rhs = bignum / R(10);
            da.thr_upd = bignum / R(std::max(1, jnb));
            da.left_seed = left ? 1 : 0;
            da.pending = safe_lo >= 0 ? pending : nullptr;
            da.safe_lo = safe_lo;
            const int grid = std::max(1, std::min((nitems - da.it0 + diag_warps - 1) / diag_warps, diag_ctas));
            // algorithmic work of the shifted solves: ~2 nrows^2 real flops per real column,
            // 4x that per complex column or (Re, Im) pair; bytes: rhs in, solution and
            // update operand out, the S/P block once
            double dfl = 0, dby = 2.0 * jnb * jnb * esz;
            for (int c = c0; c < m; c++) {
                if (L.kind[c] == kPairIm) continue;
                const int nr = L.colk[c] < r1 ? L.colk[c] - r0 : jnb;
                const double w = (CPLX || L.kind[c] == kPairRe) ? 4.0 : 1.0;
                const double cols = L.kind[c] == kPairRe ? 2.0 : 1.0;
                dfl += 2.0 * nr * nr * w;
                dby += cols * (double(nr < jnb ? 0 : jnb) + jnb + 2.0 * bpad) * esz;
            }
            tr.run(kTDiag, dfl, dby, st, [&] {
                if constexpr (CPLX) {
                    diag_solve_cplx<R><<<grid, diag_threads, diag_smem, st>>>(da);
                } else if constexpr (std::is_same<R, double>::value) {
                    if (diag_tc) {
                        // first slot with an active column (slots in column order, k ascending)
                        const int s0 = int(std::lower_bound(sc.slot_k.begin(), sc.slot_k.end(), r0) -
                                           sc.slot_k.begin());
                        const int per = dtc::kWarps * dtc::kSlots;
                        const int tgrid = std::max(1, (sc.nslots - s0 + per - 1) / per);
                        dtc::diag_solve_real_tc<<<tgrid, dtc::kThreads, dtc::kSmemBytes, st>>>(da, sc.d_slots, s0,
                                                                                               sc.nslots);
                    } else {
                        diag_solve_real<R><<<grid, diag_threads, diag_smem, st>>>(da);
                    }
                } else {
                    diag_solve_real<R><<<grid, diag_threads, diag_smem, st>>>(da);
                }
            });
        };
        const int nbk = (int)blocks.size();
        // the P strips of the identity are zero: the standard problem updates with S only
        const int nstrips = o.p_identity ? 1 : 2;
        for (int gi = 0; !ahead && gi < nbk; gi += group) {
            const int ge = std::min(nbk, gi + group);  // blocks [gi, ge); blocks[gi] is the lowest
            const int q0 = blocks[ge - 1].first, q1 = blocks[gi].second;
            const int acols = q1 - q0, kq = round_up(acols, kKPad);
            // the group reads columns [q0, q1) of S and P (right problem: the caller's columns;
            // left problem: rows [n - q1, n - q0) of the caller's S and P, transposed)
            if (o.cols_ready && !left) o.cols_ready(false, q0, st);
            left_rows(n - q0);
            for (int bi = gi; bi < ge; bi++) {
                const int r0 = blocks[bi].first, r1 = blocks[bi].second, jnb = r1 - r0, ys = r0 - q0;
                // the lowest block also writes the zero padding of the group's operand rows
                diag_solve(r0, r1, ys, kq, ys + jnb, kq - (ys + jnb), -1, jnb + (bi == gi ? kq - acols : 0));
                const int c0 = first_col(r0);
                if (bi + 1 < ge && c0 < m) {  // rows [q0, r0) (window from an even row)
                    const int w0 = q0 & ~1, mlo = q0 & 1;
                    GemmSeg<E> sg[2] = {strip(Sp, lsp, w0, r0, jnb, ys), strip(Pp, lpp, w0, r0, jnb, kq + ys)};
                    update(w0, mlo, mlo + (r0 - q0), c0, nstrips, sg, nstrips * double(jnb), st);
                }
            }
            const int c0 = first_col(q0);
            if (q0 > 0 && c0 < m) {
                GemmSeg<E> sg[2] = {strip(Sp, lsp, 0, q0, acols, 0), strip(Pp, lpp, 0, q0, acols, kq)};
                update(0, 0, q0, c0, nstrips, sg, nstrips * double(acols), st);
            }
            XTG_CK(cudaGetLastError());
        }
        // Look-ahead (ahead == true).  Pair p owns rows [u0_p, l1_p); the next pair's rows are
        // [a0, u0_p).  On the main stream: solve L_p, small update of U_p, solve U_p; wait for
        // the trailing update of pair p-1 (it writes rows [0, u0_p)); apply deferred guard
        // factors to rows [0, u0_p); update the next pair's rows [a0, u0_p) (small GEMM).  On
        // the second stream: the trailing update of rows [0, a0), which overlaps the solves of
        // pair p+1.  Pairs alternate between two update operands Y; a solve defers guard
        // scaling of rows [0, u0_p), the only rows the concurrent update writes.
        cudaStream_t st2 = nullptr;
        cudaEvent_t ev_main = nullptr, ev_tr = nullptr;
        struct Guard {
            cudaStream_t &s;
            cudaEvent_t &a, &b;
            ~Guard()
            {
                if (a) cudaEventDestroy(a);
                if (b) cudaEventDestroy(b);
                if (s) cudaStreamDestroy(s);
            }
        } guard{st2, ev_main, ev_tr};
        if (ahead) {
            // the second stream starts from events of this one: all of S and P first
            if (o.cols_ready && !left) o.cols_ready(false, 0, st);
            left_rows(n);
            // slice buffers of the trailing updates are sized here, on the main stream: growing
            // them inside a launch on the second stream would not be ordered with its use
            if constexpr (std::is_same<E, double>::value) {
                if (nsplit_side) {
                    const int kmax = 4 * kBlock;
                    auto reserve = [&](int bk, int bn, size_t esz_) {
                        const size_t an = (size_t)nsplit_side * round_up(n, split::BM) * round_up(kmax, bk) * esz_;
                        const size_t bn_ = (size_t)nsplit_side * round_up(m, bn) * round_up(kmax, bk) * esz_;
                        if (an > sbuf.acap) { sbuf.A = scr.get<unsigned char>(an); sbuf.acap = an; }
                        if (bn_ > sbuf.bcap) { sbuf.B = scr.get<unsigned char>(bn_); sbuf.bcap = bn_; }
                        const size_t mp = round_up(n, split::BM), np = round_up(m, bn);
                        if (mp > sbuf.ecap_a) { sbuf.ea = scr.get<int>(mp); sbuf.ecap_a = mp; }
                        if (np > sbuf.ecap_b) { sbuf.eb = scr.get<int>(np); sbuf.ecap_b = np; }
                    };
                    if (o.split_kind == split::kI8)
                        reserve(split::Cfg<split::kI8>::BK, split::Cfg<split::kI8>::BN, 1);
                    else
                        reserve(split::Cfg<split::kBF16>::BK, split::Cfg<split::kBF16>::BN, 2);
                    if (scr.err) { set_last_error(cudaGetErrorString(scr.err)); return 1; }
                }
            }
            XTG_CK(cudaStreamCreateWithFlags(&st2, cudaStreamNonBlocking));
            XTG_CK(cudaEventCreateWithFlags(&ev_main, cudaEventDisableTiming));
            XTG_CK(cudaEventCreateWithFlags(&ev_tr, cudaEventDisableTiming));
        }
        bool tr_pending = false;  // a trailing update is queued on st2 and not yet waited for
        int pidx = 0;
        for (int bi = 0; ahead && bi < nbk;) {
            const int l0 = blocks[bi].first, l1 = blocks[bi].second, jl = l1 - l0, bl = round_up(jl, kKPad);
            Y = Ybuf[pidx & 1];
            if (bi + 1 == nbk) {  // unpaired top block
                if (tr_pending) {
                    XTG_CK(cudaStreamWaitEvent(st, ev_tr, 0));
                    tr_pending = false;
                    apply_pending_kernel<E, R><<<(m * 32 + 255) / 256, 256, 0, st>>>(X, ldx, pending, m, l1);
                }
                diag_solve(l0, l1, 0, bl, 0, 0, -1);
                const int c0 = first_col(l0);
                if (l0 > 0 && c0 < m) {
                    GemmSeg<E> sg[2] = {strip(Sp, lsp, 0, l0, jl, 0), strip(Pp, lpp, 0, l0, jl, bl)};
                    update(0, 0, l0, c0, 2, sg, 2.0 * jl, st);
                }
                XTG_CK(cudaGetLastError());
                bi += 1;
                continue;
            }
            const int u0 = blocks[bi + 1].first, ju = l0 - u0, bu = round_up(ju, kKPad), bh = bu + bl;
            const int safe = u0;  // rows [0, u0) belong to the concurrent trailing update
            diag_solve(l0, l1, bu, bh, 0, 0, safe);
            const int c0l = first_col(l0);
            if (c0l < m) {  // rows of U (window from an even row) += L's contribution
                const int w0 = u0 & ~1, mlo = u0 & 1;
                GemmSeg<E> sg[2] = {strip(Sp, lsp, w0, l0, jl, bu), strip(Pp, lpp, w0, l0, jl, bh + bu)};
                update(w0, mlo, mlo + ju, c0l, 2, sg, 2.0 * jl, st);
            }
            diag_solve(u0, l0, 0, bh, bu, bl, safe);
            const int c0u = first_col(u0);
            if (tr_pending) {
                XTG_CK(cudaStreamWaitEvent(st, ev_tr, 0));
                tr_pending = false;
            }
            if (u0 > 0) apply_pending_kernel<E, R><<<(m * 32 + 255) / 256, 256, 0, st>>>(X, ldx, pending, m, u0);
            if (u0 > 0 && c0u < m) {
                // the next pair's rows [a0, u0): its U block's start, or the top block's
                const int a0 = bi + 3 < nbk ? blocks[bi + 3].first : blocks[bi + 2].first;
                const int w0 = a0 & ~1, mlo = a0 & 1;
                GemmSeg<E> sa[4] = {strip(Sp, lsp, w0, u0, ju, 0), strip(Sp, lsp, w0, l0, jl, bu),
                                    strip(Pp, lpp, w0, u0, ju, bh), strip(Pp, lpp, w0, l0, jl, bh + bu)};
                update(w0, mlo, mlo + (u0 - a0), c0u, 4, sa, 2.0 * (ju + jl), st);
                if (a0 > 0) {
                    XTG_CK(cudaEventRecord(ev_main, st));
                    XTG_CK(cudaStreamWaitEvent(st2, ev_main, 0));
                    GemmSeg<E> sg[4] = {strip(Sp, lsp, 0, u0, ju, 0), strip(Sp, lsp, 0, l0, jl, bu),
                                        strip(Pp, lpp, 0, u0, ju, bh), strip(Pp, lpp, 0, l0, jl, bh + bu)};
                    update(0, 0, a0, c0u, 4, sg, 2.0 * (ju + jl), st2);
                    XTG_CK(cudaEventRecord(ev_tr, st2));
                    tr_pending = true;
                }
            }
            XTG_CK(cudaGetLastError());
            bi += 2;
            pidx += 1;
        }
        // every deferred factor was applied within its own pair (the top block scales at once)
        if (tr_pending) XTG_CK(cudaStreamWaitEvent(st, ev_tr, 0));

        // LAPACK xTREVC3's phase for real 2x2 pairs (before the back-transform, which is linear)
        if constexpr (!CPLX) {
            if (o.lapack_pairs) {
                lapack_pair_phase_kernel<R><<<(m * 32 + 255) / 256, 256, 0, st>>>(
                    reinterpret_cast<R *>(X), ldx, m, d_colk, d_kext, d_kind, reinterpret_cast<const R *>(Sp), lsp,
                    left ? 1 : 0);
                XTG_CK(cudaGetLastError());
            }
        }

        // ---- refinement flags (split form) ---------------------------------------------------
        // Sketched residual of every computed column in problem coordinates: columns whose
        // residual exceeds the bound are flagged and solved again in FP64 after the call's
        // split pass (see the end of solve_device).
        if constexpr (!CPLX && std::is_same<R, double>::value) {
            if (flags) {
                using namespace refine;
                if (sk_pending) {
                    XTG_CK(cudaStreamWaitEvent(st, sk_ev[1], 0));
                    sk_pending = false;
                } else if (matrix_sketch(st)) {
                    return 1;
                }
                XTG_CK(cudaMemsetAsync(sk_T, 0, (size_t)sk_nch * m * 2 * K * sizeof(E), st));
                XTG_CK(cudaMemsetAsync(sk_x2, 0, (size_t)sk_nch * m * sizeof(E), st));
                tr.run(kTPrep, 0, 0.5 * (double)n * m * esz, st, [&] {
                    sketch_columns_kernel<<<dim3((m + SK_COLS - 1) / SK_COLS, sk_nch), 256, 0, st>>>(
                        sk_G2, X, ldx, m, d_kext, sk_T, sk_x2);
                });
                XTG_CK(cudaGetLastError());
                if (refine_side(sc, coef, sk_T, sk_x2, flags, st, scr)) return 1;
            }
        }

        // ---- write-back / back-transform -----------------------------------------------------
        // nothing has been written to VL / VR so far: a rejected plan stops here
        if (const int g = gate()) return g;
        E *V = left ? VL : VR;
        const int ldv = left ? ldvl : ldvr;
        // row panels: Z / Q arrive by rows (host-pointer path); each panel's rows of V are
        // computed as soon as its rows of Z / Q are up (V rows = Z rows X)
        const bool rpanels = do_back && o.back_rows_ready && o.rows_done && !o.normalize && !zc_in;
        if (rpanels) {
            E *Zc = scr.get<E>((size_t)ld_n * n);
            if (scr.err) { set_last_error(cudaGetErrorString(scr.err)); return 1; }
            if (zc_keep) *zc_keep = Zc;
            double bk = 0;
            for (int c = 0; c < m; c++) bk += L.kext[c];
            for (int r0 = 0; r0 < n;) {
                const int r1 = std::min(n, std::max(r0 + 1, o.back_rows_ready(left, r0 + 1, st)));
                const int rows = r1 - r0;
                if (left) {  // rows [r0, r1) of the column-reversed Q
                    dim3 g((rows + 255) / 256, n);
                    tr.run(kTPrep, 0, 2.0 * rows * n * esz, st, [&] {
                        rev_columns_kernel<E><<<g, 256, 0, st>>>(V + r0, ldv, Zc + r0, ld_n, rows, n);
                    });
                } else {
                    XTG_CK(cudaMemcpy2DAsync(Zc + r0, (size_t)ld_n * sizeof(E), V + r0, (size_t)ldv * sizeof(E),
                                             (size_t)rows * sizeof(E), n, cudaMemcpyDeviceToDevice, st));
                }
                GemmArgs<E> g;
                g.M = rows;
                g.N = m;
                g.mlo = 0;
                g.nseg = 1;
                g.seg[0] = strip(Zc, ld_n, r0, 0, n, 0);
                g.K = g.seg[0].K;
                g.B = X;
                g.ldb = ldx;
                g.brows = n;
                g.C = V + r0;
                g.ldc = ldv;
                g.ccol = d_outcol;
                g.kext = d_kext;
                g.accumulate = 0;
                g.reuse_b = r0 > 0;  // the same X for every panel
                const double bf = 2.0 * rows * bk * cfl;
                const double bb = ((double)rows * n + bk + (double)rows * m) * esz;
                gemm(g, st, kTBack, bf, bb);
                o.rows_done(left, st, r0, r1);
                r0 = r1;
            }
        } else if (do_back) {
            if (o.back_ready[left ? 1 : 0]) XTG_CK(cudaStreamWaitEvent(st, o.back_ready[left ? 1 : 0], 0));
            // copy of Z (right) or column-reversed Q (left), so V can be overwritten; a later
            // pass of the same call (the refinement) reuses it
            E *Zc = zc_in;
            if (!Zc) {
                Zc = scr.get<E>((size_t)ld_n * n);
                if (scr.err) { set_last_error(cudaGetErrorString(scr.err)); return 1; }
                if (left) {
                    dim3 g((n + 255) / 256, n);
                    tr.run(kTPrep, 0, 2.0 * n * n * esz, st,
                           [&] { rev_columns_kernel<E><<<g, 256, 0, st>>>(V, ldv, Zc, ld_n, n, n); });
                } else {
                    XTG_CK(cudaMemcpy2DAsync(Zc, (size_t)ld_n * sizeof(E), V, (size_t)ldv * sizeof(E), n * sizeof(E),
                                             n, cudaMemcpyDeviceToDevice, st));
                }
            }
            if (zc_keep) *zc_keep = Zc;
            // column chunks of equal work (sum of kext), never splitting a complex pair, so
            // that a caller can download each chunk's output columns while the next runs
            std::vector<int> cuts = {0};
            if (o.cols_done && !o.normalize) {
                double tot = 0;
                for (int c = 0; c < m; c++) tot += L.kext[c];
                const int nch = std::min(4, m);
                double acc = 0;
                for (int c = 0; c < m; c++) {
                    acc += L.kext[c];
                    const int nxt = c + 1;
                    if ((int)cuts.size() < nch && nxt < m && acc >= tot * cuts.size() / nch && L.kind[nxt] != kPairIm)
                        cuts.push_back(nxt);
                }
            }
            cuts.push_back(m);
            for (size_t q = 0; q + 1 < cuts.size(); q++) {
                const int c0 = cuts[q], c1 = cuts[q + 1];
                GemmArgs<E> g;
                g.M = n;
                g.N = c1 - c0;
                g.mlo = 0;
                g.nseg = 1;
                g.seg[0] = strip(Zc, ld_n, 0, 0, n, 0);
                g.K = g.seg[0].K;
                g.B = X + (size_t)c0 * ldx;
                g.ldb = ldx;
                g.brows = n;
                g.C = V;
                g.ldc = ldv;
                g.ccol = d_outcol + c0;
                g.kext = d_kext + c0;
                g.accumulate = 0;
                double bk = 0;
                for (int c = c0; c < c1; c++) bk += L.kext[c];
                const double bf = 2.0 * n * bk * cfl;
                const double bb = ((double)n * L.kext[c1 - 1] + bk + (double)n * (c1 - c0)) * esz;
                gemm(g, st, kTBack, bf, bb);
                if (o.cols_done && !o.normalize) {
                    int o0 = m, o1 = 0;
                    for (int c = c0; c < c1; c++) {
                        o0 = std::min(o0, L.outcol[c]);
                        o1 = std::max(o1, L.outcol[c] + 1);
                    }
                    if (o1 - o0 == c1 - c0) o.cols_done(left, st, o0, o1);  // a contiguous block of outputs
                }
            }
        } else {
            dim3 g(std::max(1, std::min((n + 255) / 256, 64)), m);
            tr.run(kTWriteback, 0, 2.0 * n * m * esz, st, [&] {
                writeback_kernel<E><<<g, 256, 0, st>>>(X, ldx, V, ldv, n, m, d_outcol, d_kext, left ? 1 : 0);
            });
        }
        XTG_CK(cudaGetLastError());

        if (o.normalize) {
            if constexpr (CPLX) {
                cplx<R> *Vc = reinterpret_cast<cplx<R> *>(V);
                tr.run(kTNormalize, 0, 2.0 * n * m * esz, st, [&] {
                    if (n <= 1024) normalize_cplx_1p_kernel<R, 4><<<m, 256, 0, st>>>(Vc, ldv, n, d_outcol, m);
                    else if (n <= 2048) normalize_cplx_1p_kernel<R, 8><<<m, 256, 0, st>>>(Vc, ldv, n, d_outcol, m);
                    else if (n <= 4096) normalize_cplx_1p_kernel<R, 16><<<m, 256, 0, st>>>(Vc, ldv, n, d_outcol, m);
                    else if (n <= 8192) normalize_cplx_1p_kernel<R, 32><<<m, 256, 0, st>>>(Vc, ldv, n, d_outcol, m);
                    else normalize_cplx_kernel<R><<<m, 256, 0, st>>>(Vc, ldv, n, d_outcol, m);  // two passes
                });
            } else {
                const int ni = nitems;
                tr.run(kTNormalize, 0, 2.0 * n * m * esz, st, [&] {
                    if (n <= 1024)
                        normalize_real_1p_kernel<R, 4><<<ni, 256, 0, st>>>(V, ldv, n, d_items, d_outcol, d_kind, ni);
                    else if (n <= 2048)
                        normalize_real_1p_kernel<R, 8><<<ni, 256, 0, st>>>(V, ldv, n, d_items, d_outcol, d_kind, ni);
                    else if (n <= 4096)
                        normalize_real_1p_kernel<R, 16><<<ni, 256, 0, st>>>(V, ldv, n, d_items, d_outcol, d_kind, ni);
                    else if (n <= 8192)
                        normalize_real_1p_kernel<R, 32><<<ni, 256, 0, st>>>(V, ldv, n, d_items, d_outcol, d_kind, ni);
                    else
                        normalize_real_kernel<R><<<m, 256, 0, st>>>(V, ldv, n, d_outcol, d_kind, m);  // two passes
                });
            }
            XTG_CK(cudaGetLastError());
        }
        if (split_err != cudaSuccess) {
            set_last_error(std::string("split-precision GEMM launch: ") + cudaGetErrorString(split_err));
            return 1;
        }
        if (o.side_done) o.side_done(left, st);
        return 0;
    };

    // The two sides are independent problems: with both requested they run concurrently,
    // the left one on a second stream (serially while tracing, so that kernel times are
    // not inflated by overlap).
    // A side returns 0, 1 (CUDA error) or 2 (plan rejected by the structure check: nothing
    // was written to VL / VR; the call runs again with the subdiagonal read back).
    auto rerun = [&]() -> int {
        XTG_CK(cudaStreamSynchronize(st));
        Options o2 = opt;
        o2.read_sub = 1;
        return solve_device<R, CPLX>(side, howmny, select, n, S_, lds, P_, ldp, alpha_, alphai_, beta_, VL_, ldvl,
                                     VR_, ldvr, m_total, o2, st);
    };
    E *zc_kept[2] = {nullptr, nullptr};  // each side's copy of Z / reversed Q (refinement pass)
    Scratch scr2(st);                    // the left side's scratch when it runs on its own stream
    if (want_r && want_l && !tr.on && !opt.arena) {
        cudaError_t e = cudaSuccess;
        CallRes *fk = res.get(&e);
        scr2.st = fk->side;
        XTG_CK(e);
        XTG_CK(cudaEventRecord(fk->fork, st));
        XTG_CK(cudaStreamWaitEvent(fk->side, fk->fork, 0));
        int rr = 0, rl = 0;
        rr = run_side(false, st, scr, opt, side_cols[0], false, nullptr, &zc_kept[0], d_flags);
        if (rr == 0) rl = run_side(true, fk->side, scr2, opt, side_cols[1], false, nullptr, &zc_kept[1],
                                   d_flags ? d_flags + m_total : nullptr);
        XTG_CK(cudaEventRecord(fk->join, fk->side));
        XTG_CK(cudaStreamWaitEvent(st, fk->join, 0));
        if (rr == 1 || rl == 1) {
            cudaStreamSynchronize(fk->side);
            return 1;
        }
        if (rr == 2 || rl == 2) return rerun();
    } else {
        const size_t mark = scr.used;
        int rc = want_r ? run_side(false, st, scr, opt, side_cols[0], false, nullptr, &zc_kept[0], d_flags) : 0;
        // arena: the right side's slices are reused; its kernels precede the left side's
        // on the same stream
        if (opt.arena) scr.used = mark;
        if (rc == 0 && want_l)
            rc = run_side(true, st, scr, opt, side_cols[1], false, nullptr, &zc_kept[1],
                          d_flags ? d_flags + m_total : nullptr);
        if (rc == 2) return rerun();
        if (rc) return 1;
    }
    XTG_CK(cudaStreamSynchronize(st));
    int refined = 0;
    if (refine_on) {
        // the FP64 pass over the flagged eigenvectors of each side, on the call's stream
        Options ro = opt;
        ro.staged = nullptr;
        ro.host_norms = nullptr;
        ro.cols_ready = nullptr;
        ro.rows_ready = nullptr;
        ro.side_done = nullptr;
        ro.cols_done = nullptr;
        ro.back_ready[0] = ro.back_ready[1] = nullptr;
        ro.back_rows_ready = nullptr;
        ro.rows_done = nullptr;
        for (int sd = 0; sd < 2; sd++) {
            if (!(sd ? want_l : want_r)) continue;
            const SideCols &sc = side_cols[sd];
            const uint8_t *fl = h_flags + (sd ? m_total : 0);
            std::vector<char> keep(n, 0);
            int cnt = 0;
            for (int c = 0; c < sc.L.m; c++)
                if (fl[c]) {
                    keep[sc.L.src[c]] = 1;
                    cnt++;
                }
            if (!cnt) continue;
            refined += cnt;
            SideCols sub;
            if (build_cols(sd == 1, sub, &keep)) return 1;
            const int rc = run_side(sd == 1, st, scr, ro, sub, true, zc_kept[sd], nullptr, nullptr);
            if (rc) return rc == 2 ? rerun() : 1;
            if (opt.cols_done || opt.side_done) {
                // the host-pointer path: download the rewritten output columns again
                std::vector<int> oc(sub.L.outcol);
                std::sort(oc.begin(), oc.end());
                for (size_t a = 0; a < oc.size();) {
                    size_t b = a + 1;
                    while (b < oc.size() && oc[b] == oc[b - 1] + 1) b++;
                    if (opt.cols_done) opt.cols_done(sd == 1, st, oc[a], oc[b - 1] + 1);
                    a = b;
                }
                if (!opt.cols_done) opt.side_done(sd == 1, st);
            }
        }
        XTG_CK(cudaStreamSynchronize(st));
    }
    g_refined = refined;
    tr.flush();
    if (d_err) {
        int h_err = 0;
        XTG_CK(cudaMemcpy(&h_err, d_err, sizeof(int), cudaMemcpyDeviceToHost));
        if (h_err) {
            set_last_error("split-precision GEMM: a bounded wait in the tensor-core pipeline expired");
            return 1;
        }
    }
    return 0;
}

template int solve_device<double, false>(char, char, const int *, int, const void *, int, const void *, int,
                                         const void *, const void *, const void *, void *, int, void *, int, int,
                                         const Options &, cudaStream_t);
template int solve_device<float, false>(char, char, const int *, int, const void *, int, const void *, int,
                                        const void *, const void *, const void *, void *, int, void *, int, int,
                                        const Options &, cudaStream_t);
template int solve_device<double, true>(char, char, const int *, int, const void *, int, const void *, int,
                                        const void *, const void *, const void *, void *, int, void *, int, int,
                                        const Options &, cudaStream_t);
template int solve_device<float, true>(char, char, const int *, int, const void *, int, const void *, int,
                                       const void *, const void *, const void *, void *, int, void *, int, int,
                                       const Options &, cudaStream_t);


template <class R, bool CPLX>
int eig_cond_device(int n, const void *A_, int lda, const void *B_, int ldb, const void *VL_, int ldvl,
                    const void *VR_, int ldvr, int m, const std::vector<int> &items, const std::vector<uint8_t> &kinds,
                    void *s_dev, cudaStream_t st)
{
    using E = typename std::conditional<CPLX, cplx<R>, R>::type;
    if (n <= 0 || m <= 0 || items.empty()) return 0;
    int dev = 0;
    XTG_CK(cudaGetDevice(&dev));
    configure_device(dev);
    Scratch scr(st);
    const int ldx = round_up(n, 32), ni = (int)items.size();
    E *AX = scr.get<E>((size_t)ldx * m);
    E *BX = scr.get<E>((size_t)ldx * m);
    int *d_items = scr.get<int>(2 * (size_t)ni);
    uint8_t *d_kinds = scr.get<uint8_t>((size_t)ni);
    if (scr.err) { set_last_error(cudaGetErrorString(scr.err)); return 1; }
    std::vector<int> ints(items);
    ints.insert(ints.end(), items.begin(), items.end());  // S index = first column
    XTG_CK(cudaMemcpyAsync(d_items, ints.data(), ints.size() * sizeof(int), cudaMemcpyHostToDevice, st));
    XTG_CK(cudaMemcpyAsync(d_kinds, kinds.data(), kinds.size(), cudaMemcpyHostToDevice, st));
    for (int which = 0; which < 2; which++) {  // AX = A VR, BX = B VR (K = n, padding masked)
        GemmArgs<E> g;
        g.M = n;
        g.N = m;
        g.mlo = 0;
        g.nseg = 1;
        g.seg[0].A = static_cast<const E *>(which ? B_ : A_);
        g.seg[0].lda = which ? ldb : lda;
        g.seg[0].acols = n;
        g.seg[0].K = round_up(n, kKPad);
        g.seg[0].boff = 0;
        g.K = g.seg[0].K;
        g.B = static_cast<const E *>(VR_);
        g.ldb = ldvr;
        g.brows = n;
        g.C = which ? BX : AX;
        g.ldc = ldx;
        g.ccol = nullptr;
        g.kext = nullptr;
        g.accumulate = 0;
        launch_gemm<E>(g, false, st);
        XTG_CK(cudaGetLastError());
    }
    eig_cond_kernel<R><<<(ni * 32 + 255) / 256, 256, 0, st>>>(
        ni, d_items, d_kinds, n, reinterpret_cast<const R *>(AX), reinterpret_cast<const R *>(BX), ldx,
        static_cast<const R *>(VL_), ldvl, static_cast<const R *>(VR_), ldvr, static_cast<R *>(s_dev), d_items + ni);
    XTG_CK(cudaGetLastError());
    XTG_CK(cudaStreamSynchronize(st));
    return 0;
}

template int eig_cond_device<double, false>(int, const void *, int, const void *, int, const void *, int, const void *,
                                             int, int, const std::vector<int> &, const std::vector<uint8_t> &, void *,
                                             cudaStream_t);
template int eig_cond_device<float, false>(int, const void *, int, const void *, int, const void *, int, const void *,
                                            int, int, const std::vector<int> &, const std::vector<uint8_t> &, void *,
                                            cudaStream_t);
template int eig_cond_device<double, true>(int, const void *, int, const void *, int, const void *, int, const void *,
                                            int, int, const std::vector<int> &, const std::vector<uint8_t> &, void *,
                                            cudaStream_t);
template int eig_cond_device<float, true>(int, const void *, int, const void *, int, const void *, int, const void *,
                                           int, int, const std::vector<int> &, const std::vector<uint8_t> &, void *,
                                           cudaStream_t);

}  // namespace xtg
