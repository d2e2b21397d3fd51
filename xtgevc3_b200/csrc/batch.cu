// Host side of the batched form: plan creation (argument checks, unit queue, workspace
// layout, tile configuration), CUDA-graph capture of {reset the queue, persistent kernel},
// launch, status read-back and the tile-configuration tuner.
#include "../../include/xtgevc3.h"
#include "engine.cuh"
#include "kernels_batch.cuh"

#include <algorithm>
#include <atomic>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <numeric>
#include <string>
#include <vector>

struct xtgevc3_batch {
    char prec = 'd';
    unsigned config = 0;
    int count = 0, grid = 0, nunits = 0;
    size_t smem = 0;
    void *d_pencils = nullptr;
    int4 *d_units = nullptr;
    long long *d_woff = nullptr;
    unsigned char *d_ws = nullptr;
    int *d_ctrl = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
};

namespace {

using namespace xtg;
using batch::THREADS;

static_assert(sizeof(xtgevc3_dpencil) == 7 * 4 + 4 + 9 * 8, "pencil descriptor layout");
static_assert(sizeof(xtgevc3_spencil) == 7 * 4 + 4 + 9 * 8, "pencil descriptor layout");

constexpr unsigned kDefaultD = XTGEVC3_BATCH_CONFIG(16, 64);
constexpr unsigned kDefaultS = XTGEVC3_BATCH_CONFIG(32, 64);
const unsigned kCandidates[] = {XTGEVC3_BATCH_CONFIG(16, 32), XTGEVC3_BATCH_CONFIG(16, 64),
                                XTGEVC3_BATCH_CONFIG(32, 32), XTGEVC3_BATCH_CONFIG(32, 64)};

std::atomic<unsigned> g_default_d{0}, g_default_s{0};
std::once_flag g_env_once;

unsigned parse_one(const char *s)
{
    int nt = 0, h = 0;
    if (std::sscanf(s, "%dx%d", &nt, &h) != 2) return 0;
    return XTGEVC3_BATCH_CONFIG(nt, h);
}

void read_env()
{
    const char *e = std::getenv("XTGEVC3_BATCH_CONFIG");
    if (!e) return;
    std::string s(e);
    size_t pos = 0;
    while (pos < s.size()) {
        size_t end = s.find(',', pos);
        if (end == std::string::npos) end = s.size();
        std::string item = s.substr(pos, end - pos);
        if (item.size() > 2 && item[1] == ':') {
            unsigned c = parse_one(item.c_str() + 2);
            if (item[0] == 'd' && c) g_default_d.store(c);
            if (item[0] == 's' && c) g_default_s.store(c);
        }
        pos = end + 1;
    }
}

unsigned default_config(char prec)
{
    std::call_once(g_env_once, read_env);
    unsigned c = prec == 'd' ? g_default_d.load() : g_default_s.load();
    return c ? c : (prec == 'd' ? kDefaultD : kDefaultS);
}

template <class T>
using KernelFn = void (*)(batch::Args<T>);

template <class T>
bool kernel_for(unsigned config, int xrows, KernelFn<T> *fn, size_t *smem)
{
    const int nt = (int)(config >> 8), h = (int)(config & 255u);
#define XTG_BATCH_CASE(NT_, H_)                                        \
    if (nt == NT_ && h == H_) {                                        \
        *fn = batch::batch_kernel<T, NT_, H_>;                         \
        *smem = batch::smem_bytes<T, NT_, H_>(xrows);                  \
        return true;                                                   \
    }
    XTG_BATCH_CASE(16, 32)
    XTG_BATCH_CASE(16, 64)
    XTG_BATCH_CASE(32, 32)
    XTG_BATCH_CASE(32, 64)
#undef XTG_BATCH_CASE
    return false;
}

template <class T>
bool fits(unsigned config, int xrows, int max_smem)
{
    KernelFn<T> fn;
    size_t smem;
    return kernel_for<T>(config, xrows, &fn, &smem) && smem <= (size_t)max_smem;
}

bool overlaps(const void *a, size_t abytes, const void *b, size_t bbytes)
{
    const char *x = static_cast<const char *>(a), *y = static_cast<const char *>(b);
    return a && b && x < y + bbytes && y < x + abytes;
}

void destroy(xtgevc3_batch *b)
{
    if (!b) return;
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    cudaFree(b->d_pencils);
    cudaFree(b->d_units);
    cudaFree(b->d_woff);
    cudaFree(b->d_ws);
    cudaFree(b->d_ctrl);
    delete b;
}

int bad_arg(const std::string &msg)
{
    set_last_error(msg);
    return -1;
}

#define XTG_BCK(call)                                                                        \
    do {                                                                                     \
        cudaError_t e_ = (call);                                                             \
        if (e_ != cudaSuccess) {                                                             \
            set_last_error(std::string(#call) + ": " + cudaGetErrorString(e_));             \
            destroy(b);                                                                      \
            return 1;                                                                        \
        }                                                                                    \
    } while (0)

template <class T>
int create(char side, char howmny, int count, const typename batch::PencilOf<T>::type *pencils, unsigned config,
           xtgevc3_batch **out)
{
    using PencilT = typename batch::PencilOf<T>::type;
    const char prec = sizeof(T) == 8 ? 'd' : 's';
    if (!out) return bad_arg("batched: plan pointer is NULL");
    *out = nullptr;
    set_last_error("");
    const bool right = side == 'R' || side == 'B', left = side == 'L' || side == 'B';
    if (!right && !left) return bad_arg("batched: side must be 'R', 'L' or 'B'");
    if (howmny != 'A' && howmny != 'B') return bad_arg("batched: howmny must be 'A' or 'B'");
    if (count < 0 || (count > 0 && !pencils)) return bad_arg("batched: bad pencil array");
    const bool back = howmny == 'B';
    int nmax = 0;
    for (int p = 0; p < count; p++) {
        const PencilT &d = pencils[p];
        const std::string at = "batched: pencil " + std::to_string(p) + ": ";
        if (d.n < 0) return bad_arg(at + "n < 0");
        nmax = std::max(nmax, d.n);
        if (d.n == 0) continue;
        const size_t n = (size_t)d.n;
        if (!d.S || !d.P || !d.alphar || !d.alphai || !d.beta) return bad_arg(at + "NULL input array");
        if (d.lds < d.n || d.ldp < d.n) return bad_arg(at + "lds/ldp < n");
        if (right) {
            if (!d.VR || d.ldvr < d.n) return bad_arg(at + "VR is NULL or ldvr < n");
            if (back && (!d.Z || d.ldz < d.n)) return bad_arg(at + "Z is NULL or ldz < n");
            if (back && overlaps(d.VR, d.ldvr * n * sizeof(T), d.Z, d.ldz * n * sizeof(T)))
                return bad_arg(at + "VR overlaps Z (the batched form does not work in place)");
        }
        if (left) {
            if (!d.VL || d.ldvl < d.n) return bad_arg(at + "VL is NULL or ldvl < n");
            if (back && (!d.Q || d.ldq < d.n)) return bad_arg(at + "Q is NULL or ldq < n");
            if (back && overlaps(d.VL, d.ldvl * n * sizeof(T), d.Q, d.ldq * n * sizeof(T)))
                return bad_arg(at + "VL overlaps Q (the batched form does not work in place)");
        }
    }
    if (config == 0) config = default_config(prec);
    const int nt = (int)(config >> 8);
    const int xrows = std::max(8, (nmax + 7) / 8 * 8);
    KernelFn<T> fn = nullptr;
    size_t smem = 0;
    if (!kernel_for<T>(config, xrows, &fn, &smem))
        return bad_arg("batched: unknown tile configuration " + std::to_string(config >> 8) + "x" +
                       std::to_string(config & 255u));

    xtgevc3_batch *b = new xtgevc3_batch;
    b->prec = prec;
    b->config = config;
    b->count = count;
    b->smem = smem;
    int dev = 0, sms = 0, max_smem = 0;
    XTG_BCK(cudaGetDevice(&dev));
    XTG_BCK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    XTG_BCK(cudaDeviceGetAttribute(&max_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    if (smem > (size_t)max_smem) {
        destroy(b);
        return bad_arg("batched: order " + std::to_string(nmax) + " needs " + std::to_string(smem) +
                       " bytes of shared memory per block with tiles " + std::to_string(nt) + "x" +
                       std::to_string(config & 255u) + " (the device offers " + std::to_string(max_smem) + ")");
    }
    XTG_BCK(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int occ = 0;
    XTG_BCK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fn, THREADS, smem));
    occ = std::max(occ, 1);

    // units: every prep unit first (largest pencils first), then per pencil (largest
    // first) its tiles from the last (the most work) down, both sides interleaved
    std::vector<int> order(count);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return pencils[x].n > pencils[y].n; });
    // Testing controls, read when a plan is created; neither changes anything when unset.
    //   XTGEVC3_BATCH_SPIN_LIMIT=k       polls of a pencil's ready flag (128 ns apart) before a
    //                                    compute unit gives up (default 2^24, ~2 s)
    //   XTGEVC3_BATCH_WITHHOLD_READY=p   leave out pencil p's prep unit: its ready flag is never
    //                                    set, every wait for it expires, the kernel records the
    //                                    timeout and xtgevc3_batched_wait returns 3
    long long spin_limit = 1ll << 24;
    int withhold = -1;
    if (const char *v = std::getenv("XTGEVC3_BATCH_SPIN_LIMIT")) spin_limit = std::max(1ll, std::atoll(v));
    if (const char *v = std::getenv("XTGEVC3_BATCH_WITHHOLD_READY")) withhold = std::atoi(v);
    std::vector<int4> units;
    for (int p : order)
        if (p != withhold) units.push_back(make_int4(0, p, 0, 0));
    for (int p : order) {
        const int n = pencils[p].n;
        if (n == 0) continue;
        for (int t = batch::max_tiles(n, nt) - 1; t >= 0; t--) {
            if (right) units.push_back(make_int4(1, p, 0, t));
            if (left) units.push_back(make_int4(1, p, 1, t));
        }
    }
    std::vector<long long> woff(std::max(count, 1), 0);
    size_t ws = 0;
    for (int p = 0; p < count; p++) {
        woff[p] = (long long)ws;
        ws += batch::work_layout<T>(nullptr, pencils[p].n, nt, nullptr);
    }
    b->nunits = (int)units.size();
    b->grid = std::max(1, std::min(sms * occ, b->nunits));
    XTG_BCK(cudaMalloc(&b->d_pencils, std::max<size_t>(1, count * sizeof(PencilT))));
    XTG_BCK(cudaMalloc(&b->d_units, std::max<size_t>(1, units.size()) * sizeof(int4)));
    XTG_BCK(cudaMalloc(&b->d_woff, woff.size() * sizeof(long long)));
    XTG_BCK(cudaMalloc(&b->d_ws, std::max<size_t>(ws, 256)));
    XTG_BCK(cudaMalloc(&b->d_ctrl, (2 + (size_t)count) * sizeof(int)));
    if (count) XTG_BCK(cudaMemcpy(b->d_pencils, pencils, count * sizeof(PencilT), cudaMemcpyHostToDevice));
    if (!units.empty())
        XTG_BCK(cudaMemcpy(b->d_units, units.data(), units.size() * sizeof(int4), cudaMemcpyHostToDevice));
    XTG_BCK(cudaMemcpy(b->d_woff, woff.data(), woff.size() * sizeof(long long), cudaMemcpyHostToDevice));

    batch::Args<T> a;
    a.pencils = static_cast<const PencilT *>(b->d_pencils);
    a.units = b->d_units;
    a.nunits = b->nunits;
    a.ws = b->d_ws;
    a.woff = b->d_woff;
    a.ctrl = b->d_ctrl;
    a.back = back ? 1 : 0;
    a.xrows = xrows;
    a.spin_limit = spin_limit;  // default ~2 s of 128 ns sleeps: far beyond any prep unit

    cudaStream_t cs = nullptr;
    XTG_BCK(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
    cudaError_t e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
        cudaMemsetAsync(b->d_ctrl, 0, (2 + (size_t)count) * sizeof(int), cs);
        fn<<<b->grid, THREADS, smem, cs>>>(a);
        e = cudaStreamEndCapture(cs, &b->graph);
    }
    cudaStreamDestroy(cs);
    XTG_BCK(e);
    XTG_BCK(cudaGraphInstantiate(&b->exec, b->graph, 0));
    *out = b;
    return 0;
}

template <class T>
int tune(char side, char howmny, int count, const typename batch::PencilOf<T>::type *pencils, int reps,
         unsigned *best, float *best_ms)
{
    const char prec = sizeof(T) == 8 ? 'd' : 's';
    int dev = 0, max_smem = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&max_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess) {
        set_last_error("batched tune: no CUDA device");
        return 1;
    }
    int nmax = 0;
    for (int p = 0; p < count && pencils; p++) nmax = std::max(nmax, pencils[p].n);
    const int xrows = std::max(8, (nmax + 7) / 8 * 8);
    reps = std::max(reps, 1);
    unsigned bc = 0;
    float bms = 0;
    cudaStream_t st = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess || cudaEventCreate(&e0) != cudaSuccess ||
        cudaEventCreate(&e1) != cudaSuccess) {
        set_last_error("batched tune: stream/event creation failed");
        return 1;
    }
    int rc = 0;
    for (unsigned c : kCandidates) {
        if (!fits<T>(c, xrows, max_smem)) continue;
        xtgevc3_batch *b = nullptr;
        rc = create<T>(side, howmny, count, pencils, c, &b);
        if (rc) break;
        rc = xtgevc3_batched_run(b, st);
        if (!rc) rc = xtgevc3_batched_wait(b, st);
        float ms = 0;
        if (!rc) {
            cudaEventRecord(e0, st);
            for (int r = 0; r < reps && !rc; r++) rc = xtgevc3_batched_run(b, st);
            cudaEventRecord(e1, st);
            if (!rc) rc = xtgevc3_batched_wait(b, st);
            cudaEventElapsedTime(&ms, e0, e1);
            ms /= reps;
        }
        destroy(b);
        if (rc) break;
        if (!bc || ms < bms) {
            bc = c;
            bms = ms;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaStreamDestroy(st);
    if (rc) return rc;
    if (!bc) {
        set_last_error("batched tune: no tile configuration fits this batch");
        return -1;
    }
    xtgevc3_batched_set_default(prec, bc);
    if (best) *best = bc;
    if (best_ms) *best_ms = bms;
    return 0;
}

}  // namespace

extern "C" {

int xtgevc3_dtgevc3_batched_create(char side, char howmny, int count, const xtgevc3_dpencil *pencils,
                                   unsigned config, xtgevc3_batch **plan)
{
    return create<double>(side, howmny, count, pencils, config, plan);
}

int xtgevc3_stgevc3_batched_create(char side, char howmny, int count, const xtgevc3_spencil *pencils,
                                   unsigned config, xtgevc3_batch **plan)
{
    return create<float>(side, howmny, count, pencils, config, plan);
}

int xtgevc3_batched_run(xtgevc3_batch *plan, void *stream)
{
    if (!plan) return bad_arg("batched: plan is NULL");
    cudaError_t e = cudaGraphLaunch(plan->exec, static_cast<cudaStream_t>(stream));
    if (e != cudaSuccess) {
        set_last_error(std::string("cudaGraphLaunch: ") + cudaGetErrorString(e));
        return 1;
    }
    xtg::count_launches(1);
    return 0;
}

int xtgevc3_batched_wait(xtgevc3_batch *plan, void *stream)
{
    if (!plan) return bad_arg("batched: plan is NULL");
    cudaError_t e = cudaStreamSynchronize(static_cast<cudaStream_t>(stream));
    int status = 0;
    if (e == cudaSuccess) e = cudaMemcpy(&status, plan->d_ctrl + 1, sizeof(int), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) {
        set_last_error(std::string("batched wait: ") + cudaGetErrorString(e));
        return 1;
    }
    if (status & xtg::kErrWaitTimeout) {
        set_last_error("batched: a bounded wait of the work queue expired; results are incomplete");
        return 3;
    }
    return 0;
}

void xtgevc3_batched_destroy(xtgevc3_batch *plan) { destroy(plan); }

int xtgevc3_batched_info(const xtgevc3_batch *plan, unsigned *config, int *grid, int *units)
{
    if (!plan) return bad_arg("batched: plan is NULL");
    if (config) *config = plan->config;
    if (grid) *grid = plan->grid;
    if (units) *units = plan->nunits;
    return 0;
}

int xtgevc3_dtgevc3_batched_tune(char side, char howmny, int count, const xtgevc3_dpencil *pencils, int reps,
                                 unsigned *best, float *best_ms)
{
    return tune<double>(side, howmny, count, pencils, reps, best, best_ms);
}

int xtgevc3_stgevc3_batched_tune(char side, char howmny, int count, const xtgevc3_spencil *pencils, int reps,
                                 unsigned *best, float *best_ms)
{
    return tune<float>(side, howmny, count, pencils, reps, best, best_ms);
}

void xtgevc3_batched_set_default(char prec, unsigned config)
{
    std::call_once(g_env_once, read_env);
    if (prec == 'd') g_default_d.store(config);
    if (prec == 's') g_default_s.store(config);
}

unsigned xtgevc3_batched_get_default(char prec) { return default_config(prec); }

}  // extern "C"
