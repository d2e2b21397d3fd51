// Allocation-free device entry point: xtgevc3_dtgevc3_dev_noalloc.
//
// Who needs it: code that must not call cudaMalloc (or any allocating routine) at the
// point where it computes eigenvectors -- for example an application whose framework
// has already reserved the device memory for its own pool, a real-time loop where a
// device allocation (which may synchronise the device) is not acceptable, or a library
// invoked from inside another allocator's bookkeeping.  The regular device entry point
// takes its scratch from the CUDA stream-ordered pool; this one takes it from a fixed
// block of device memory that is part of the library image.
//
// The block: g_noalloc_scratch below, kNoAllocBytes = 8 MiB, declared at file scope.
// Every GPU on which the library is loaded holds these 8 MiB until the process exits.
// That bounds the problem size: a call is accepted when the scratch it needs fits
// (arena_bytes_needed); for SIDE='B', HOWMNY='B' that is n <= 478.  Larger calls are
// rejected before any device work with return code 2 and a message in
// xtgevc3_last_error().
//
// Host code cannot use the symbol's name as a device address (it names a host-side
// shadow), so the address is looked up with cudaGetSymbolAddress once per device, with
// that device current, on the first call made on it.  A lookup that fails is not
// remembered: the next call on that device tries again.  Every call blocks the calling
// thread until its result is complete (it synchronises its stream), so the entry point
// cannot be used inside a stream capture.
//
// All calls share the one block, and it keeps whatever the previous call left in it: the
// computation zeroes what must start at zero itself.  Two calls whose work overlaps on the
// GPU (different streams without ordering, several host threads) race on the block; the
// caller must order them, e.g. issue them on one stream.
#include "../../include/xtgevc3.h"
#include "args.h"
#include "engine.cuh"

#include <cstdio>
#include <mutex>
#include <string>

namespace {

constexpr size_t kNoAllocBytes = size_t(8) << 20;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

constexpr int kMaxDevices = 64;
std::mutex g_addr_mu;
void *g_addr[kMaxDevices];  // device address of the block, per device; set once a lookup succeeds

// The largest order n whose SIDE='B', HOWMNY='B' call fits the block (all eigenvectors).
int max_order_both_sides()
{
    static const int nmax = [] {
        int n = 1;
        while (xtg::arena_bytes_needed(n + 1, n + 1, true, true, true, false, false, sizeof(double)) <= kNoAllocBytes)
            n++;
        return n;
    }();
    return nmax;
}

// Device address of the block on device `dev` (current), looked up on first use.
cudaError_t scratch_address(int dev, void **addr)
{
    std::lock_guard<std::mutex> lk(g_addr_mu);
    if (!g_addr[dev]) {
        void *p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) {
            cudaGetLastError();  // the failed lookup is not left pending for later calls
            return e != cudaSuccess ? e : cudaErrorInvalidSymbol;
        }
        g_addr[dev] = p;
    }
    *addr = g_addr[dev];
    return cudaSuccess;
}

}  // namespace

extern "C" int xtgevc3_dtgevc3_dev_noalloc(void *stream, char side, char howmny, const int *select, int n,
                                           const double *S, int lds, const double *P, int ldp, const double *alphar,
                                           const double *alphai, const double *beta, double *VL, int ldvl,
                                           double *VR, int ldvr, int mm, int *m, int *info)
{
    int dummy = 0;
    if (!info) info = &dummy;
    int count = 0;
    if (xtg::check_args<double>(false, howmny, select, n, alphai, mm, m, info, &count)) return 0;
    *info = 0;
    xtg::set_last_error("");
    if (count == 0) return 0;

    const bool right = (side == 'R' || side == 'B') && VR;
    const bool left = (side == 'L' || side == 'B') && VL;
    if (!right && !left) return 0;
    const size_t need = xtg::arena_bytes_needed(n, count, right, left, howmny == 'B', false, false, sizeof(double));
    if (need > kNoAllocBytes) {
        char msg[256];
        std::snprintf(msg, sizeof msg,
                      "xtgevc3_dtgevc3_dev_noalloc: n=%d with %d eigenvector columns needs %zu bytes of scratch; "
                      "the static scratch holds %zu bytes (SIDE='B', HOWMNY='B': n <= %d)",
                      n, count, need, kNoAllocBytes, max_order_both_sides());
        xtg::set_last_error(msg);
        return 2;
    }

    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
        xtg::set_last_error(std::string("xtgevc3_dtgevc3_dev_noalloc: cudaGetDevice: ") + cudaGetErrorString(e));
        *info = 1;
        return 1;
    }
    void *scratch = nullptr;
    e = scratch_address(dev, &scratch);
    if (e != cudaSuccess) {
        xtg::set_last_error(std::string("xtgevc3_dtgevc3_dev_noalloc: cudaGetSymbolAddress: ") +
                            cudaGetErrorString(e));
        *info = 1;
        return 1;
    }

    xtg::Options opt;
    opt.arena = scratch;
    opt.arena_bytes = kNoAllocBytes;
    const int rc = xtg::solve_device<double, false>(side, howmny, select, n, S, lds, P, ldp, alphar, alphai, beta,
                                                    left ? VL : nullptr, ldvl, right ? VR : nullptr, ldvr, count, opt,
                                                    static_cast<cudaStream_t>(stream));
    if (rc) *info = 1;
    return rc;
}
