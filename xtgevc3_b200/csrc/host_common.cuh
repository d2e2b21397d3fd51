// Host-side helpers shared by the drivers of the device algorithm: CUDA error checks,
// per-call scratch memory and the GEMM launcher.
#pragma once
#include "engine.cuh"
#include "kernels_gemm.cuh"

#include <string>
#include <type_traits>
#include <vector>

namespace xtg {

#define XTG_CK(call)                                                                              \
    do {                                                                                          \
        cudaError_t e_ = (call);                                                                  \
        if (e_ != cudaSuccess) {                                                                  \
            set_last_error(std::string(#call) + ": " + cudaGetErrorString(e_));                   \
            return 1;                                                                             \
        }                                                                                         \
    } while (0)

static inline int round_up(int v, int q) { return (v + q - 1) / q * q; }

// Scratch of one call.  Default: stream-ordered allocations from the device's pool (which
// keeps freed memory for reuse).  Arena mode: 256-byte aligned slices of a caller-owned
// device buffer, nothing allocated or freed; `used` can be rewound to reuse a region once
// the work using it is ordered before the next user on the same stream.
struct Scratch {
    cudaStream_t st;
    std::vector<void *> ptrs;
    cudaError_t err = cudaSuccess;
    unsigned char *arena = nullptr;
    size_t cap = 0, used = 0;
    explicit Scratch(cudaStream_t s) : st(s) {}
    Scratch(cudaStream_t s, void *a, size_t c) : st(s), arena(static_cast<unsigned char *>(a)), cap(c) {}
    template <class T>
    T *get(size_t count)
    {
        if (count == 0) count = 1;
        const size_t bytes = count * sizeof(T);
        if (arena) {
            const size_t off = (used + 255) & ~size_t(255);
            if (off + bytes > cap) {
                err = cudaErrorMemoryAllocation;
                return nullptr;
            }
            used = off + bytes;
            return reinterpret_cast<T *>(arena + off);
        }
        void *p = nullptr;
        cudaError_t e = cudaMallocAsync(&p, bytes, st);
        if (e != cudaSuccess) {
            err = e;
            return nullptr;
        }
        ptrs.push_back(p);
        return static_cast<T *>(p);
    }
    ~Scratch()
    {
        for (void *p : ptrs) cudaFreeAsync(p, st);
    }
};

template <class E>
inline void launch_gemm(const GemmArgs<E> &g, bool simt, cudaStream_t st)
{
    if constexpr (std::is_same<E, double>::value) {
        // the cp.async path copies 16-byte pairs of rows: even leading dimensions and
        // 16-byte aligned bases only (caller-given ld may be odd on the device API)
        auto al = [](const void *p) { return (reinterpret_cast<uintptr_t>(p) & 15) == 0; };
        bool ok = (g.ldb % 2 == 0) && al(g.B) && (g.C != nullptr), odd = false;
        for (int s = 0; s < g.nseg; s++) {
            ok = ok && (g.seg[s].lda % 2 == 0) && al(g.seg[s].A);
            odd = odd || (g.seg[s].boff % 2 != 0);  // B rows at an odd offset: 8-byte loads
        }
        if (!simt && ok) {
            // up to 128 output rows (the update of a group's upper block: 64 or 65): 64-row
            // tiles, so that no tile computes rows past M and twice as many CTAs share the work
            if (g.M <= 128) {
                using T = dmma::Tile<64>;
                dim3 grid((g.M + 63) / 64, (g.N + dmma::BN - 1) / dmma::BN);
                if (g.accumulate) {
                    if (odd) gemm_dmma<1, 64, true><<<grid, T::NT, T::SMEM_BYTES, st>>>(g);
                    else gemm_dmma<1, 64><<<grid, T::NT, T::SMEM_BYTES, st>>>(g);
                } else {
                    if (odd) gemm_dmma<0, 64, true><<<grid, T::NT, T::SMEM_BYTES, st>>>(g);
                    else gemm_dmma<0, 64><<<grid, T::NT, T::SMEM_BYTES, st>>>(g);
                }
                return;
            }
            using T = dmma::Tile<128>;
            dim3 grid((g.M + 127) / 128, (g.N + dmma::BN - 1) / dmma::BN);
            if (g.accumulate) {
                if (odd) gemm_dmma<1, 128, true><<<grid, T::NT, T::SMEM_BYTES, st>>>(g);
                else gemm_dmma<1><<<grid, T::NT, T::SMEM_BYTES, st>>>(g);
            } else {
                if (odd) gemm_dmma<0, 128, true><<<grid, T::NT, T::SMEM_BYTES, st>>>(g);
                else gemm_dmma<0><<<grid, T::NT, T::SMEM_BYTES, st>>>(g);
            }
            return;
        }
    }
    if constexpr (std::is_same<E, cplx<double>>::value) {
        // cp.async of 16-byte complex elements: 16-byte aligned operands only
        auto al = [](const void *p) { return (reinterpret_cast<uintptr_t>(p) & 15) == 0; };
        bool ok = al(g.B) && (g.C != nullptr) && al(g.C);
        for (int s = 0; s < g.nseg; s++) ok = ok && al(g.seg[s].A);
        if (!simt && ok) {
            dim3 grid((g.M + zmma::BM - 1) / zmma::BM, (g.N + zmma::BN - 1) / zmma::BN);
            if (g.accumulate) gemm_dmma_cplx<1><<<grid, 256, zmma::SMEM_BYTES, st>>>(g);
            else gemm_dmma_cplx<0><<<grid, 256, zmma::SMEM_BYTES, st>>>(g);
            return;
        }
    }
    dim3 grid((g.M + 63) / 64, (g.N + 63) / 64);
    gemm_simt<E><<<grid, 256, 0, st>>>(g);
}

}  // namespace xtg
