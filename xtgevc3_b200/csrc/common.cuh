// Shared device/host definitions for the xTGEVC3 CUDA path (sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <cfloat>

namespace xtg {

// Complex number stored as interleaved (re, im), the layout of std::complex<R>.
template <class R>
struct alignas(2 * sizeof(R)) cplx {
    R x, y;
    cplx() = default;
    __host__ __device__ constexpr cplx(R r, R i = R(0)) : x(r), y(i) {}
};

template <class R> __host__ __device__ __forceinline__ cplx<R> operator+(cplx<R> a, cplx<R> b) { return {a.x + b.x, a.y + b.y}; }
template <class R> __host__ __device__ __forceinline__ cplx<R> operator-(cplx<R> a, cplx<R> b) { return {a.x - b.x, a.y - b.y}; }
template <class R> __host__ __device__ __forceinline__ cplx<R> operator-(cplx<R> a) { return {-a.x, -a.y}; }
template <class R> __host__ __device__ __forceinline__ cplx<R> operator*(cplx<R> a, cplx<R> b) { return {a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x}; }
template <class R> __host__ __device__ __forceinline__ cplx<R> operator*(R s, cplx<R> a) { return {s * a.x, s * a.y}; }
template <class R> __host__ __device__ __forceinline__ cplx<R> conjg(cplx<R> a) { return {a.x, -a.y}; }
template <class R> __host__ __device__ __forceinline__ R l1abs(cplx<R> a) { return fabs(a.x) + fabs(a.y); }
__host__ __device__ __forceinline__ float l1abs(cplx<float> a) { return fabsf(a.x) + fabsf(a.y); }

// Smith's algorithm for a / b (avoids the overflow of the textbook formula).
template <class R>
__host__ __device__ __forceinline__ cplx<R> cdiv(cplx<R> a, cplx<R> b)
{
    if (fabs(b.x) >= fabs(b.y)) {
        R r = b.y / b.x, d = b.x + r * b.y;
        return {(a.x + a.y * r) / d, (a.y - a.x * r) / d};
    } else {
        R r = b.x / b.y, d = b.y + r * b.x;
        return {(a.x * r + a.y) / d, (a.y * r - a.x) / d};
    }
}

template <class R> struct limits;
template <> struct limits<double> {
    static constexpr double safemin = DBL_MIN;
    static constexpr double eps = DBL_EPSILON;
    static constexpr double big = DBL_MAX;
};
template <> struct limits<float> {
    static constexpr float safemin = FLT_MIN;
    static constexpr float eps = FLT_EPSILON;
    static constexpr float big = FLT_MAX;
};

// Row-block size of the right-looking substitution (rows per diagonal block).
constexpr int kBlock = 64;
// Row blocks per group of the substitution (one trailing GEMM per group, K = 2 x its
// rows): FP64 DMMA updates, and the split-precision updates, whose per-tile fixed costs a
// longer K amortises.
constexpr int kGroupBlocks = 2;
constexpr int kGroupBlocksSplit = 8;
// K-granule of the update GEMM; each half of the stacked update operand is padded to it.
constexpr int kKPad = 16;

// Column kinds of the computed eigenvector matrix X (real arithmetic only).
enum : uint8_t { kReal = 0, kPairRe = 1, kPairIm = 2 };

// Status word written by kernels (bit flags), read back by the host after a call.
enum : int { kErrNone = 0, kErrWaitTimeout = 1, kErrBadShape = 2 };

}  // namespace xtg
