// C-ABI and C++ drop-in entry points: argument decoding, selection count, LWORK query and
// INFO codes exactly as the upstream driver (src/dtgevc3.cpp:1172-1244,
// src/ztgevc3.cpp:457-517), then host<->device staging and the device algorithm.
#include "../../include/tgevc3.h"
#include "../../include/xtgevc3.h"
#include "args.h"
#include "engine.cuh"

#include <atomic>
#include <complex>
#include <cstring>
#include <vector>

namespace {

std::atomic<unsigned> g_flags{0};

xtg::Options make_opts(unsigned flags)
{
    xtg::Options o;
    o.normalize = (flags & XTGEVC3_NORMALIZE) ? 1 : 0;
    o.simt = (flags & XTGEVC3_SIMT) ? 1 : 0;
    o.lookahead = (flags & XTGEVC3_LOOKAHEAD) ? 1 : 0;
    if (flags & XTGEVC3_SPLIT) {
        const int s = (int)((flags >> 8) & 15u);
        o.split_kind = (flags & XTGEVC3_SPLIT_INT8) ? 1 : 0;
        o.split = s > 0 ? s : (o.split_kind ? 7 : 6);
    }
    return o;
}

int req_work(int n, int bs) { return 2 * n * (bs + 1) + 4 * (bs + 1) * (bs + 1) + 2 * (bs + 1); }

using xtg::check_args;

// LWORK rule of the upstream driver (block size 32 shrunk until the workspace fits).
template <class W>
bool check_work(int n, W *work, int lwork, int *info)
{
    int bs = 32;
    int req = req_work(n, bs);
    if (lwork != -1 && lwork < req) {
        for (bs = bs - 1; bs >= 1; bs--) {
            req = req_work(n, bs);
            if (lwork >= req) break;
        }
    }
    if (lwork == -1) {
        work[0] = W(req);
        *info = 0;
        return true;
    }
    if (lwork < req) {
        *info = -19;
        return true;
    }
    *info = 0;
    return false;
}

inline int round_up(int v, int q) { return (v + q - 1) / q * q; }

// Host pointers: stage S, P (and Q/Z for HOWMNY='B') on the device, run, copy back.
template <class R, bool CPLX>
int run_host(char side, char howmny, const int *select, int n, const void *S, int lds, const void *P, int ldp,
             const void *alpha, const void *alphai, const void *beta, void *VL, int ldvl, void *VR, int ldvr,
             int count, unsigned flags)
{
    using E = typename std::conditional<CPLX, std::complex<R>, R>::type;
    const bool want_r = (side == 'R' || side == 'B') && VR;
    const bool want_l = (side == 'L' || side == 'B') && VL;
    if (!want_r && !want_l) return 0;
    const bool back = howmny == 'B';
    cudaStream_t st = cudaStreamPerThread;
    const int ld = round_up(n, 32);
    const size_t mat = (size_t)ld * n * sizeof(E);
    const size_t vcols = (size_t)std::max(count, back ? n : 0);
    void *dS = nullptr, *dP = nullptr, *dVL = nullptr, *dVR = nullptr;
    auto fail = [&](cudaError_t e, const char *what) {
        xtg::set_last_error(std::string(what) + ": " + cudaGetErrorString(e));
        if (dS) cudaFreeAsync(dS, st);
        if (dP) cudaFreeAsync(dP, st);
        if (dVL) cudaFreeAsync(dVL, st);
        if (dVR) cudaFreeAsync(dVR, st);
        cudaStreamSynchronize(st);
        return 1;
    };
    cudaError_t e;
    if ((e = cudaMallocAsync(&dS, mat, st)) != cudaSuccess) return fail(e, "cudaMallocAsync");
    if ((e = cudaMallocAsync(&dP, mat, st)) != cudaSuccess) return fail(e, "cudaMallocAsync");
    if (want_l && (e = cudaMallocAsync(&dVL, (size_t)ld * vcols * sizeof(E), st)) != cudaSuccess)
        return fail(e, "cudaMallocAsync");
    if (want_r && (e = cudaMallocAsync(&dVR, (size_t)ld * vcols * sizeof(E), st)) != cudaSuccess)
        return fail(e, "cudaMallocAsync");
    const size_t w = (size_t)n * sizeof(E);
    if ((e = cudaMemcpy2DAsync(dS, ld * sizeof(E), S, (size_t)lds * sizeof(E), w, n, cudaMemcpyHostToDevice, st)))
        return fail(e, "H2D S");
    if ((e = cudaMemcpy2DAsync(dP, ld * sizeof(E), P, (size_t)ldp * sizeof(E), w, n, cudaMemcpyHostToDevice, st)))
        return fail(e, "H2D P");
    if (back) {
        if (want_l && (e = cudaMemcpy2DAsync(dVL, ld * sizeof(E), VL, (size_t)ldvl * sizeof(E), w, n,
                                             cudaMemcpyHostToDevice, st)))
            return fail(e, "H2D Q");
        if (want_r && (e = cudaMemcpy2DAsync(dVR, ld * sizeof(E), VR, (size_t)ldvr * sizeof(E), w, n,
                                             cudaMemcpyHostToDevice, st)))
            return fail(e, "H2D Z");
    }
    int rc = xtg::solve_device<R, CPLX>(side, howmny, select, n, dS, ld, dP, ld, alpha, alphai, beta,
                                        want_l ? dVL : nullptr, ld, want_r ? dVR : nullptr, ld, count,
                                        make_opts(flags), st);
    if (rc) {
        std::string msg = xtg::last_error();
        fail(cudaSuccess, "device");
        xtg::set_last_error(msg);
        return 1;
    }
    if (want_l && (e = cudaMemcpy2DAsync(VL, (size_t)ldvl * sizeof(E), dVL, ld * sizeof(E), w, count,
                                         cudaMemcpyDeviceToHost, st)))
        return fail(e, "D2H VL");
    if (want_r && (e = cudaMemcpy2DAsync(VR, (size_t)ldvr * sizeof(E), dVR, ld * sizeof(E), w, count,
                                         cudaMemcpyDeviceToHost, st)))
        return fail(e, "D2H VR");
    cudaFreeAsync(dS, st);
    cudaFreeAsync(dP, st);
    if (dVL) cudaFreeAsync(dVL, st);
    if (dVR) cudaFreeAsync(dVR, st);
    if ((e = cudaStreamSynchronize(st)) != cudaSuccess) {
        xtg::set_last_error(std::string("cudaStreamSynchronize: ") + cudaGetErrorString(e));
        return 1;
    }
    return 0;
}

template <class R, bool CPLX, class W>
void drop_in(char side, char howmny, const int *select, int n, const void *S, int lds, const void *P, int ldp,
             const void *alpha, const R *alphai, const void *beta, void *VL, int ldvl, void *VR, int ldvr, int mm,
             int *m, W *work, int lwork, int *info)
{
    int count = 0;
    if (check_args<R>(CPLX, howmny, select, n, alphai, mm, m, info, &count)) return;
    if (check_work<W>(n, work, lwork, info)) return;
    xtg::set_last_error("");
    if (count == 0) return;
    if (run_host<R, CPLX>(side, howmny, select, n, S, lds, P, ldp, alpha, alphai, beta, VL, ldvl, VR, ldvr, count,
                          g_flags.load()))
        *info = 1;
}

template <class R, bool CPLX>
int device_form(unsigned flags, void *stream, char side, char howmny, const int *select, int n, const void *S,
                int lds, const void *P, int ldp, const void *alpha, const R *alphai, const void *beta, void *VL,
                int ldvl, void *VR, int ldvr, int mm, int *m, int *info)
{
    int count = 0;
    int dummy = 0;
    if (!info) info = &dummy;
    if (check_args<R>(CPLX, howmny, select, n, alphai, mm, m, info, &count)) return 0;
    *info = 0;
    xtg::set_last_error("");
    if (count == 0) return 0;
    int rc = xtg::solve_device<R, CPLX>(side, howmny, select, n, S, lds, P, ldp, alpha, alphai, beta, VL, ldvl, VR,
                                        ldvr, count, make_opts(flags), static_cast<cudaStream_t>(stream));
    if (rc) *info = 1;
    return rc;
}

}  // namespace

// ---------------------------------------------------------------------------------------
// C linkage
// ---------------------------------------------------------------------------------------
extern "C" {

void xtgevc3_set_flags(unsigned flags) { g_flags.store(flags); }
unsigned xtgevc3_get_flags(void) { return g_flags.load(); }
const char *xtgevc3_last_error(void) { return xtg::last_error(); }

void xtgevc3_trace_enable(int on) { xtg::trace_enable(on); }
void xtgevc3_trace_reset(void) { xtg::trace_reset(); }
int xtgevc3_trace_get(int cls, long long *launches, double *ms, double *flops, double *bytes)
{
    return xtg::trace_get(cls, launches, ms, flops, bytes);
}
const char *xtgevc3_trace_name(int cls) { return xtg::trace_name(cls); }
long long xtgevc3_launch_count(void) { return xtg::launch_count(); }

void xtgevc3_dtgevc3(char side, char howmny, const int *select, int n, const double *S, int lds, const double *P,
                     int ldp, const double *alphar, const double *alphai, const double *beta, double *VL, int ldvl,
                     double *VR, int ldvr, int mm, int *m, double *work, int lwork, int *info)
{
    drop_in<double, false, double>(side, howmny, select, n, S, lds, P, ldp, alphar, alphai, beta, VL, ldvl, VR,
                                   ldvr, mm, m, work, lwork, info);
}

void xtgevc3_stgevc3(char side, char howmny, const int *select, int n, const float *S, int lds, const float *P,
                     int ldp, const float *alphar, const float *alphai, const float *beta, float *VL, int ldvl,
                     float *VR, int ldvr, int mm, int *m, float *work, int lwork, int *info)
{
    drop_in<float, false, float>(side, howmny, select, n, S, lds, P, ldp, alphar, alphai, beta, VL, ldvl, VR, ldvr,
                                 mm, m, work, lwork, info);
}

void xtgevc3_ztgevc3(char side, char howmny, const int *select, int n, const double *S, int lds, const double *P,
                     int ldp, const double *alpha, const double *beta, double *VL, int ldvl, double *VR, int ldvr,
                     int mm, int *m, double *work, int lwork, int *info)
{
    drop_in<double, true, std::complex<double>>(side, howmny, select, n, S, lds, P, ldp, alpha, nullptr, beta, VL,
                                                ldvl, VR, ldvr, mm, m,
                                                reinterpret_cast<std::complex<double> *>(work), lwork, info);
}

void xtgevc3_ctgevc3(char side, char howmny, const int *select, int n, const float *S, int lds, const float *P,
                     int ldp, const float *alpha, const float *beta, float *VL, int ldvl, float *VR, int ldvr, int mm,
                     int *m, float *work, int lwork, int *info)
{
    drop_in<float, true, std::complex<float>>(side, howmny, select, n, S, lds, P, ldp, alpha, nullptr, beta, VL,
                                              ldvl, VR, ldvr, mm, m, reinterpret_cast<std::complex<float> *>(work),
                                              lwork, info);
}

int xtgevc3_dtgevc3_dev(unsigned flags, void *stream, char side, char howmny, const int *select, int n,
                        const double *S, int lds, const double *P, int ldp, const double *alphar,
                        const double *alphai, const double *beta, double *VL, int ldvl, double *VR, int ldvr, int mm,
                        int *m, int *info)
{
    return device_form<double, false>(flags, stream, side, howmny, select, n, S, lds, P, ldp, alphar, alphai, beta,
                                      VL, ldvl, VR, ldvr, mm, m, info);
}

int xtgevc3_stgevc3_dev(unsigned flags, void *stream, char side, char howmny, const int *select, int n,
                        const float *S, int lds, const float *P, int ldp, const float *alphar, const float *alphai,
                        const float *beta, float *VL, int ldvl, float *VR, int ldvr, int mm, int *m, int *info)
{
    return device_form<float, false>(flags, stream, side, howmny, select, n, S, lds, P, ldp, alphar, alphai, beta,
                                     VL, ldvl, VR, ldvr, mm, m, info);
}

int xtgevc3_ztgevc3_dev(unsigned flags, void *stream, char side, char howmny, const int *select, int n,
                        const double *S, int lds, const double *P, int ldp, const double *alpha, const double *beta,
                        double *VL, int ldvl, double *VR, int ldvr, int mm, int *m, int *info)
{
    return device_form<double, true>(flags, stream, side, howmny, select, n, S, lds, P, ldp, alpha, nullptr, beta,
                                     VL, ldvl, VR, ldvr, mm, m, info);
}

int xtgevc3_ctgevc3_dev(unsigned flags, void *stream, char side, char howmny, const int *select, int n,
                        const float *S, int lds, const float *P, int ldp, const float *alpha, const float *beta,
                        float *VL, int ldvl, float *VR, int ldvr, int mm, int *m, int *info)
{
    return device_form<float, true>(flags, stream, side, howmny, select, n, S, lds, P, ldp, alpha, nullptr, beta,
                                    VL, ldvl, VR, ldvr, mm, m, info);
}

}  // extern "C"

// ---------------------------------------------------------------------------------------
// C++ linkage: the upstream prototypes (include/tgevc3.h), same symbols as the CPU library
// ---------------------------------------------------------------------------------------
void dtgevc3(char side, char howmny, const int *select, int n, const double *S, int lds, const double *P, int ldp,
             const double *alphar, const double *alphai, const double *beta, double *__restrict VL, int ldvl,
             double *__restrict VR, int ldvr, int mm, int *m, double *__restrict work, int lwork, int *info)
{
    xtgevc3_dtgevc3(side, howmny, select, n, S, lds, P, ldp, alphar, alphai, beta, VL, ldvl, VR, ldvr, mm, m, work,
                    lwork, info);
}

void stgevc3(char side, char howmny, const int *select, int n, const float *S, int lds, const float *P, int ldp,
             const float *alphar, const float *alphai, const float *beta, float *__restrict VL, int ldvl,
             float *__restrict VR, int ldvr, int mm, int *m, float *__restrict work, int lwork, int *info)
{
    xtgevc3_stgevc3(side, howmny, select, n, S, lds, P, ldp, alphar, alphai, beta, VL, ldvl, VR, ldvr, mm, m, work,
                    lwork, info);
}

void ztgevc3(char side, char howmny, const int *select, int n, const std::complex<double> *S, int lds,
             const std::complex<double> *P, int ldp, const std::complex<double> *alpha,
             const std::complex<double> *beta, std::complex<double> *__restrict VL, int ldvl,
             std::complex<double> *__restrict VR, int ldvr, int mm, int *m, std::complex<double> *__restrict work,
             int lwork, int *info)
{
    xtgevc3_ztgevc3(side, howmny, select, n, reinterpret_cast<const double *>(S), lds,
                    reinterpret_cast<const double *>(P), ldp, reinterpret_cast<const double *>(alpha),
                    reinterpret_cast<const double *>(beta), reinterpret_cast<double *>(VL), ldvl,
                    reinterpret_cast<double *>(VR), ldvr, mm, m, reinterpret_cast<double *>(work), lwork, info);
}

void ctgevc3(char side, char howmny, const int *select, int n, const std::complex<float> *S, int lds,
             const std::complex<float> *P, int ldp, const std::complex<float> *alpha, const std::complex<float> *beta,
             std::complex<float> *__restrict VL, int ldvl, std::complex<float> *__restrict VR, int ldvr, int mm,
             int *m, std::complex<float> *__restrict work, int lwork, int *info)
{
    xtgevc3_ctgevc3(side, howmny, select, n, reinterpret_cast<const float *>(S), lds,
                    reinterpret_cast<const float *>(P), ldp, reinterpret_cast<const float *>(alpha),
                    reinterpret_cast<const float *>(beta), reinterpret_cast<float *>(VL), ldvl,
                    reinterpret_cast<float *>(VR), ldvr, mm, m, reinterpret_cast<float *>(work), lwork, info);
}
