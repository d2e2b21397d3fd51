// C-ABI and C++ drop-in entry points: argument decoding, selection count, LWORK query and
// INFO codes exactly as the upstream driver (src/dtgevc3.cpp:1172-1244,
// src/ztgevc3.cpp:457-517), then host<->device staging and the device algorithm.
#include "../../include/tgevc3.h"
#include "../../include/xtgevc3.h"
#include "args.h"
#include "engine.cuh"

#include <algorithm>
#include <atomic>
#include <cctype>
#include <climits>
#include <cmath>
#include <cstdint>
#include <complex>
#include <cstdlib>
#include <cstring>
#include <thread>
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
        const int s = (int)((flags >> 8) & 31u);
        o.split_kind = (flags & XTGEVC3_SPLIT_CRT) ? 2 : (flags & XTGEVC3_SPLIT_INT8) ? 1 : 0;
        o.split = s > 0 ? s : (o.split_kind == 2 ? 14 : o.split_kind ? 7 : 6);
        o.refine = (flags & XTGEVC3_SPLIT_NO_REFINE) ? 0 : 1;
        if (const char *v = std::getenv("XTGEVC3_REFINE_BOUND")) o.refine_bound = std::atof(v);
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

// Sum of |a[0..last]| as the device reduction forms it (colsum_kernel): 32 partial sums over
// rows l, l + 32, ... in increasing row order, then the xor butterfly of its shuffles.  The
// same additions in the same order give the same value, bit for bit.
template <class R>
R col_abs_sum(const R *a, int last)
{
    R s[32] = {};
    int r0 = 0;
    for (; r0 + 32 <= last + 1; r0 += 32)
        for (int l = 0; l < 32; l++) s[l] += std::fabs(a[r0 + l]);
    for (int l = 0; r0 + l <= last; l++) s[l] += std::fabs(a[r0 + l]);
    for (int o = 16; o > 0; o >>= 1) {
        R t[32];
        for (int l = 0; l < 32; l++) t[l] = s[l] + s[l ^ o];
        std::copy(t, t + 32, s);
    }
    return s[0];
}

// anorm, bnorm of a real pencil (column sums over rows <= col + 1, then their maximum, as
// colsum_kernel and colmax_kernel compute them), on host threads that run while the call
// queues its work; P = nullptr is the identity (every column sums to 1).
template <class R>
struct HostNorms {
    const R *S = nullptr, *P = nullptr;
    int lds = 0, ldp = 0, n = 0;
    std::vector<R> sums;
    std::vector<std::thread> th;
    bool partial = false;  // a thread could not be started: finish() sums every column itself
    void columns(int t, int nt)
    {
        for (int j0 = 64 * t; j0 < n; j0 += 64 * nt)
            for (int j = j0; j < std::min(n, j0 + 64); j++) {
                const int last = std::min(j + 1, n - 1);
                sums[j] = col_abs_sum(S + (size_t)j * lds, last);
                sums[(size_t)n + j] = P ? col_abs_sum(P + (size_t)j * ldp, last) : R(1);
            }
    }
    void start(const R *S_, int lds_, const R *P_, int ldp_, int n_)
    {
        S = S_, P = P_, lds = lds_, ldp = ldp_, n = n_;
        sums.assign(2 * (size_t)n, R(0));
        const int hw = (int)std::thread::hardware_concurrency();
        const int nt = std::max(1, std::min({hw > 0 ? hw : 1, 32, (n + 63) / 64}));
        try {
            for (int t = 0; t < nt; t++) th.emplace_back([this, t, nt] { columns(t, nt); });
        } catch (...) {
            partial = true;
        }
    }
    void join()
    {
        for (auto &x : th)
            if (x.joinable()) x.join();
        th.clear();
    }
    void finish(double *out)
    {
        join();
        if (partial) columns(0, 1);
        R a = 0, b = 0;
        for (int j = 0; j < n; j++) {
            a = std::fmax(a, sums[j]);
            b = std::fmax(b, sums[(size_t)n + j]);
        }
        out[0] = a;
        out[1] = b;
    }
    ~HostNorms() { join(); }
};

// Host pointers: stage S, P (and Q/Z for HOWMNY='B') on the device, run, copy back.
// S and P travel as their upper trapezoid only (every kernel reads rows <= col + 1), in
// pieces; the device copies are zeroed first so the rest holds no garbage.  Real types: the
// pieces go up on the input stream while the call runs, after its small copies: column
// panels from the right (the right side's groups read columns right to left) alternating
// with row strips from the top (the left side's groups read rows top to bottom), each
// piece what the ones before left of the trapezoid; every group waits for the pieces it
// reads, and the norms come from host threads.  Complex types: column panels on the call's
// stream before the solve.  Q and Z upload on the input stream behind S and P (each side's
// back-transform waits for its matrix), and each side's result downloads on a third stream
// as soon as that side's kernels are queued, behind the other side's work.
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
    const int ld = round_up(n, 32);
    const size_t mat = (size_t)ld * n * sizeof(E);
    const size_t vcols = (size_t)std::max(count, back ? n : 0);
    struct Res {
        cudaStream_t st = nullptr, sin = nullptr, sout = nullptr;
        cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};  // Z ready, Q ready, right done, left done
        std::vector<cudaEvent_t> pev;  // piece k of S and P on the device (real types)
        std::vector<cudaEvent_t> zev, qev;  // row panel k of Z / Q on the device (HOWMNY='B')
        void *dS = nullptr, *dP = nullptr, *dVL = nullptr, *dVR = nullptr;
        ~Res()
        {
            // every stream is synchronised before its buffers go
            for (cudaStream_t q : {st, sin, sout})
                if (q) cudaStreamSynchronize(q);
            for (void *p : {dS, dP, dVL, dVR})
                if (p) cudaFree(p);
            for (cudaEvent_t e : ev)
                if (e) cudaEventDestroy(e);
            for (auto *v : {&pev, &zev, &qev})
                for (cudaEvent_t e : *v)
                    if (e) cudaEventDestroy(e);
            for (cudaStream_t q : {st, sin, sout})
                if (q) cudaStreamDestroy(q);
        }
    } r;
    auto fail = [&](cudaError_t e, const char *what) {
        xtg::set_last_error(std::string(what) + ": " + cudaGetErrorString(e));
        return 1;
    };
    constexpr bool kPanels = !CPLX;  // S, P go up behind the solve, norms from the host
    HostNorms<R> hn;                 // its threads read only the caller's S and P
    if constexpr (kPanels) hn.start(static_cast<const R *>(S), lds, static_cast<const R *>(P), ldp, n);
    cudaError_t e;
    // The call's stream (the right side's kernels) at the highest priority: with both sides
    // requested, the right side finishes first and its result goes down while the left side
    // (on a pooled side stream at the default priority) still computes.
    int prio_lo = 0, prio_hi = 0;
    if ((e = cudaDeviceGetStreamPriorityRange(&prio_lo, &prio_hi)) != cudaSuccess) return fail(e, "stream priorities");
    if ((e = cudaStreamCreateWithPriority(&r.st, cudaStreamNonBlocking, prio_hi)) != cudaSuccess)
        return fail(e, "stream");
    for (cudaStream_t *q : {&r.sin, &r.sout})
        if ((e = cudaStreamCreateWithFlags(q, cudaStreamNonBlocking)) != cudaSuccess) return fail(e, "stream");
    for (cudaEvent_t &ev : r.ev)
        if ((e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming)) != cudaSuccess) return fail(e, "event");
    if ((e = cudaMallocAsync(&r.dS, mat, r.st)) != cudaSuccess) return fail(e, "cudaMallocAsync");
    // P = nullptr: the standard problem (P = I, built by the solver)
    if (P && (e = cudaMallocAsync(&r.dP, mat, r.st)) != cudaSuccess) return fail(e, "cudaMallocAsync");
    if (want_l && (e = cudaMallocAsync(&r.dVL, (size_t)ld * vcols * sizeof(E), r.st)) != cudaSuccess)
        return fail(e, "cudaMallocAsync");
    if (want_r && (e = cudaMallocAsync(&r.dVR, (size_t)ld * vcols * sizeof(E), r.st)) != cudaSuccess)
        return fail(e, "cudaMallocAsync");
    const int panel = 512;
    // rows [r0, r1) x columns [c0, c1) of S or P, on stream q
    auto put = [&](int which, int r0, int r1, int c0, int c1, cudaStream_t q) {
        void *dst = which ? r.dP : r.dS;
        const void *src = which ? P : S;
        const int lsrc = which ? ldp : lds;
        return cudaMemcpy2DAsync(static_cast<E *>(dst) + (size_t)r0 + (size_t)c0 * ld, ld * sizeof(E),
                                 static_cast<const E *>(src) + (size_t)r0 + (size_t)c0 * lsrc, (size_t)lsrc * sizeof(E),
                                 (size_t)(r1 - r0) * sizeof(E), c1 - c0, cudaMemcpyHostToDevice, q);
    };
    for (int which = 0; which < (P ? 2 : 1); which++) {
        if ((e = cudaMemsetAsync(which ? r.dP : r.dS, 0, mat, r.st)) != cudaSuccess) return fail(e, "cudaMemsetAsync");
        if (!kPanels)
            for (int j0 = 0; j0 < n; j0 += panel) {
                const int j1 = std::min(n, j0 + panel);
                if ((e = put(which, 0, std::min(n, j1 + 1), j0, j1, r.st)) != cudaSuccess)
                    return fail(e, which ? "H2D P" : "H2D S");
            }
    }
    // Upload plan of the trapezoid (rows <= col + 1), real types.  State (cf, rt): columns >= cf
    // and rows < rt are on the device; what is left is rows >= rt of columns < cf, nonempty
    // while 1 <= cf and rt <= cf.  A column panel takes columns [cf - panel, cf) from row rt
    // down; a row strip takes rows [rt, rt + panel) of columns [rt - 1, cf).  Each piece
    // records the state after it.
    struct Piece {
        int r0, r1, c0, c1, cfrom, rto;
    };
    std::vector<Piece> plan;
    if (kPanels) {
        int cf = n, rt = 0;
        while (cf >= 1 && rt <= cf) {
            const int c0 = std::max(cf - panel, 0), rhi = std::min(n, cf + 1);
            plan.push_back({rt, rhi, c0, cf, c0, rt});
            cf = c0;
            if (!(cf >= 1 && rt <= cf)) break;
            const int r1 = std::min(rt + panel, n), cl = std::max(rt - 1, 0);
            plan.push_back({rt, r1, cl, cf, cf, r1});
            rt = r1;
        }
        r.pev.assign(plan.size(), nullptr);
        for (cudaEvent_t &ev : r.pev)
            if ((e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming)) != cudaSuccess) return fail(e, "event");
    }
    // Row panels of Z and Q (HOWMNY='B'): uploaded alternately behind S and P; the
    // back-transform of a side follows its panels, and each panel's rows of the result go
    // down at once (without normalisation, which needs whole columns).
    std::vector<int> qz_end;  // end row of panel k
    if (back) {
        // panel boundaries at multiples of 64 rows (the GEMM operands stay aligned)
        const int np = std::max(1, std::min(4, n / 2048));
        for (int k = 1; k < np; k++) qz_end.push_back((int)((long long)n * k / np) / 64 * 64);
        qz_end.push_back(n);
        r.zev.assign(np, nullptr);
        r.qev.assign(np, nullptr);
        for (auto *v : {&r.zev, &r.qev})
            for (cudaEvent_t &ev : *v)
                if ((e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming)) != cudaSuccess) return fail(e, "event");
    }
    xtg::Options opt = make_opts(flags);
    if (!P) {  // xTREVC3 conventions
        opt.p_identity = 1;
        opt.lapack_pairs = 1;
        opt.normalize = 1;
    }
    // The input stream's copies (S and P of real pencils, then Q and Z) go after every copy
    // that the solve's first kernels need: the eigenvalues and the column lists (the solver
    // calls `staged` once those are queued).  Queued earlier, their elements would hold those
    // small copies behind them on the copy engine; Q and Z, which only the back-transforms
    // need, go last so as not to split the link's bandwidth with S and P.  The wait also
    // orders the input stream after the zeroing of S and P and the allocations of the
    // buffers it writes.
    cudaError_t in_err = cudaSuccess;
    // stream q waits for the first piece after which `done` holds (columns [col, n) or rows
    // [0, rows) all up; the last piece completes everything).  Function scope: opt's hooks
    // below call it from inside the solve.
    auto wait_piece = [&](cudaStream_t q, auto done) -> int {
        if (plan.empty()) return -1;
        size_t k = 0;
        while (k + 1 < plan.size() && !done(plan[k])) k++;
        cudaError_t x = cudaStreamWaitEvent(q, r.pev[k], 0);
        if (x != cudaSuccess) in_err = x;
        return (int)k;
    };
    if (kPanels) {
        opt.host_S = S;
        opt.host_lds = lds;
        opt.host_norms = [&](double *out) { hn.finish(out); };
        opt.cols_ready = [&](bool, int col, cudaStream_t q) {
            wait_piece(q, [&](const Piece &p) { return p.cfrom <= col; });
        };
        opt.rows_ready = [&](int rows, cudaStream_t q) {
            const int k = wait_piece(q, [&](const Piece &p) { return p.rto >= rows; });
            return (k < 0 || k + 1 == (int)plan.size()) ? n : plan[k].rto;
        };
    }
    if (back || kPanels) {
        opt.back_ready[0] = back && want_r ? r.ev[0] : nullptr;
        opt.back_ready[1] = back && want_l ? r.ev[1] : nullptr;
        opt.staged = [&](cudaStream_t sst) {
            cudaError_t x = cudaEventRecord(r.ev[2], sst);
            if (x == cudaSuccess) x = cudaStreamWaitEvent(r.sin, r.ev[2], 0);
            for (size_t k = 0; k < plan.size() && x == cudaSuccess; k++) {
                const Piece &p = plan[k];
                x = put(0, p.r0, p.r1, p.c0, p.c1, r.sin);
                if (x == cudaSuccess && P) x = put(1, p.r0, p.r1, p.c0, p.c1, r.sin);
                if (x == cudaSuccess) x = cudaEventRecord(r.pev[k], r.sin);
            }
            if (!back) {
                if (x != cudaSuccess) in_err = x;
                return;
            }
            // row panels of Z, then of Q (the right side, first to finish, needs Z first);
            // ev[0] / ev[1]: all of Z / Q
            for (int s = 0; s < 2 && x == cudaSuccess; s++) {
                const bool lq = s == 1;
                if (!(lq ? want_l : want_r)) continue;
                for (size_t k = 0; k < qz_end.size() && x == cudaSuccess; k++) {
                    const int r0 = k ? qz_end[k - 1] : 0, r1 = qz_end[k];
                    E *dv = static_cast<E *>(lq ? r.dVL : r.dVR);
                    const E *hv = static_cast<const E *>(lq ? VL : VR);
                    const int ldh = lq ? ldvl : ldvr;
                    x = cudaMemcpy2DAsync(dv + r0, ld * sizeof(E), hv + r0, (size_t)ldh * sizeof(E),
                                          (size_t)(r1 - r0) * sizeof(E), n, cudaMemcpyHostToDevice, r.sin);
                    if (x == cudaSuccess) x = cudaEventRecord((lq ? r.qev : r.zev)[k], r.sin);
                }
            }
            if (x == cudaSuccess && want_r) x = cudaEventRecord(r.ev[0], r.sin);
            if (x == cudaSuccess && want_l) x = cudaEventRecord(r.ev[1], r.sin);
            if (x != cudaSuccess) in_err = x;
        };
    }
    cudaError_t out_err = cudaSuccess;
    // download output columns [o0, o1) of one side once its stream reaches this point
    std::vector<std::pair<bool, int>> chunked;  // sides whose columns went out in chunks
    auto download = [&](bool left, cudaStream_t sst, int o0, int o1) {
        cudaEvent_t ev = r.ev[left ? 3 : 2];
        E *hv = static_cast<E *>(left ? VL : VR);
        const int ldh = left ? ldvl : ldvr;
        const E *dv = static_cast<const E *>(left ? r.dVL : r.dVR);
        cudaError_t x = cudaEventRecord(ev, sst);
        if (x == cudaSuccess) x = cudaStreamWaitEvent(r.sout, ev, 0);
        if (x == cudaSuccess && o1 > o0)
            x = cudaMemcpy2DAsync(hv + (size_t)o0 * ldh, (size_t)ldh * sizeof(E), dv + (size_t)o0 * ld,
                                  ld * sizeof(E), (size_t)n * sizeof(E), o1 - o0, cudaMemcpyDeviceToHost, r.sout);
        if (x != cudaSuccess) out_err = x;
    };
    if (back) opt.cols_done = [&](bool left, cudaStream_t sst, int o0, int o1) {
        download(left, sst, o0, o1);
        chunked.push_back({left, o1 - o0});
    };
    // rows [r0, r1) of every output column of one side, once its stream reaches this point
    int rows_down[2] = {0, 0};
    if (back && !qz_end.empty()) {
        opt.back_rows_ready = [&](bool left, int rows, cudaStream_t q) -> int {
            size_t k = 0;
            while (k + 1 < qz_end.size() && qz_end[k] < rows) k++;
            cudaError_t x = cudaStreamWaitEvent(q, (left ? r.qev : r.zev)[k], 0);
            if (x != cudaSuccess) in_err = x;
            return qz_end[k];
        };
        opt.rows_done = [&](bool left, cudaStream_t sst, int r0, int r1) {
            cudaEvent_t ev = r.ev[left ? 3 : 2];
            E *hv = static_cast<E *>(left ? VL : VR);
            const int ldh = left ? ldvl : ldvr;
            const E *dv = static_cast<const E *>(left ? r.dVL : r.dVR);
            cudaError_t x = cudaEventRecord(ev, sst);
            if (x == cudaSuccess) x = cudaStreamWaitEvent(r.sout, ev, 0);
            if (x == cudaSuccess && r1 > r0 && count > 0)
                x = cudaMemcpy2DAsync(hv + r0, (size_t)ldh * sizeof(E), dv + r0, ld * sizeof(E),
                                      (size_t)(r1 - r0) * sizeof(E), count, cudaMemcpyDeviceToHost, r.sout);
            if (x != cudaSuccess) out_err = x;
            rows_down[left ? 1 : 0] += r1 - r0;
        };
    }
    opt.side_done = [&](bool left, cudaStream_t sst) {
        if (rows_down[left ? 1 : 0] >= n) return;  // every row went down with its panel
        int done = 0;
        for (auto &c : chunked)
            if (c.first == left) done += c.second;
        if (done < count) download(left, sst, 0, count);
    };
    int rc = xtg::solve_device<R, CPLX>(side, howmny, select, n, r.dS, ld, r.dP, ld, alpha, alphai, beta,
                                        want_l ? r.dVL : nullptr, ld, want_r ? r.dVR : nullptr, ld, count, opt, r.st);
    if (rc) return 1;
    if (in_err != cudaSuccess) return fail(in_err, "H2D of S, P, Q, Z or a wait for it");
    if (out_err != cudaSuccess) return fail(out_err, "D2H");
    if ((e = cudaStreamSynchronize(r.sout)) != cudaSuccess) return fail(e, "cudaStreamSynchronize");
    cudaFreeAsync(r.dS, r.st);
    cudaFreeAsync(r.dP, r.st);
    if (r.dVL) cudaFreeAsync(r.dVL, r.st);
    if (r.dVR) cudaFreeAsync(r.dVR, r.st);
    r.dS = r.dP = r.dVL = r.dVR = nullptr;
    if ((e = cudaStreamSynchronize(r.st)) != cudaSuccess) return fail(e, "cudaStreamSynchronize");
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

// ---- standard problem: xTREVC3 ------------------------------------------------------------
// Eigenvectors of an upper quasi-triangular Schur factor T (T = Q^H A Q from LAPACK xHSEQR /
// xGEES) with LAPACK xTREVC3's argument meaning, INFO codes and output: the generalized
// solver with P = I and beta = 1 (P built on the device, its zero strips skipped), every
// eigenvector normalised to max |re| + |im| = 1, real pairs with LAPACK's phase.

// Eigenvalues from T's diagonal blocks.  A 2x2 block (k, k+1) is LAPACK-standardised
// (T(k,k) = T(k+1,k+1)): alpha = T(k,k) +- i sqrt|T(k,k+1)| sqrt|T(k+1,k)|, as xTREVC3 takes
// them.  d: the diagonal (complex: interleaved); sub, sup: sub- and superdiagonal (real).
template <class R, bool CPLX>
void trevc3_eigs(int n, const std::vector<R> &d, const std::vector<R> &sub, const std::vector<R> &sup,
                 std::vector<R> &alpha, std::vector<R> &alphai, std::vector<R> &beta)
{
    if constexpr (CPLX) {
        alpha = d;
        beta.assign(2 * (size_t)n, R(0));
        for (int k = 0; k < n; k++) beta[2 * (size_t)k] = R(1);
        alphai.clear();
    } else {
        alpha.assign(n, R(0));
        alphai.assign(n, R(0));
        beta.assign(n, R(1));
        for (int k = 0; k < n;) {
            alpha[k] = d[k];
            if (k + 1 < n && sub[k] != R(0)) {
                const R wi = std::sqrt(std::abs(sup[k])) * std::sqrt(std::abs(sub[k]));
                alpha[k + 1] = d[k];
                alphai[k] = wi;
                alphai[k + 1] = -wi;
                k += 2;
            } else {
                k += 1;
            }
        }
    }
}

// LAPACK xTREVC3's checks that need no eigenvalues, in its order (-1 SIDE, -2 HOWMNY, -4 N,
// -6 LDT, -8 LDVL, -10 LDVR); -11 (MM < M) follows once M is known.
inline int trevc3_pre(char side, char howmny, int n, int ldt, int ldvl, int ldvr)
{
    const bool rightv = side == 'R' || side == 'B', leftv = side == 'L' || side == 'B';
    if (!rightv && !leftv) return -1;
    if (howmny != 'A' && howmny != 'B' && howmny != 'S') return -2;
    if (n < 0) return -4;
    if (ldt < std::max(1, n)) return -6;
    if (ldvl < 1 || (leftv && ldvl < n)) return -8;
    if (ldvr < 1 || (rightv && ldvr < n)) return -10;
    return 0;
}

// M: selected eigenvectors (a pair counts twice when either of its flags is set)
template <class R, bool CPLX>
int trevc3_count(char howmny, const int *select, int n, const std::vector<R> &alphai)
{
    int num = 0;
    for (int k = 0; k < n;) {
        const bool pair = !CPLX && alphai[k] != R(0) && k + 1 < n;
        bool sel = howmny != 'S';
        if (!sel) sel = select && (select[k] != 0 || (pair && select[k + 1] != 0));
        if (sel) num += pair ? 2 : 1;
        k += pair ? 2 : 1;
    }
    return num;
}

// diagonal, sub- and superdiagonal of T (host or device memory)
template <class R, bool CPLX>
int trevc3_diagonals(const void *T, int ldt, int n, bool on_device, cudaStream_t st, std::vector<R> &d,
                     std::vector<R> &sub, std::vector<R> &sup)
{
    const int w = CPLX ? 2 : 1;  // reals per element
    d.assign((size_t)w * n, R(0));
    sub.assign(std::max(0, n - 1), R(0));
    sup.assign(std::max(0, n - 1), R(0));
    const R *t = static_cast<const R *>(T);
    const size_t step = (size_t)w * (ldt + 1);
    if (!on_device) {
        for (int k = 0; k < n; k++)
            for (int q = 0; q < w; q++) d[(size_t)w * k + q] = t[step * k + q];
        if constexpr (!CPLX)
            for (int k = 0; k + 1 < n; k++) {
                sub[k] = t[step * k + 1];
                sup[k] = t[step * k + ldt];
            }
        return 0;
    }
    cudaError_t e = cudaMemcpy2DAsync(d.data(), w * sizeof(R), t, step * sizeof(R), w * sizeof(R), n,
                                      cudaMemcpyDeviceToHost, st);
    if (!CPLX && n > 1 && e == cudaSuccess)
        e = cudaMemcpy2DAsync(sub.data(), sizeof(R), t + 1, step * sizeof(R), sizeof(R), n - 1, cudaMemcpyDeviceToHost,
                              st);
    if (!CPLX && n > 1 && e == cudaSuccess)
        e = cudaMemcpy2DAsync(sup.data(), sizeof(R), t + ldt, step * sizeof(R), sizeof(R), n - 1,
                              cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
        xtg::set_last_error(std::string("xTREVC3 diagonal of T: ") + cudaGetErrorString(e));
        return 1;
    }
    return 0;
}

// Host form (LWORK >= max(1, 3n) real / max(1, 2n) complex, LRWORK >= max(1, n) complex;
// work is not used, and a query answers those minima).
template <class R, bool CPLX, class W>
void trevc3_host(char side, char howmny, const int *select, int n, const void *T, int ldt, void *VL, int ldvl,
                 void *VR, int ldvr, int mm, int *m, W *work, int lwork, R *rwork, int lrwork, int *info)
{
    side = (char)std::toupper((unsigned char)side);
    howmny = (char)std::toupper((unsigned char)howmny);
    const int minw = std::max(1, (CPLX ? 2 : 3) * n), minrw = std::max(1, n);
    const bool lquery = lwork == -1 || (CPLX && lrwork == -1);
    if (work) work[0] = W(minw);
    if (CPLX && rwork) rwork[0] = R(minrw);
    xtg::set_last_error("");
    *info = trevc3_pre(side, howmny, n, ldt, ldvl, ldvr);
    if (*info) return;
    std::vector<R> d, sub, sup, alpha, alphai, beta;
    trevc3_diagonals<R, CPLX>(T, ldt, n, false, nullptr, d, sub, sup);
    trevc3_eigs<R, CPLX>(n, d, sub, sup, alpha, alphai, beta);
    const int count = trevc3_count<R, CPLX>(howmny, select, n, alphai);
    if (m) *m = count;
    if (mm < count) *info = -11;
    else if (lwork < minw && !lquery) *info = -14;
    else if (CPLX && lrwork < minrw && !lquery) *info = -16;
    if (*info || lquery || count == 0) return;
    if (run_host<R, CPLX>(side, howmny, select, n, T, ldt, nullptr, 0, alpha.data(), CPLX ? nullptr : alphai.data(),
                          beta.data(), VL, ldvl, VR, ldvr, count, g_flags.load()))
        *info = 1;
}

// Device form: T, VL, VR on the current device, select on the host.
template <class R, bool CPLX>
int trevc3_device(unsigned flags, void *stream, char side, char howmny, const int *select, int n, const void *T,
                  int ldt, void *VL, int ldvl, void *VR, int ldvr, int mm, int *m, int *info)
{
    int dummy = 0;
    if (!info) info = &dummy;
    side = (char)std::toupper((unsigned char)side);
    howmny = (char)std::toupper((unsigned char)howmny);
    xtg::set_last_error("");
    *info = trevc3_pre(side, howmny, n, ldt, ldvl, ldvr);
    if (*info) return 0;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    std::vector<R> d, sub, sup, alpha, alphai, beta;
    if (n > 0 && trevc3_diagonals<R, CPLX>(T, ldt, n, true, st, d, sub, sup)) {
        *info = 1;
        return 1;
    }
    trevc3_eigs<R, CPLX>(n, d, sub, sup, alpha, alphai, beta);
    const int count = trevc3_count<R, CPLX>(howmny, select, n, alphai);
    if (m) *m = count;
    if (mm < count) {
        *info = -11;
        return 0;
    }
    if (count == 0) return 0;
    xtg::Options opt = make_opts(flags);
    opt.p_identity = 1;
    opt.lapack_pairs = 1;
    opt.normalize = 1;
    const int rc = xtg::solve_device<R, CPLX>(side, howmny, select, n, T, ldt, nullptr, 0, alpha.data(),
                                              CPLX ? nullptr : alphai.data(), beta.data(), VL, ldvl, VR, ldvr, count,
                                              opt, st);
    if (rc) *info = 1;
    return rc;
}

// ---- condition numbers: xTGSNA --------------------------------------------------------------
// LAPACK xTGSNA's arguments and INFO order.  S (JOB = 'E' / 'B') from the eigenvectors; DIF
// (JOB = 'V' / 'B'): a reordered copy per eigenvalue and xTGSYL's estimate (tgsna_dif.cu).  A
// real pair is A(k+1, k) != 0.
// argument checks that need no data, in LAPACK's order
inline int tgsna_check(char job, char howmny, int n, int lda, int ldb, int ldvl, int ldvr, bool cplx)
{
    (void)cplx;
    if (job != 'E' && job != 'V' && job != 'B') return -1;
    const bool wants = job != 'V';
    if (howmny != 'A' && howmny != 'S') return -2;
    if (n < 0) return -4;
    if (lda < std::max(1, n)) return -6;
    if (ldb < std::max(1, n)) return -8;
    if (wants && ldvl < n) return -10;
    if (wants && ldvr < n) return -12;
    return 0;
}

// M and the eigenvalue list (sub: A's subdiagonal, n - 1 entries, real pencils); -15 if MM < M
template <class R, bool CPLX>
int tgsna_plan(char howmny, const int *select, int n, int mm, const std::vector<R> &sub, int *m,
               std::vector<int> &items, std::vector<uint8_t> &kinds, std::vector<int> *rows = nullptr)
{
    int ks = 0;
    for (int k = 0; k < n;) {
        const bool pair = !CPLX && k + 1 < n && sub[k] != R(0);
        const bool sel = howmny == 'A' || (select && (select[k] != 0 || (pair && select[k + 1] != 0)));
        if (sel) {
            items.push_back(ks);
            kinds.push_back(CPLX ? 2 : (pair ? 1 : 0));
            if (rows) rows->push_back(k);
            ks += pair ? 2 : 1;
        }
        k += pair ? 2 : 1;
    }
    if (m) *m = ks;
    if (mm < ks) return -15;
    return 0;
}

template <class R, bool CPLX>
int tgsna_subdiag(const void *A, int lda, int n, bool on_device, cudaStream_t st, std::vector<R> &sub)
{
    sub.assign(std::max(0, n - 1), R(0));
    if (CPLX || n < 2) return 0;
    const R *a = static_cast<const R *>(A);
    if (!on_device) {
        for (int k = 0; k + 1 < n; k++) sub[k] = a[(size_t)k * (lda + 1) + 1];
        return 0;
    }
    cudaError_t e = cudaMemcpy2DAsync(sub.data(), sizeof(R), a + 1, (size_t)(lda + 1) * sizeof(R), sizeof(R), n - 1,
                                      cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
        xtg::set_last_error(std::string("xTGSNA subdiagonal of A: ") + cudaGetErrorString(e));
        return 1;
    }
    return 0;
}

// Device form: A, B, VL, VR and s on the device.
template <class R, bool CPLX>
int tgsna_device(void *stream, char job, char howmny, const int *select, int n, const void *A, int lda, const void *B,
                 int ldb, const void *VL, int ldvl, const void *VR, int ldvr, void *s, int mm, int *m, int *info)
{
    int dummy = 0;
    if (!info) info = &dummy;
    job = (char)std::toupper((unsigned char)job);
    howmny = (char)std::toupper((unsigned char)howmny);
    xtg::set_last_error("");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    std::vector<R> sub;
    std::vector<int> items;
    std::vector<uint8_t> kinds;
    // the subdiagonal is read only once A's leading dimension is known to be valid
    *info = tgsna_check(job, howmny, n, lda, ldb, ldvl, ldvr, CPLX);
    if (*info == 0 && job != 'E') {
        xtg::set_last_error("xTGSNA device form: JOB='E' (S); DIF on the device: xtgevc3_{d,s}tgsna_dif_dev");
        *info = -1;
    }
    if (*info) return 0;
    if (tgsna_subdiag<R, CPLX>(A, lda, n, true, st, sub)) {
        *info = 1;
        return 1;
    }
    *info = tgsna_plan<R, CPLX>(howmny, select, n, mm, sub, m, items, kinds);
    if (*info || items.empty()) return 0;
    const int count = m ? *m : 0;
    const int rc = xtg::eig_cond_device<R, CPLX>(n, A, lda, B, ldb, VL, ldvl, VR, ldvr, count, items, kinds, s, st);
    if (rc) *info = 1;
    return rc;
}

// Host form: stage A, B (and VL, VR for S) on the device, run, copy S and / or DIF back.
template <class R, bool CPLX>
void tgsna_host(char job, char howmny, const int *select, int n, const void *A, int lda, const void *B, int ldb,
                const void *VL, int ldvl, const void *VR, int ldvr, R *s, R *dif, int mm, int *m, void *work,
                int lwork, int *info)
{
    using E = typename std::conditional<CPLX, std::complex<R>, R>::type;
    job = (char)std::toupper((unsigned char)job);
    howmny = (char)std::toupper((unsigned char)howmny);
    xtg::set_last_error("");
    const bool wants = job != 'V', wantdf = job != 'E';
    // LAPACK's LWORK: N for S alone; with DIF 2 N (N + 2) + 16 (D/STGSNA) or 2 N^2 (Z/CTGSNA);
    // 1 for N = 0
    const int lwmin = n == 0 ? 1 : (wantdf ? (CPLX ? 2 * n * n : 2 * n * (n + 2) + 16) : n);
    const bool lquery = lwork == -1;
    if (work) static_cast<E *>(work)[0] = E(lwmin);
    std::vector<R> sub;
    std::vector<int> items, rows;
    std::vector<uint8_t> kinds;
    int count = 0;
    *info = tgsna_check(job, howmny, n, lda, ldb, ldvl, ldvr, CPLX);
    if (*info) return;
    tgsna_subdiag<R, CPLX>(A, lda, n, false, nullptr, sub);
    *info = tgsna_plan<R, CPLX>(howmny, select, n, mm, sub, &count, items, kinds, &rows);
    if (m) *m = count;
    if (*info == 0 && lwork < lwmin && !lquery) *info = -18;
    if (*info || lquery || items.empty()) return;
    const int ld = round_up(n, 32);
    void *dA = nullptr, *dB = nullptr, *dL = nullptr, *dR = nullptr, *dS = nullptr, *dD = nullptr;
    cudaStream_t st = nullptr;
    auto cleanup = [&]() {
        if (st) cudaStreamSynchronize(st);
        for (void *q : {dA, dB, dL, dR, dS, dD})
            if (q) cudaFree(q);
        if (st) cudaStreamDestroy(st);
    };
    cudaError_t e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
    const size_t mat = (size_t)ld * n * sizeof(E), vec = (size_t)ld * count * sizeof(E);
    for (void **q : {&dA, &dB})
        if (e == cudaSuccess) e = cudaMallocAsync(q, mat, st);
    if (wants) {
        for (void **q : {&dL, &dR})
            if (e == cudaSuccess) e = cudaMallocAsync(q, vec, st);
        if (e == cudaSuccess) e = cudaMallocAsync(&dS, (size_t)count * sizeof(R), st);
    }
    if (wantdf && e == cudaSuccess) e = cudaMallocAsync(&dD, (size_t)count * sizeof(R), st);
    if (e == cudaSuccess)
        e = cudaMemcpy2DAsync(dA, ld * sizeof(E), A, (size_t)lda * sizeof(E), n * sizeof(E), n, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess)
        e = cudaMemcpy2DAsync(dB, ld * sizeof(E), B, (size_t)ldb * sizeof(E), n * sizeof(E), n, cudaMemcpyHostToDevice, st);
    if (wants && e == cudaSuccess)
        e = cudaMemcpy2DAsync(dL, ld * sizeof(E), VL, (size_t)ldvl * sizeof(E), n * sizeof(E), count,
                              cudaMemcpyHostToDevice, st);
    if (wants && e == cudaSuccess)
        e = cudaMemcpy2DAsync(dR, ld * sizeof(E), VR, (size_t)ldvr * sizeof(E), n * sizeof(E), count,
                              cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) {
        xtg::set_last_error(std::string("xTGSNA staging: ") + cudaGetErrorString(e));
        cleanup();
        *info = 1;
        return;
    }
    if (wants && xtg::eig_cond_device<R, CPLX>(n, dA, ld, dB, ld, dL, ld, dR, ld, count, items, kinds, dS, st)) {
        cleanup();
        *info = 1;
        return;
    }
    if (wantdf) {
        int rc;
        if constexpr (CPLX) {
            rc = xtg::dif_device_cplx<R>(n, static_cast<const R *>(dA), ld, static_cast<const R *>(dB), ld, rows,
                                         items, static_cast<R *>(dD), st);
        } else {
            std::vector<uint8_t> pairs(kinds.size());
            for (size_t i = 0; i < kinds.size(); i++) pairs[i] = kinds[i] == 1;
            rc = xtg::dif_device<R>(n, static_cast<const R *>(dA), ld, static_cast<const R *>(dB), ld, rows, items,
                                    pairs, static_cast<R *>(dD), st);
        }
        if (rc) {
            cleanup();
            *info = 1;
            return;
        }
    }
    if (wants) e = cudaMemcpyAsync(s, dS, (size_t)count * sizeof(R), cudaMemcpyDeviceToHost, st);
    if (wantdf && e == cudaSuccess) e = cudaMemcpyAsync(dif, dD, (size_t)count * sizeof(R), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
        xtg::set_last_error(std::string("xTGSNA D2H: ") + cudaGetErrorString(e));
        *info = 1;
    }
    cleanup();
}

// DIF alone, device pointers: the checks of xTGSNA with JOB = 'V'.  Complex A, B interleaved.
template <class R, bool CPLX>
int tgsna_dif_device(void *stream, char howmny, const int *select, int n, const R *A, int lda, const R *B, int ldb,
                     R *dif, int mm, int *m, int *info)
{
    int dummy = 0;
    if (!info) info = &dummy;
    howmny = (char)std::toupper((unsigned char)howmny);
    xtg::set_last_error("");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    std::vector<R> sub;
    std::vector<int> items, rows;
    std::vector<uint8_t> kinds;
    *info = tgsna_check('V', howmny, n, lda, ldb, 0, 0, CPLX);
    if (*info) return 0;
    if (tgsna_subdiag<R, CPLX>(A, lda, n, true, st, sub)) {
        *info = 1;
        return 1;
    }
    int count = 0;
    *info = tgsna_plan<R, CPLX>(howmny, select, n, mm, sub, &count, items, kinds, &rows);
    if (m) *m = count;
    if (*info || items.empty()) return 0;
    int rc;
    if constexpr (CPLX) {
        rc = xtg::dif_device_cplx<R>(n, A, lda, B, ldb, rows, items, dif, st);
    } else {
        std::vector<uint8_t> pairs(kinds.size());
        for (size_t i = 0; i < kinds.size(); i++) pairs[i] = kinds[i] == 1;
        rc = xtg::dif_device<R>(n, A, lda, B, ldb, rows, items, pairs, dif, st);
    }
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
int xtgevc3_split_refined(void) { return xtg::refined_columns(); }

int xtgevc3_split_gemm_dev(void *stream, int kind, int slices, int M, int N, int K, const double *A, int lda,
                           const double *B, int ldb, double *C, int ldc, int accumulate)
{
    xtg::set_last_error("");
    if (kind < 0 || kind > 2 || M < 0 || N < 0 || K < 0 || (M > 0 && lda < M) || (K > 0 && ldb < K) ||
        (M > 0 && ldc < M)) {
        xtg::set_last_error("xtgevc3_split_gemm_dev: bad argument");
        return -1;
    }
    if (slices <= 0) slices = kind == 2 ? 14 : kind == 1 ? 7 : 6;
    return xtg::split_gemm_device(kind, slices, M, N, K, A, lda, B, ldb, C, ldc, accumulate,
                                  static_cast<cudaStream_t>(stream));
}

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

void xtgevc3_dtrevc3(char side, char howmny, const int *select, int n, const double *T, int ldt, double *VL,
                     int ldvl, double *VR, int ldvr, int mm, int *m, double *work, int lwork, int *info)
{
    trevc3_host<double, false, double>(side, howmny, select, n, T, ldt, VL, ldvl, VR, ldvr, mm, m, work, lwork,
                                       nullptr, 0, info);
}

void xtgevc3_strevc3(char side, char howmny, const int *select, int n, const float *T, int ldt, float *VL, int ldvl,
                     float *VR, int ldvr, int mm, int *m, float *work, int lwork, int *info)
{
    trevc3_host<float, false, float>(side, howmny, select, n, T, ldt, VL, ldvl, VR, ldvr, mm, m, work, lwork, nullptr,
                                     0, info);
}

void xtgevc3_ztrevc3(char side, char howmny, const int *select, int n, const double *T, int ldt, double *VL,
                     int ldvl, double *VR, int ldvr, int mm, int *m, double *work, int lwork, double *rwork,
                     int lrwork, int *info)
{
    trevc3_host<double, true, std::complex<double>>(side, howmny, select, n, T, ldt, VL, ldvl, VR, ldvr, mm, m,
                                                    reinterpret_cast<std::complex<double> *>(work), lwork, rwork,
                                                    lrwork, info);
}

void xtgevc3_ctrevc3(char side, char howmny, const int *select, int n, const float *T, int ldt, float *VL, int ldvl,
                     float *VR, int ldvr, int mm, int *m, float *work, int lwork, float *rwork, int lrwork, int *info)
{
    trevc3_host<float, true, std::complex<float>>(side, howmny, select, n, T, ldt, VL, ldvl, VR, ldvr, mm, m,
                                                  reinterpret_cast<std::complex<float> *>(work), lwork, rwork, lrwork,
                                                  info);
}

int xtgevc3_dtrevc3_dev(unsigned flags, void *stream, char side, char howmny, const int *select, int n,
                        const double *T, int ldt, double *VL, int ldvl, double *VR, int ldvr, int mm, int *m, int *info)
{
    return trevc3_device<double, false>(flags, stream, side, howmny, select, n, T, ldt, VL, ldvl, VR, ldvr, mm, m,
                                        info);
}

int xtgevc3_strevc3_dev(unsigned flags, void *stream, char side, char howmny, const int *select, int n,
                        const float *T, int ldt, float *VL, int ldvl, float *VR, int ldvr, int mm, int *m, int *info)
{
    return trevc3_device<float, false>(flags, stream, side, howmny, select, n, T, ldt, VL, ldvl, VR, ldvr, mm, m,
                                       info);
}

int xtgevc3_ztrevc3_dev(unsigned flags, void *stream, char side, char howmny, const int *select, int n,
                        const double *T, int ldt, double *VL, int ldvl, double *VR, int ldvr, int mm, int *m, int *info)
{
    return trevc3_device<double, true>(flags, stream, side, howmny, select, n, T, ldt, VL, ldvl, VR, ldvr, mm, m,
                                       info);
}

int xtgevc3_ctrevc3_dev(unsigned flags, void *stream, char side, char howmny, const int *select, int n,
                        const float *T, int ldt, float *VL, int ldvl, float *VR, int ldvr, int mm, int *m, int *info)
{
    return trevc3_device<float, true>(flags, stream, side, howmny, select, n, T, ldt, VL, ldvl, VR, ldvr, mm, m,
                                      info);
}

void xtgevc3_dtgsna(char job, char howmny, const int *select, int n, const double *A, int lda, const double *B,
                    int ldb, const double *VL, int ldvl, const double *VR, int ldvr, double *s, double *dif, int mm, int *m,
                    double *work, int lwork, int *iwork, int *info)
{
    (void)iwork;
    tgsna_host<double, false>(job, howmny, select, n, A, lda, B, ldb, VL, ldvl, VR, ldvr, s, dif, mm, m, work, lwork,
                          info);
}

int xtgevc3_dtgsna_dev(void *stream, char job, char howmny, const int *select, int n, const double *A, int lda,
                        const double *B, int ldb, const double *VL, int ldvl, const double *VR, int ldvr, double *s, int mm,
                        int *m, int *info)
{
    return tgsna_device<double, false>(stream, job, howmny, select, n, A, lda, B, ldb, VL, ldvl, VR, ldvr, s, mm, m, info);
}

void xtgevc3_stgsna(char job, char howmny, const int *select, int n, const float *A, int lda, const float *B,
                    int ldb, const float *VL, int ldvl, const float *VR, int ldvr, float *s, float *dif, int mm, int *m,
                    float *work, int lwork, int *iwork, int *info)
{
    (void)iwork;
    tgsna_host<float, false>(job, howmny, select, n, A, lda, B, ldb, VL, ldvl, VR, ldvr, s, dif, mm, m, work, lwork,
                          info);
}

int xtgevc3_stgsna_dev(void *stream, char job, char howmny, const int *select, int n, const float *A, int lda,
                        const float *B, int ldb, const float *VL, int ldvl, const float *VR, int ldvr, float *s, int mm,
                        int *m, int *info)
{
    return tgsna_device<float, false>(stream, job, howmny, select, n, A, lda, B, ldb, VL, ldvl, VR, ldvr, s, mm, m, info);
}

void xtgevc3_ztgsna(char job, char howmny, const int *select, int n, const double *A, int lda, const double *B,
                    int ldb, const double *VL, int ldvl, const double *VR, int ldvr, double *s, double *dif, int mm, int *m,
                    double *work, int lwork, int *iwork, int *info)
{
    (void)iwork;
    tgsna_host<double, true>(job, howmny, select, n, A, lda, B, ldb, VL, ldvl, VR, ldvr, s, dif, mm, m, work, lwork,
                          info);
}

int xtgevc3_ztgsna_dev(void *stream, char job, char howmny, const int *select, int n, const double *A, int lda,
                        const double *B, int ldb, const double *VL, int ldvl, const double *VR, int ldvr, double *s, int mm,
                        int *m, int *info)
{
    return tgsna_device<double, true>(stream, job, howmny, select, n, A, lda, B, ldb, VL, ldvl, VR, ldvr, s, mm, m, info);
}

void xtgevc3_ctgsna(char job, char howmny, const int *select, int n, const float *A, int lda, const float *B,
                    int ldb, const float *VL, int ldvl, const float *VR, int ldvr, float *s, float *dif, int mm, int *m,
                    float *work, int lwork, int *iwork, int *info)
{
    (void)iwork;
    tgsna_host<float, true>(job, howmny, select, n, A, lda, B, ldb, VL, ldvl, VR, ldvr, s, dif, mm, m, work, lwork,
                          info);
}

int xtgevc3_ctgsna_dev(void *stream, char job, char howmny, const int *select, int n, const float *A, int lda,
                        const float *B, int ldb, const float *VL, int ldvl, const float *VR, int ldvr, float *s, int mm,
                        int *m, int *info)
{
    return tgsna_device<float, true>(stream, job, howmny, select, n, A, lda, B, ldb, VL, ldvl, VR, ldvr, s, mm, m, info);
}

int xtgevc3_dtgsna_dif_dev(void *stream, char howmny, const int *select, int n, const double *A, int lda,
                           const double *B, int ldb, double *dif, int mm, int *m, int *info)
{
    return tgsna_dif_device<double, false>(stream, howmny, select, n, A, lda, B, ldb, dif, mm, m, info);
}

int xtgevc3_stgsna_dif_dev(void *stream, char howmny, const int *select, int n, const float *A, int lda,
                           const float *B, int ldb, float *dif, int mm, int *m, int *info)
{
    return tgsna_dif_device<float, false>(stream, howmny, select, n, A, lda, B, ldb, dif, mm, m, info);
}

int xtgevc3_ztgsna_dif_dev(void *stream, char howmny, const int *select, int n, const double *A, int lda,
                           const double *B, int ldb, double *dif, int mm, int *m, int *info)
{
    return tgsna_dif_device<double, true>(stream, howmny, select, n, A, lda, B, ldb, dif, mm, m, info);
}

int xtgevc3_ctgsna_dif_dev(void *stream, char howmny, const int *select, int n, const float *A, int lda,
                           const float *B, int ldb, float *dif, int mm, int *m, int *info)
{
    return tgsna_dif_device<float, true>(stream, howmny, select, n, A, lda, B, ldb, dif, mm, m, info);
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
