// Adjoint of the right eigenvectors (xtgevc3_adjoint): dL/dS and dL/dP from dL/dX.
//
// X is the output of the forward with SIDE='R', HOWMNY='A' (all right eigenvectors in the
// Schur basis; with HOWMNY='B' the caller first maps dL/dV to dL/dX = Z^T dL/dV).  The
// eigenvalues (alpha, beta) are inputs held fixed, as are the per-column overflow scale
// factors of the forward (their effect is read back from X itself); the diagonal blocks
// are recomputed from S and P, not stored.  See kernels_adjoint.cuh for the formulas.
//
// Steps on the device (stream `st`):
//   1. pencil norms and the argmax columns, shift coefficients of every column;
//   2. the reversed transposed pencil (F S^T F, F P^T F) and the right-hand sides
//      R = F conj(G) (rows below each column's eigenvalue row only);
//   3. blocked back substitution of R, bottom to top, with the forward's kernels: per
//      row block the truncated shifted solves, then one update GEMM of the rows above;
//   4. the GEMM operands AS, AP from the solution, X^T, and dS = AS X^T, dP = AP X^T;
//   5. (real pencils) the seed and norm terms of the complex pairs; the mask of the
//      entries the forward reads.
#include "../../include/xtgevc3.h"
#include "engine.cuh"
#include "host_common.cuh"
#include "kernels_adjoint.cuh"
#include "kernels_misc.cuh"

#include <algorithm>
#include <mutex>
#include <vector>

namespace xtg {
namespace {

std::once_flag g_adj_once[64];

void configure_adjoint(int dev)
{
    if (dev < 0 || dev >= 64) return;
    std::call_once(g_adj_once[dev], []() {
        cudaFuncSetAttribute(diag_adjoint_real<double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             2 * kBlock * kSmLd * (int)sizeof(double));
        cudaFuncSetAttribute(diag_adjoint_real<float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             2 * kBlock * kSmLd * (int)sizeof(float));
        cudaFuncSetAttribute(diag_adjoint_cplx<double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             2 * kBlock * kSmLd * (int)sizeof(cplx<double>));
        cudaFuncSetAttribute(diag_adjoint_cplx<float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             2 * kBlock * kSmLd * (int)sizeof(cplx<float>));
    });
}

template <class R, bool CPLX>
int adjoint_device(int n, const void *S_, int lds, const void *P_, int ldp, const void *alpha_, const void *alphai_,
                   const void *beta_, const void *X_, int ldx, const void *G_, int ldg, void *dS_, int ldds, void *dP_,
                   int lddp, cudaStream_t st)
{
    using E = typename std::conditional<CPLX, cplx<R>, R>::type;
    if (n <= 0) return 0;
    const E *S = static_cast<const E *>(S_), *P = static_cast<const E *>(P_);
    const E *X = static_cast<const E *>(X_), *G = static_cast<const E *>(G_);
    E *dS = static_cast<E *>(dS_), *dP = static_cast<E *>(dP_);
    int dev = 0;
    XTG_CK(cudaGetDevice(&dev));
    configure_device(dev);
    configure_adjoint(dev);
    XTG_CK(cudaGetLastError());

    // ---- column structure (all right eigenvectors, ascending eigenvalue order) ------------
    const int m = n;
    const R *alphai = static_cast<const R *>(alphai_);
    std::vector<int> colk(m);
    std::vector<uint8_t> kind(m, kReal);
    std::vector<char> pairstart(n + 1, 0);
    std::vector<int> items, pairs;
    for (int k = 0; k < n;) {
        const bool pair = !CPLX && alphai[k] != R(0) && k + 1 < n;
        items.push_back(k);
        if (pair) {
            colk[k] = colk[k + 1] = k;
            kind[k] = kPairRe;
            kind[k + 1] = kPairIm;
            pairstart[k] = 1;
            pairs.push_back(k);
            k += 2;
        } else {
            colk[k] = k;
            k += 1;
        }
    }
    std::vector<char> sub(n, 0);
    if constexpr (!CPLX) {
        if (n > 1) {
            std::vector<E> d(n - 1);
            XTG_CK(cudaMemcpy2DAsync(d.data(), sizeof(E), S + 1, (size_t)(lds + 1) * sizeof(E), sizeof(E), n - 1,
                                     cudaMemcpyDeviceToHost, st));
            XTG_CK(cudaStreamSynchronize(st));
            for (int k = 0; k + 1 < n; k++) sub[k] = d[k] != E(0);
        }
    }
    // row blocks of the reversed orientation, bottom to top; a 2x2 block is never split
    auto split = [&](int j) -> bool {
        if (CPLX || j <= 0 || j >= n) return false;
        const int kq = n - 1 - j;
        return sub[kq] || pairstart[kq];
    };
    std::vector<std::pair<int, int>> blocks;
    for (int cur = n; cur > 0;) {
        int j = std::max(0, cur - kBlock);
        if (j > 0 && split(j)) j += 1;
        blocks.push_back({j, cur});
        cur = j;
    }

    // ---- buffers ---------------------------------------------------------------------------
    Scratch scr(st);
    const int ld_n = round_up(n, 32);
    const int ncoef = CPLX ? 6 : 4;
    const int ldy = 2 * kBlock;
    R *d_eig = scr.get<R>(CPLX ? 4 * (size_t)n : 3 * (size_t)n);
    R *d_sums = scr.get<R>(2 * (size_t)n);
    R *d_norms = scr.get<R>(4);
    int *d_jmax = scr.get<int>(2);
    R *coef = scr.get<R>((size_t)ncoef * m);
    int *d_ints = scr.get<int>(3 * (size_t)m + pairs.size() + 1);
    uint8_t *d_kind = scr.get<uint8_t>((size_t)m);
    E *St = scr.get<E>((size_t)ld_n * n);
    E *Pt = scr.get<E>((size_t)ld_n * n);
    E *Rs = scr.get<E>((size_t)ld_n * m);
    E *Y = scr.get<E>((size_t)ldy * m);
    E *AS = scr.get<E>((size_t)ld_n * m);
    E *AP = scr.get<E>((size_t)ld_n * m);
    E *Xt = scr.get<E>((size_t)ld_n * n);
    if (scr.err) {
        set_last_error(std::string("adjoint scratch: ") + cudaGetErrorString(scr.err));
        return 1;
    }
    R *d_dnorm = d_norms + 2;
    std::vector<int> ints(3 * (size_t)m + pairs.size() + 1, 0);
    std::copy(colk.begin(), colk.end(), ints.begin());
    std::copy(items.begin(), items.end(), ints.begin() + m);
    std::copy(pairs.begin(), pairs.end(), ints.begin() + 3 * m);
    std::vector<int> tops(m);
    for (int c = 0; c < m; c++) tops[c] = n - colk[c];
    std::copy(tops.begin(), tops.end(), ints.begin() + 2 * m);
    XTG_CK(cudaMemcpyAsync(d_ints, ints.data(), ints.size() * sizeof(int), cudaMemcpyHostToDevice, st));
    XTG_CK(cudaMemcpyAsync(d_kind, kind.data(), m, cudaMemcpyHostToDevice, st));
    const int *d_colk = d_ints, *d_items = d_ints + m, *d_tops = d_ints + 2 * m, *d_pairs = d_ints + 3 * m;
    if (CPLX) {
        XTG_CK(cudaMemcpyAsync(d_eig, alpha_, 2 * n * sizeof(R), cudaMemcpyHostToDevice, st));
        XTG_CK(cudaMemcpyAsync(d_eig + 2 * n, beta_, 2 * n * sizeof(R), cudaMemcpyHostToDevice, st));
    } else {
        XTG_CK(cudaMemcpyAsync(d_eig, alpha_, n * sizeof(R), cudaMemcpyHostToDevice, st));
        XTG_CK(cudaMemcpyAsync(d_eig + n, alphai_, n * sizeof(R), cudaMemcpyHostToDevice, st));
        XTG_CK(cudaMemcpyAsync(d_eig + 2 * n, beta_, n * sizeof(R), cudaMemcpyHostToDevice, st));
    }
    XTG_CK(cudaMemsetAsync(d_dnorm, 0, 2 * sizeof(R), st));

    long long nl = 0;
    // 1. norms, argmax columns, coefficients (right problem: no conjugation)
    colsum_kernel<E, R><<<(n + 7) / 8, 256, 0, st>>>(S, lds, P, ldp, n, CPLX ? 0 : 1, d_sums);
    colargmax_kernel<R><<<1, 1024, 0, st>>>(d_sums, n, d_norms, d_jmax);
    if constexpr (CPLX) {
        coef_cplx_kernel<R><<<(m + 127) / 128, 128, 0, st>>>(reinterpret_cast<const cplx<R> *>(d_eig),
                                                             reinterpret_cast<const cplx<R> *>(d_eig + 2 * n), d_colk,
                                                             m, 0, d_norms, coef);
    } else {
        coef_real_kernel<R><<<(m + 127) / 128, 128, 0, st>>>(d_eig, d_eig + n, d_eig + 2 * n, d_colk, d_kind, m, 0,
                                                             d_norms, coef);
    }
    // 2. reversed transposed pencil (plain transpose: the solves are with W^T, not W^H)
    {
        dim3 g((n + 31) / 32, (n + 31) / 32), b(32, 8);
        rev_transpose_kernel<E><<<g, b, 0, st>>>(S, lds, St, ld_n, n, 0);
        rev_transpose_kernel<E><<<g, b, 0, st>>>(P, ldp, Pt, ld_n, n, 0);
        adj_rhs_kernel<E><<<dim3(std::max(1, std::min((n + 255) / 256, 64)), m), 256, 0, st>>>(
            G, ldg, Rs, ld_n, n, m, d_colk, CPLX ? nullptr : d_kind);
        nl += 6;
    }
    XTG_CK(cudaGetLastError());

    // 3. blocked back substitution in reversed orientation.  Column c (eigenvalue k_c) is
    // active in block [r0, r1) while its top row n - k_c lies below r1: columns with
    // k_c > n - r1, a suffix of the ascending column order.
    const size_t diag_smem = 2 * kBlock * kSmLd * sizeof(E);
    const double cfl = CPLX ? 4.0 : 1.0;
    (void)cfl;
    for (const auto &blk : blocks) {
        const int r0 = blk.first, r1 = blk.second, jnb = r1 - r0, bpad = round_up(jnb, kKPad);
        const int c0 = int(std::upper_bound(colk.begin(), colk.end(), n - r1) - colk.begin());
        if (c0 >= m) break;  // no column reaches this block, nor any block above it
        DiagArgs<R> da{};
        da.S = reinterpret_cast<const R *>(St);
        da.P = reinterpret_cast<const R *>(Pt);
        da.lds = ld_n;
        da.ldp = ld_n;
        da.n = n;
        da.r0 = r0;
        da.r1 = r1;
        da.ys_off = 0;
        da.yhalf = bpad;
        da.ypad = bpad;
        da.zl_off = 0;
        da.zl_len = 0;
        da.items = d_items;
        da.it0 = int(std::lower_bound(items.begin(), items.end(), c0) - items.begin());
        da.nitems = (int)items.size();
        da.colk = d_tops;
        da.kind = d_kind;
        da.coef = coef;
        da.X = reinterpret_cast<R *>(Rs);
        da.ldx = ld_n;
        da.Y = reinterpret_cast<R *>(Y);
        da.ldy = ldy;
        da.thr_rhs = da.thr_upd = R(0);
        da.left_seed = 0;
        da.pending = nullptr;
        da.safe_lo = 0;
        const int grid = std::max(1, std::min((da.nitems - da.it0 + 7) / 8, 2 * 148));
        if constexpr (CPLX) diag_adjoint_cplx<R><<<grid, 256, diag_smem, st>>>(da);
        else diag_adjoint_real<R><<<grid, 256, diag_smem, st>>>(da);
        nl += 1;
        if (r0 > 0) {
            GemmArgs<E> g;
            g.M = r0;
            g.N = m - c0;
            g.mlo = 0;
            g.nseg = 2;
            g.seg[0].A = St + (size_t)r0 * ld_n;
            g.seg[0].lda = ld_n;
            g.seg[0].acols = jnb;
            g.seg[0].K = bpad;
            g.seg[0].boff = 0;
            g.seg[1].A = Pt + (size_t)r0 * ld_n;
            g.seg[1].lda = ld_n;
            g.seg[1].acols = jnb;
            g.seg[1].K = bpad;
            g.seg[1].boff = bpad;
            g.K = 2 * bpad;
            g.B = Y + (size_t)c0 * ldy;
            g.ldb = ldy;
            g.brows = ldy;
            g.C = Rs + (size_t)c0 * ld_n;
            g.ldc = ld_n;
            g.ccol = nullptr;
            g.kext = nullptr;
            g.accumulate = 1;
            launch_gemm<E>(g, false, st);
            nl += 1;
        }
        XTG_CK(cudaGetLastError());
    }

    // 4. gradient GEMMs dS = AS X^T, dP = AP X^T (complex: conjugated operands)
    {
        dim3 go(std::max(1, std::min((n + 255) / 256, 64)), m);
        if constexpr (CPLX)
            adj_operands_cplx<R><<<go, 256, 0, st>>>(Rs, ld_n, n, m, d_colk, coef, AS, AP, ld_n);
        else
            adj_operands_real<R><<<go, 256, 0, st>>>(Rs, ld_n, n, m, d_colk, d_kind, coef, AS, AP, ld_n);
        dim3 g((n + 31) / 32, (m + 31) / 32), b(32, 8);
        transpose_kernel<E><<<g, b, 0, st>>>(X, ldx, Xt, ld_n, n, m, CPLX ? 1 : 0);
        nl += 2;
        for (int q = 0; q < 2; q++) {
            GemmArgs<E> gg;
            gg.M = n;
            gg.N = n;
            gg.mlo = 0;
            gg.nseg = 1;
            gg.seg[0].A = q == 0 ? AS : AP;
            gg.seg[0].lda = ld_n;
            gg.seg[0].acols = m;
            gg.seg[0].K = round_up(m, kKPad);
            gg.seg[0].boff = 0;
            gg.K = gg.seg[0].K;
            gg.B = Xt;
            gg.ldb = ld_n;
            gg.brows = m;
            gg.C = q == 0 ? dS : dP;
            gg.ldc = q == 0 ? ldds : lddp;
            gg.ccol = nullptr;
            gg.kext = nullptr;
            gg.accumulate = 0;
            launch_gemm<E>(gg, false, st);
            nl += 1;
        }
    }
    // 5. pair terms, mask and norm terms
    if constexpr (!CPLX) {
        const int np = (int)pairs.size();
        if (np > 0) {
            adj_pair_terms<R><<<(np + 7) / 8, 256, 0, st>>>(S, lds, P, ldp, X, ldx, G, ldg, Rs, ld_n, n, d_pairs, np,
                                                           coef, d_eig, d_norms, dS, ldds, dP, lddp, d_dnorm);
            nl += 1;
        }
    }
    adj_finalize_kernel<E, R><<<dim3(std::max(1, std::min((n + 255) / 256, 64)), n), 256, 0, st>>>(
        dS, ldds, dP, lddp, S, lds, P, ldp, n, d_dnorm, d_jmax);
    nl += 1;
    XTG_CK(cudaGetLastError());
    count_launches(nl + 3);
    XTG_CK(cudaStreamSynchronize(st));
    return 0;
}

}  // namespace
}  // namespace xtg

extern "C" {

int xtgevc3_adjoint(char prec, void *stream, int n, const void *S, int lds, const void *P, int ldp,
                    const void *alpha, const void *alphai, const void *beta, const void *X, int ldx, const void *G,
                    int ldg, void *dS, int ldds, void *dP, int lddp)
{
    xtg::set_last_error("");
    if (n < 0 || (n > 0 && (!S || !P || !alpha || !beta || !X || !G || !dS || !dP))) {
        xtg::set_last_error("xtgevc3_adjoint: NULL argument or n < 0");
        return -1;
    }
    const int ldmin = n > 0 ? n : 1;
    if (lds < ldmin || ldp < ldmin || ldx < ldmin || ldg < ldmin || ldds < ldmin || lddp < ldmin) {
        xtg::set_last_error("xtgevc3_adjoint: a leading dimension is smaller than n");
        return -1;
    }
    if ((prec == 'd' || prec == 's') && n > 0 && !alphai) {
        xtg::set_last_error("xtgevc3_adjoint: alphai is NULL");
        return -1;
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    switch (prec) {
    case 'd':
        return xtg::adjoint_device<double, false>(n, S, lds, P, ldp, alpha, alphai, beta, X, ldx, G, ldg, dS, ldds,
                                                  dP, lddp, st);
    case 's':
        return xtg::adjoint_device<float, false>(n, S, lds, P, ldp, alpha, alphai, beta, X, ldx, G, ldg, dS, ldds, dP,
                                                 lddp, st);
    case 'z':
        return xtg::adjoint_device<double, true>(n, S, lds, P, ldp, alpha, nullptr, beta, X, ldx, G, ldg, dS, ldds,
                                                 dP, lddp, st);
    case 'c':
        return xtg::adjoint_device<float, true>(n, S, lds, P, ldp, alpha, nullptr, beta, X, ldx, G, ldg, dS, ldds, dP,
                                                lddp, st);
    default:
        xtg::set_last_error("xtgevc3_adjoint: prec must be 'd', 's', 'z' or 'c'");
        return -1;
    }
}

}  // extern "C"
