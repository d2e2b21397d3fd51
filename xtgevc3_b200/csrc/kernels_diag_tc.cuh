// Diagonal-block shifted solves of the real double path with the updates on the FP64 tensor
// cores: the same solves as diag_solve_real (kernels_diag.cuh), arranged so that the
// eigenvectors of a warp share their row updates.
//
// Within a 64-row block the update of the rows above a solved row j is
//     r_i -= W_c(i, j) x_j = r_i + S(i, j) (-ac_c x_j) + P(i, j) (b_c x_j),
// so for eight columns at once it is a product of the block's S and P (shared by every
// column) with two 4 x 8 operands U = -ac x, V = b x (a (Re, Im) pair: b x mixes the two
// columns).  A warp holds eight such columns ("slots" of two columns: a pair, or up to two
// real columns) as m8n8k4 FP64 accumulators, eight row tiles of 8 rows: lane l holds rows
// 8 t + l / 4 of columns 2 (l % 4) and 2 (l % 4) + 1, i.e. both columns of slot l % 4.
// The rows are solved bottom to top in sub-blocks of 3 or 4 rows (never splitting a 2x2
// block of S, with a boundary at the mid-block check row):
//   * the sub-block's rows go from the accumulators to shared memory; lane j (j < 4)
//     solves them for slot j with the factors of its diagonal blocks (precomputed by the
//     whole warp: reciprocals of 1x1 pivots, the partially pivoted LU of 2x2 blocks) and
//     their mutual updates, and writes the solution back;
//   * two MMAs per row tile above the sub-block add S(rows, sub-block) U + P(rows,
//     sub-block) V to the accumulators.
// Pivots, 2x2 LU steps, the per-row cap, the mid-block check, the block checks and the
// output are those of diag_solve_real: per column, in the same places.
// Opt-in (XTGEVC3_DIAG_TC=1): it raises the solves' throughput (four pair eigenvectors per
// warp), but the solves are bound by each launch's latency, and a warp here walks 16
// sub-blocks with a solve, a barrier and an MMA update each, plus its setup, factoring and
// output: ~56 us per launch at n = 8192 against ~27 us for diag_solve_real.  A guard's
// rescaling of a column covers its accumulator entries, its solved rows, its seed and its
// rows outside the block (scale_above, scale_rows, scale_lower_y).
#pragma once
#include "kernels_diag.cuh"
#include "kernels_gemm.cuh"

namespace xtg {
namespace dtc {

constexpr int kWarps = 8;        // warps per CTA (one CTA per SM: 171 KB of shared memory)
constexpr int kThreads = 32 * kWarps;
constexpr int kSlots = 4;        // slots per warp
constexpr int kCols = 8;         // GEMM columns per warp

enum : int { kSlotEmpty = 0, kSlotPair = 1, kSlotReal = 2 };

// Per-warp shared state.
struct WarpState {
    double xs[kBlock][kCols];        // rows of the sub-block being solved, then the solution x
    double fac[kBlock][kSlots][4];   // factors per row and slot (layout below)
    double seed[kSlots][4];          // real slot: seed of column 0, 1; pair: seed0 (Re, Im), seed1
    double ac[kCols], br[kCols], bi[kCols], smin[kCols];
    double pend[kCols];              // rescale factor of a column from the sub-block solve (1: none)
    double mx[kCols];                // per-column maxima of the guards
    uint64_t swm[kSlots][2];         // 2x2 pivot swaps: bit q for the block (q-1, q), per column
    int col[kCols];                  // X column (-1: none)
    int nrows[kCols];                // rows to solve (the eigenvalue's row kl for a diagonal column)
    int kl[kCols];                   // eigenvalue row within the block (diagonal columns), else -1
    int top[kCols];                  // last stored row of the column (k, or k + 1 for a pair)
    int kind[kSlots];
};
// fac layout: real slot, column e of the slot: a 1x1 row i: fac[i][e * 2] = 1 / w_ii; a 2x2
// block (p, q): fac[p][e * 2 + 0, 1] = (a^-1, b), fac[q][e * 2 + 0, 1] = (m, u^-1).  Pair
// slot (complex): a 1x1 row: fac[i][0, 1] = 1 / w_ii; a 2x2 block: fac[p] = (a^-1, b),
// fac[q] = (m, u^-1), each complex (Re, Im).

constexpr size_t kSmemBytes = 2 * (size_t)kSmLd * kBlock * sizeof(double) + (size_t)kWarps * sizeof(WarpState);

using C = cplx<double>;

// The sub-block [j0, j0 + kb) of one real column (column e of a real slot), held by the
// slot's solver lane: rr in (right-hand side), xx out (solution rows; rows at or past nr
// keep 0).  Returns the product of the cap's rescaling factors (1: none), already applied
// to rr and xx.
__device__ __forceinline__ double solve_sub_real(double (&rr)[4], double (&xx)[4], int j0, int kb, int nr, uint64_t sec,
                                                 uint64_t sw, const WarpState &w, int slot, int e, double ac,
                                                 double br, const double *Ss, const double *Ps, double cap,
                                                 double target)
{
    double pend = 1.0;
    auto rescale = [&](double s) {
#pragma unroll
        for (int u = 0; u < 4; u++) {
            rr[u] *= s;
            xx[u] *= s;
        }
        pend *= s;
    };
    // the sub-block's factors and its S, P entries, loaded before the dependent chain
    double f0[4], f1[4], sv[4][4], pv[4][4];
#pragma unroll
    for (int u = 0; u < 4; u++) {
        const int r = min(j0 + u, kBlock - 1);
        f0[u] = w.fac[r][slot][2 * e];
        f1[u] = w.fac[r][slot][2 * e + 1];
#pragma unroll
        for (int v = 0; v < u; v++) {
            const int rv = min(j0 + v, kBlock - 1);
            sv[v][u] = Ss[rv + r * kSmLd];
            pv[v][u] = Ps[rv + r * kSmLd];
        }
    }
    bool skip = false;
#pragma unroll
    for (int u = 3; u >= 0; u--) {
        const int i = j0 + u;
        if (u >= kb || i >= nr) continue;
        if (skip) {
            skip = false;
            continue;
        }
        if (u >= 1 && ((sec >> i) & 1ull)) {  // the 2x2 block (i - 1, i)
            const int q = i;
            const bool s_w = (sw >> q) & 1ull;
            const double ia = f0[u - 1], bb = f1[u - 1];
            const double m = f0[u], iu = f1[u];
            const double rp = rr[u - 1], rq = rr[u];
            double r1 = s_w ? rq : rp, r2 = s_w ? rp : rq;
            double xq = (r2 - m * r1) * iu;
            double xp = (r1 - bb * xq) * ia;
            if (!(fabs(xq) <= cap && fabs(xp) <= cap)) {
                double s = (target / fabs(iu)) / (fabs(r2) + fabs(m) * fabs(r1));
                if (s < 1.0) {
                    rescale(s);
                    r1 = s * r1;
                    r2 = s * r2;
                }
                xq = (r2 - m * r1) * iu;
                s = (target / fabs(ia)) / (fabs(r1) + fabs(bb) * fabs(xq));
                if (s < 1.0) {
                    rescale(s);
                    r1 = s * r1;
                    xq = s * xq;
                }
                xp = (r1 - bb * xq) * ia;
            }
            xx[u - 1] = xp;
            xx[u] = xq;
            const double up = ac * xp, vp = br * xp, uq = ac * xq, vq = br * xq;
#pragma unroll
            for (int v = 0; v < 4; v++)
                if (v < u - 1)
                    rr[v] = ((rr[v] - sv[v][u - 1] * up) - sv[v][u] * uq) + (pv[v][u - 1] * vp + pv[v][u] * vq);
            skip = true;
        } else {
            const double iv = f0[u];
            double x = rr[u] * iv;
            if (!(fabs(x) <= cap)) {
                const double s = (target / fabs(iv)) / fabs(rr[u]);
                rescale(s);
                x = rr[u] * iv;
            }
            xx[u] = x;
            const double uu = ac * x, vv = br * x;
#pragma unroll
            for (int v = 0; v < 4; v++)
                if (v < u) rr[v] = (rr[v] - sv[v][u] * uu) + pv[v][u] * vv;
        }
    }
    return pend;
}

// The same for a (Re, Im) pair slot in complex arithmetic, shift b = br + i bi.
__device__ __forceinline__ double solve_sub_pair(C (&rr)[4], C (&xx)[4], int j0, int kb, int nr, uint64_t sec,
                                                 uint64_t sw, const WarpState &w, int slot, double ac, C b,
                                                 const double *Ss, const double *Ps, double cap, double target)
{
    double pend = 1.0;
    auto rescale = [&](double s) {
#pragma unroll
        for (int u = 0; u < 4; u++) {
            rr[u] = s * rr[u];
            xx[u] = s * xx[u];
        }
        pend *= s;
    };
    C f0[4], f1[4];
    double sv[4][4], pv[4][4];
#pragma unroll
    for (int u = 0; u < 4; u++) {
        const int r = min(j0 + u, kBlock - 1);
        f0[u] = C(w.fac[r][slot][0], w.fac[r][slot][1]);
        f1[u] = C(w.fac[r][slot][2], w.fac[r][slot][3]);
#pragma unroll
        for (int v = 0; v < u; v++) {
            const int rv = min(j0 + v, kBlock - 1);
            sv[v][u] = Ss[rv + r * kSmLd];
            pv[v][u] = Ps[rv + r * kSmLd];
        }
    }
    bool skip = false;
#pragma unroll
    for (int u = 3; u >= 0; u--) {
        const int i = j0 + u;
        if (u >= kb || i >= nr) continue;
        if (skip) {
            skip = false;
            continue;
        }
        if (u >= 1 && ((sec >> i) & 1ull)) {
            const int q = i;
            const bool s_w = (sw >> q) & 1ull;
            const C ia = f0[u - 1], bb = f1[u - 1], m = f0[u], iu = f1[u];
            const C rp = rr[u - 1], rq = rr[u];
            C r1 = s_w ? rq : rp, r2 = s_w ? rp : rq;
            C xq = (r2 - m * r1) * iu;
            C xp = (r1 - bb * xq) * ia;
            if (!(mag(xq) <= cap && mag(xp) <= cap)) {
                double s = (target / mag(iu)) / (mag(r2) + mag(m) * mag(r1));
                if (s < 1.0) {
                    rescale(s);
                    r1 = s * r1;
                    r2 = s * r2;
                }
                xq = (r2 - m * r1) * iu;
                s = (target / mag(ia)) / (mag(r1) + mag(bb) * mag(xq));
                if (s < 1.0) {
                    rescale(s);
                    r1 = s * r1;
                    xq = s * xq;
                }
                xp = (r1 - bb * xq) * ia;
            }
            xx[u - 1] = xp;
            xx[u] = xq;
            const C up = ac * xp, vp = b * xp, uq = ac * xq, vq = b * xq;
#pragma unroll
            for (int v = 0; v < 4; v++)
                if (v < u - 1)
                    rr[v] = ((rr[v] - sv[v][u - 1] * up) - sv[v][u] * uq) + (pv[v][u - 1] * vp + pv[v][u] * vq);
            skip = true;
        } else {
            const C iv = f0[u];
            C x = rr[u] * iv;
            if (!(mag(x) <= cap)) {
                const double s = (target / mag(iv)) / mag(rr[u]);
                rescale(s);
                x = rr[u] * iv;
            }
            xx[u] = x;
            const C uu = ac * x, vv = b * x;
#pragma unroll
            for (int v = 0; v < 4; v++)
                if (v < u) rr[v] = (rr[v] - sv[v][u] * uu) + pv[v][u] * vv;
        }
    }
    return pend;
}

// Factors of row i of slot j (every column of the slot), as factor_rows computes them per
// lane; returns the 2x2 pivot swap of the block ending at row i, per column of the slot.
__device__ __forceinline__ void factor_task(WarpState &w, int j, int i, uint64_t sec, const double *Ss,
                                            const double *Ps, bool &sw0, bool &sw1)
{
    sw0 = sw1 = false;
    const int kind = w.kind[j];
    if (kind == kSlotPair) {
        const int g = 2 * j, nr = w.nrows[g];
        if (i >= nr) return;
        const double ac = w.ac[g], br = w.br[g], bi = w.bi[g], smin = w.smin[g];
        auto W = [&](int r, int c) -> C {
            const double s = Ss[r + c * kSmLd], p = Ps[r + c * kSmLd];
            return C(ac * s - br * p, -bi * p);
        };
        const bool in2 = ((sec >> i) & 1ull) || (i + 1 < nr && ((sec >> (i + 1)) & 1ull));
        if (!in2) {
            const C v = rcp(floor_pivot(W(i, i), smin));
            w.fac[i][j][0] = v.x;
            w.fac[i][j][1] = v.y;
        }
        if (i >= 1 && ((sec >> i) & 1ull)) {
            const C w11 = W(i - 1, i - 1), w12 = W(i - 1, i), w21 = W(i, i - 1), w22 = W(i, i);
            const bool s_w = mag(w21) > mag(w11);
            const C pa = s_w ? w21 : w11, pb = s_w ? w22 : w12, pc = s_w ? w11 : w21, pd = s_w ? w12 : w22;
            const C ia = rcp(floor_pivot(pa, smin));
            const C m = pc * ia;
            const C fu = rcp(floor_pivot(pd - m * pb, smin));
            double *fp = w.fac[i - 1][j], *fq = w.fac[i][j];
            fp[0] = ia.x; fp[1] = ia.y; fp[2] = pb.x; fp[3] = pb.y;
            fq[0] = m.x; fq[1] = m.y; fq[2] = fu.x; fq[3] = fu.y;
            sw0 = s_w;
        }
    } else if (kind == kSlotReal) {
#pragma unroll
        for (int e = 0; e < 2; e++) {
            const int g = 2 * j + e, nr = w.nrows[g];
            if (w.col[g] < 0 || i >= nr) continue;
            const double ac = w.ac[g], br = w.br[g], smin = w.smin[g];
            auto W = [&](int r, int c) -> double { return ac * Ss[r + c * kSmLd] - br * Ps[r + c * kSmLd]; };
            const bool in2 = ((sec >> i) & 1ull) || (i + 1 < nr && ((sec >> (i + 1)) & 1ull));
            if (!in2) w.fac[i][j][2 * e] = rcp(floor_pivot(W(i, i), smin));
            if (i >= 1 && ((sec >> i) & 1ull)) {
                const double w11 = W(i - 1, i - 1), w12 = W(i - 1, i), w21 = W(i, i - 1), w22 = W(i, i);
                const bool s_w = fabs(w21) > fabs(w11);
                const double pa = s_w ? w21 : w11, pb = s_w ? w22 : w12, pc = s_w ? w11 : w21, pd = s_w ? w12 : w22;
                const double ia = rcp(floor_pivot(pa, smin));
                const double m = pc * ia;
                w.fac[i - 1][j][2 * e] = ia;
                w.fac[i - 1][j][2 * e + 1] = pb;
                w.fac[i][j][2 * e] = m;
                w.fac[i][j][2 * e + 1] = rcp(floor_pivot(pd - m * pb, smin));
                (e ? sw1 : sw0) = s_w;
            }
        }
    }
}

// Rescale column g of the warp by s (a pair slot: both columns, its seeds once): the
// accumulator entries (every lane holding the column), the solved rows [xlo, 64) in xs,
// the seeds, and, for a column whose eigenvalue lies below the block, its stored rows
// outside the block.  Warp-uniform.
__device__ __forceinline__ void rescale_col(const DiagArgs<double> &a, WarpState &w, double (&acc)[8][2], int g,
                                            double s, int xlo, int lane)
{
    const int j = g >> 1;
    const bool pair = w.kind[j] == kSlotPair;
    const int g0 = pair ? 2 * j : g, g1 = pair ? 2 * j + 1 : g;
    if ((lane & 3) == j) {
#pragma unroll
        for (int t = 0; t < 8; t++) {
            if (pair || (g & 1) == 0) acc[t][0] *= s;
            if (pair || (g & 1) == 1) acc[t][1] *= s;
        }
    }
    for (int i = xlo + lane; i < kBlock; i += 32) {
        w.xs[i][g0] *= s;
        if (pair) w.xs[i][g1] *= s;
    }
    if (lane == 0) {
        if (pair) {
#pragma unroll
            for (int q = 0; q < 4; q++) w.seed[j][q] *= s;
        } else {
            w.seed[j][g & 1] *= s;
        }
    }
    if (w.kl[g] < 0) {  // not a diagonal column: rows stored outside the block
        for (int h = g0; h <= g1; h++) {
            const int c = w.col[h];
            double *colr = a.X + (size_t)c * a.ldx;
            scale_above(a, colr, c, s, lane);
            scale_rows(colr, a.r1, w.top[h] + 1, s, lane);
            scale_lower_y(a, a.Y + (size_t)c * a.ldy, s, lane);
        }
    }
    __syncwarp();
}

// Per-column maxima of the eight columns, from one value per lane and column of the slot
// (lanes with the same lane % 4 hold the same two columns); a pair slot combines both.
__device__ __forceinline__ void column_max(WarpState &w, double m0, double m1, int lane)
{
#pragma unroll
    for (int o = 4; o < 32; o <<= 1) {
        m0 = fmax(m0, __shfl_xor_sync(0xffffffffu, m0, o));
        m1 = fmax(m1, __shfl_xor_sync(0xffffffffu, m1, o));
    }
    if (lane < 4) {
        if (w.kind[lane] == kSlotPair) m0 = m1 = fmax(m0, m1);
        w.mx[2 * lane] = m0;
        w.mx[2 * lane + 1] = m1;
    }
    __syncwarp();
}

// One row block of the substitution (DiagArgs as for diag_solve_real; its item list is not
// used).  slots[s]: (first column, second column or -1) of slot s, in column order; slot s0
// is the first with an active column.  Grid: ceil((nslots - s0) / 32), kThreads threads,
// kSmemBytes of dynamic shared memory.
__global__ void __launch_bounds__(kThreads, 1) diag_solve_real_tc(DiagArgs<double> a, const int2 *slots, int s0,
                                                                  int nslots)
{
    extern __shared__ __align__(16) unsigned char smem_dtc[];
    __shared__ uint64_t s_sec;
    double *Ss = reinterpret_cast<double *>(smem_dtc);
    double *Ps = Ss + kSmLd * kBlock;
    WarpState &w = reinterpret_cast<WarpState *>(Ps + kSmLd * kBlock)[threadIdx.x >> 5];
    const int lane = threadIdx.x & 31;
    const int jnb = a.r1 - a.r0;
    const int sbase = s0 + (blockIdx.x * kWarps + (threadIdx.x >> 5)) * kSlots;

    // ---- the warp's columns (lane g < 8: column g, slot g / 2) --------------------------
    if (lane < kCols) {
        const int g = lane, j = g >> 1, e = g & 1;
        int c = -1, kind = kSlotEmpty;
        if (sbase + j < nslots) {
            const int2 sl = slots[sbase + j];
            const bool pair = sl.x >= 0 && a.kind[sl.x] == kPairRe;
            kind = sl.x < 0 ? kSlotEmpty : (pair ? kSlotPair : kSlotReal);
            c = e == 0 ? sl.x : (pair ? sl.x + 1 : sl.y);
        }
        const int citem = (kind == kSlotPair) ? c - e : c;  // the item's (Re) column carries the coefficients
        int k = -1;
        if (c >= 0) k = a.colk[c];
        if (c >= 0 && k < a.r0) c = -1;  // eigenvalue above the block: the column is zero here
        w.col[g] = c;
        if (e == 0) w.kind[j] = kind;
        const bool diag = c >= 0 && k < a.r1;
        w.kl[g] = diag ? k - a.r0 : -1;
        w.nrows[g] = c < 0 ? 0 : (diag ? k - a.r0 : jnb);
        w.top[g] = kind == kSlotPair ? k + 1 : k;
        w.ac[g] = c >= 0 ? a.coef[4 * citem + 0] : 0.0;
        w.br[g] = c >= 0 ? a.coef[4 * citem + 1] : 0.0;
        w.bi[g] = c >= 0 ? a.coef[4 * citem + 2] : 0.0;
        w.smin[g] = c >= 0 ? a.coef[4 * citem + 3] : 0.0;
        w.pend[g] = 1.0;
    }
    if (lane < kSlots) w.swm[lane][0] = w.swm[lane][1] = 0ull;
    load_block<double, 16>(a.S, a.lds, a.P, a.ldp, a.r0, jnb, 1, Ss, Ps);
    __syncthreads();
    pair_mask(Ss, jnb, &s_sec);
    __syncthreads();
    if (sbase >= nslots) return;  // no CTA-wide barrier below
    const uint64_t sec = s_sec;

    // ---- seeds of the diagonal columns (lane j < 4: slot j) -----------------------------
    if (lane < kSlots) {
        const int j = lane;
        double sd[4] = {0.0, 0.0, 0.0, 0.0};
        if (w.kind[j] == kSlotPair && w.kl[2 * j] >= 0) {
            const int g = 2 * j, kl = w.kl[g];
            const double ac = w.ac[g], br = w.br[g], bi = w.bi[g];
            auto W = [&](int r, int cc) -> C {
                const double s = Ss[r + cc * kSmLd], p = Ps[r + cc * kSmLd];
                return C(ac * s - br * p, -bi * p);
            };
            C sd0, sd1;
            if (!a.left_seed) {  // (x_k, x_k+1) = (-w12, w11), src/dtgevc3.cpp:727-740
                sd0 = -W(kl, kl + 1);
                sd1 = W(kl, kl);
            } else {             // the left problem's seed, mirrored
                sd0 = W(kl + 1, kl + 1);
                sd1 = -W(kl + 1, kl);
            }
            sd[0] = sd0.x; sd[1] = sd0.y; sd[2] = sd1.x; sd[3] = sd1.y;
        } else if (w.kind[j] == kSlotReal) {
            sd[0] = w.kl[2 * j] >= 0 ? 1.0 : 0.0;
            sd[1] = w.kl[2 * j + 1] >= 0 ? 1.0 : 0.0;
        }
#pragma unroll
        for (int q = 0; q < 4; q++) w.seed[j][q] = sd[q];
    }
    __syncwarp();

    // ---- right-hand sides into the accumulators -----------------------------------------
    const int js = lane & 3, gr = lane >> 2;  // this lane's slot and row within a tile
    const int kindj = w.kind[js];
    double acc[8][2];
#pragma unroll
    for (int t = 0; t < 8; t++) {
        const int row = 8 * t + gr;
        acc[t][0] = acc[t][1] = 0.0;
        if (kindj == kSlotPair) {
            const int g = 2 * js, c = w.col[g];
            if (c >= 0 && row < w.nrows[g]) {
                if (w.kl[g] >= 0) {
                    const double ac = w.ac[g], br = w.br[g], bi = w.bi[g];
                    const int kl = w.kl[g];
                    auto W = [&](int r, int cc) -> C {
                        const double s = Ss[r + cc * kSmLd], p = Ps[r + cc * kSmLd];
                        return C(ac * s - br * p, -bi * p);
                    };
                    const C v = -(W(row, kl) * C(w.seed[js][0], w.seed[js][1]) +
                                  W(row, kl + 1) * C(w.seed[js][2], w.seed[js][3]));
                    acc[t][0] = v.x;
                    acc[t][1] = v.y;
                } else {
                    acc[t][0] = a.X[(size_t)(a.r0 + row) + (size_t)c * a.ldx];
                    acc[t][1] = a.X[(size_t)(a.r0 + row) + (size_t)(c + 1) * a.ldx];
                }
            }
        } else if (kindj == kSlotReal) {
#pragma unroll
            for (int e = 0; e < 2; e++) {
                const int g = 2 * js + e, c = w.col[g];
                if (c >= 0 && row < w.nrows[g]) {
                    const int kl = w.kl[g];
                    acc[t][e] = kl >= 0 ? -(w.ac[g] * Ss[row + kl * kSmLd] - w.br[g] * Ps[row + kl * kSmLd])
                                        : a.X[(size_t)(a.r0 + row) + (size_t)c * a.ldx];
                }
            }
        }
    }
    // block check of the right-hand side: max |rhs| > bignum/10 (src/dtgevc3.cpp:688-698)
    {
        double m0 = 0.0, m1 = 0.0;
#pragma unroll
        for (int t = 0; t < 8; t++) {
            m0 = fmax(m0, fabs(acc[t][0]));
            m1 = fmax(m1, fabs(acc[t][1]));
        }
        column_max(w, m0, m1, lane);
        for (int g = 0; g < kCols; g++) {
            const int j = g >> 1;
            if (w.kind[j] == kSlotPair && (g & 1)) continue;
            if (w.col[g] < 0 || w.nrows[g] == 0 || !(w.mx[g] > a.thr_rhs)) continue;
            rescale_col(a, w, acc, g, a.thr_rhs / w.mx[g], kBlock, lane);
        }
    }

    // ---- factors of every diagonal block (8 tasks per lane: rows lane, lane + 32) -------
#pragma unroll 2
    for (int u = 0; u < 8; u++) {
        const int j = u >> 1, i = lane + 32 * (u & 1);
        bool sw0, sw1;
        factor_task(w, j, i, sec, Ss, Ps, sw0, sw1);
        const uint32_t b0 = __ballot_sync(0xffffffffu, sw0), b1 = __ballot_sync(0xffffffffu, sw1);
        if (lane == 0) {
            w.swm[j][0] |= (uint64_t)b0 << (32 * (u & 1));
            w.swm[j][1] |= (uint64_t)b1 << (32 * (u & 1));
        }
    }
    __syncwarp();

    // ---- blocked back substitution ------------------------------------------------------
    const double cap = limits<double>::big / 4096.0, target = a.thr_rhs;
    // the column of this lane's B operand entries (lane / 4)
    const int bn = lane >> 2;
    const bool b_on = w.col[bn] >= 0, b_pair = w.kind[bn >> 1] == kSlotPair;
    const int b_nr = w.nrows[bn];
    const double b_ac = w.ac[bn], b_br = w.br[bn], b_bi = w.bi[bn];
    int nmax = 0;
    for (int g = 0; g < kCols; g++) nmax = max(nmax, w.nrows[g]);
    // the mid-block check runs once the rows at and above kMidRow are solved; a 2x2 block
    // (kMidRow - 1, kMidRow) belongs to the upper part
    const int mb = ((sec >> kMidRow) & 1ull) ? kMidRow - 1 : kMidRow;
    bool mid_due = nmax > kMidRow;
    int j1 = nmax;
    while (j1 > 0) {
        int kb = min(4, j1);
        if (j1 > mb && j1 - kb < mb) kb = j1 - mb;
        if (j1 - kb >= 1 && ((sec >> (j1 - kb)) & 1ull)) kb -= 1;  // no split 2x2 block
        // 2x2 blocks never touch (greedy pairing), and neither the mid row nor a diagonal
        // column's row starts inside one, so kb >= 1 here; the floor keeps the loop finite
        kb = max(kb, 1);
        const int j0 = j1 - kb;
        // A operands of the update below: S, P rows [0, j0) of columns [j0, j0 + kb), loaded
        // before the solve (they do not depend on it)
        double sa[8], pa[8];
        {
            const int k = lane & 3, kc = min(j0 + k, kBlock - 1);
#pragma unroll
            for (int t = 0; t < 8; t++) {
                const int row = 8 * t + gr;
                const bool in = k < kb && row < j0;
                sa[t] = in ? Ss[row + kc * kSmLd] : 0.0;
                pa[t] = in ? Ps[row + kc * kSmLd] : 0.0;
            }
        }
        // the sub-block's rows to shared memory
#pragma unroll
        for (int t = 0; t < 8; t++) {
            const int row = 8 * t + gr;
            if (row >= j0 && row < j1) {
                w.xs[row][2 * js] = acc[t][0];
                w.xs[row][2 * js + 1] = acc[t][1];
            }
        }
        __syncwarp();
        if (lane < kSlots) {  // solver lane of slot `lane`
            const int j = lane;
            if (w.kind[j] == kSlotPair) {
                const int g = 2 * j, nr = w.nrows[g];
                if (w.col[g] >= 0 && j0 < nr) {
                    C rr[4], xx[4];
#pragma unroll
                    for (int u = 0; u < 4; u++) {
                        const bool in = u < kb && j0 + u < nr;
                        rr[u] = in ? C(w.xs[j0 + u][g], w.xs[j0 + u][g + 1]) : C(0.0, 0.0);
                        xx[u] = C(0.0, 0.0);
                    }
                    const double pend = solve_sub_pair(rr, xx, j0, kb, nr, sec, w.swm[j][0], w, j, w.ac[g],
                                                       C(w.br[g], w.bi[g]), Ss, Ps, cap, target);
#pragma unroll
                    for (int u = 0; u < 4; u++)
                        if (u < kb && j0 + u < nr) {
                            w.xs[j0 + u][g] = xx[u].x;
                            w.xs[j0 + u][g + 1] = xx[u].y;
                        }
                    w.pend[g] = w.pend[g + 1] = pend;
                }
            } else if (w.kind[j] == kSlotReal) {
#pragma unroll
                for (int e = 0; e < 2; e++) {
                    const int g = 2 * j + e, nr = w.nrows[g];
                    if (w.col[g] < 0 || j0 >= nr) continue;
                    double rr[4], xx[4];
#pragma unroll
                    for (int u = 0; u < 4; u++) {
                        rr[u] = (u < kb && j0 + u < nr) ? w.xs[j0 + u][g] : 0.0;
                        xx[u] = 0.0;
                    }
                    const double pend = solve_sub_real(rr, xx, j0, kb, nr, sec, w.swm[j][e], w, j, e, w.ac[g],
                                                       w.br[g], Ss, Ps, cap, target);
#pragma unroll
                    for (int u = 0; u < 4; u++)
                        if (u < kb && j0 + u < nr) w.xs[j0 + u][g] = xx[u];
                    w.pend[g] = pend;
                }
            }
        }
        __syncwarp();
        // a per-row cap fired: the rest of the column (the sub-block is already scaled)
        bool fired = false;
        if (lane < kCols) fired = w.pend[lane] != 1.0;
        if (__any_sync(0xffffffffu, fired))
        for (int g = 0; g < kCols; g++) {
            const double s = w.pend[g];
            if (s == 1.0) continue;
            const bool pair = w.kind[g >> 1] == kSlotPair;
            if (!(pair && (g & 1))) rescale_col(a, w, acc, g, s, j1, lane);
            __syncwarp();
            if (lane == 0) w.pend[g] = 1.0;
            __syncwarp();
        }
        // B operands: row j0 + lane % 4 of column lane / 4, U = -ac x, V = b x
        double bu = 0.0, bv = 0.0;
        {
            const int k = lane & 3, row = j0 + k;
            if (k < kb && b_on && row < b_nr) {
                if (b_pair) {
                    const double xr = w.xs[row][bn & ~1], xi = w.xs[row][bn | 1];
                    bu = -b_ac * ((bn & 1) ? xi : xr);
                    bv = (bn & 1) ? b_br * xi + b_bi * xr : b_br * xr - b_bi * xi;
                } else {
                    const double x = w.xs[row][bn];
                    bu = -b_ac * x;
                    bv = b_br * x;
                }
            }
        }
        // rows above the sub-block: acc += S(rows, j0 + k) U, then + P(rows, j0 + k) V (the
        // S products of all tiles first: independent MMAs back to back)
#pragma unroll
        for (int t = 0; t < 8; t++)
            if (8 * t < j0) dmma884(acc[t][0], acc[t][1], sa[t], bu);
#pragma unroll
        for (int t = 0; t < 8; t++)
            if (8 * t < j0) dmma884(acc[t][0], acc[t][1], pa[t], bv);
        // mid-block check of the columns with rows below kMidRow: rows [0, mb)
        if (mid_due && j0 == mb) {
            mid_due = false;
            double m0 = 0.0, m1 = 0.0;
#pragma unroll
            for (int t = 0; t < 4; t++) {
                if (8 * t + gr < mb) {
                    m0 = fmax(m0, fabs(acc[t][0]));
                    m1 = fmax(m1, fabs(acc[t][1]));
                }
            }
            column_max(w, m0, m1, lane);
            for (int g = 0; g < kCols; g++) {
                if (w.kind[g >> 1] == kSlotPair && (g & 1)) continue;
                if (w.col[g] < 0 || w.nrows[g] <= kMidRow || !(w.mx[g] > a.thr_rhs)) continue;
                rescale_col(a, w, acc, g, a.thr_rhs / w.mx[g], mb, lane);
            }
        }
        j1 = j0;
    }

    // ---- block check before the update: max(|ac x|, |b x|) > bignum / jnb (src/dtgevc3.cpp:1404-1426)
    {
        double m0 = 0.0, m1 = 0.0;
        if (kindj == kSlotPair) {
            const int g = 2 * js;
            if (w.col[g] >= 0) {
                const int nr = w.nrows[g], kl = w.kl[g];
                const double ac = w.ac[g];
                const C b(w.br[g], w.bi[g]);
                const C sd0(w.seed[js][0], w.seed[js][1]), sd1(w.seed[js][2], w.seed[js][3]);
                for (int i = gr; i < kBlock; i += 8) {
                    C x(0.0, 0.0);
                    if (i < nr) x = C(w.xs[i][g], w.xs[i][g + 1]);
                    else if (kl >= 0 && i == kl) x = sd0;
                    else if (kl >= 0 && i == kl + 1) x = sd1;
                    const C ys = ac * x, yp = b * x;
                    m0 = fmax(m0, fmax(fmax(fabs(ys.x), fabs(ys.y)), fmax(fabs(yp.x), fabs(yp.y))));
                }
            }
        } else if (kindj == kSlotReal) {
#pragma unroll
            for (int e = 0; e < 2; e++) {
                const int g = 2 * js + e;
                if (w.col[g] < 0) continue;
                const int nr = w.nrows[g], kl = w.kl[g];
                const double ac = w.ac[g], br = w.br[g], sd = w.seed[js][e];
                double m = 0.0;
                for (int i = gr; i < kBlock; i += 8) {
                    const double x = i < nr ? w.xs[i][g] : (i == kl ? sd : 0.0);
                    m = fmax(m, fmax(fabs(ac * x), fabs(br * x)));
                }
                if (e) m1 = m;
                else m0 = m;
            }
        }
        column_max(w, m0, m1, lane);
        for (int g = 0; g < kCols; g++) {
            if (w.kind[g >> 1] == kSlotPair && (g & 1)) continue;
            if (w.col[g] < 0 || !(w.mx[g] > a.thr_upd)) continue;
            rescale_col(a, w, acc, g, a.thr_upd / w.mx[g], 0, lane);
        }
    }

    // ---- output: X rows of the block, the update operand rows ----------------------------
    for (int g = 0; g < kCols; g++) {
        const int c = w.col[g];
        if (c < 0) continue;
        const int j = g >> 1, e = g & 1, gb = g & ~1;
        const bool pair = w.kind[j] == kSlotPair;
        const int nr = w.nrows[g], kl = w.kl[g];
        const double ac = w.ac[g], br = w.br[g], bi = w.bi[g];
        // seeds at rows kl (and kl + 1): this column's, and for a pair both columns'
        const double sa0 = pair ? w.seed[j][0] : w.seed[j][e], sa1 = pair ? w.seed[j][2] : 0.0;  // Re / real
        const double sb0 = pair ? w.seed[j][1] : 0.0, sb1 = pair ? w.seed[j][3] : 0.0;            // Im
        double *colr = a.X + (size_t)c * a.ldx;
        double *ycol = a.Y + (size_t)c * a.ldy;
        for (int i = lane; i < a.ypad; i += 32) {
            double ys = 0.0, yp = 0.0;
            if (i < jnb) {
                double xr, xi = 0.0;
                if (i < nr) {
                    xr = w.xs[i][pair ? gb : g];
                    if (pair) xi = w.xs[i][gb + 1];
                } else {
                    xr = (kl >= 0 && i == kl) ? sa0 : ((pair && kl >= 0 && i == kl + 1) ? sa1 : 0.0);
                    xi = (kl >= 0 && i == kl) ? sb0 : ((pair && kl >= 0 && i == kl + 1) ? sb1 : 0.0);
                }
                const double x = (pair && e) ? xi : xr;
                ys = -ac * x;
                yp = pair ? (e ? br * xi + bi * xr : br * xr - bi * xi) : br * x;
                colr[a.r0 + i] = x;
            }
            ycol[a.ys_off + i] = ys;
            ycol[a.ys_off + a.yhalf + i] = yp;
        }
        if (kl >= 0)
            for (int i = lane; i < a.zl_len; i += 32) {
                ycol[a.zl_off + i] = 0.0;
                ycol[a.zl_off + a.yhalf + i] = 0.0;
            }
    }
}

}  // namespace dtc
}  // namespace xtg
