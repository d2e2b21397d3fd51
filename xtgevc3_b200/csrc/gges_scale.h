// xGGES's scaling of the input pencil (host code): LAPACK xGGES scales A (and B) when its
// largest entry in modulus lies outside [smlnum, bignum] (smlnum = sqrt(safmin) / eps, bignum =
// 1 / smlnum), runs the QZ step on the scaled pencil, and scales the Schur form and the
// eigenvalues back at the end.  The multiplications follow xLASCL: cfrom -> cto as a product of
// factors that neither overflow nor underflow (safmin or 1 / safmin while the ratio is out of
// range, then the remaining ratio), each applied to every entry in turn.  Real pencils also
// take DGGES's guard before the eigenvalues are scaled back: a complex pair whose alphar or
// alphai (or beta) would overflow or underflow in the unscaling is first rescaled by
// |A(i, i) / alphar(i)| (or |A(i, i+1) / alphai(i)|, |B(i, i) / beta(i)|).
#pragma once

#include <cmath>
#include <limits>

namespace xtg {
namespace gs {

template <class R>
struct Lim {
    static constexpr R safmin = std::numeric_limits<R>::min();   // xLAMCH('S')
    static constexpr R prec = std::numeric_limits<R>::epsilon();  // xLAMCH('P')
};

// xLASCL's factors taking cfrom to cto (at most 8; 0 when the ratio is exactly 1)
template <class R>
int lascl_steps(R cfrom, R cto, R *mul)
{
    const R smlnum = Lim<R>::safmin, bignum = R(1) / smlnum;
    R cfromc = cfrom, ctoc = cto;
    int k = 0;
    for (bool done = false; !done && k < 8;) {
        const R cfrom1 = cfromc * smlnum;
        R m;
        if (cfrom1 == cfromc) {  // cfromc infinite
            m = ctoc / cfromc;
            done = true;
        } else {
            const R cto1 = ctoc / bignum;
            if (cto1 == ctoc) {  // ctoc 0 or infinite
                m = ctoc;
                done = true;
            } else if (std::fabs(cfrom1) > std::fabs(ctoc) && ctoc != R(0)) {
                m = smlnum;
                cfromc = cfrom1;
            } else if (std::fabs(cto1) > std::fabs(cfromc)) {
                m = bignum;
                ctoc = cto1;
            } else {
                m = ctoc / cfromc;
                done = true;
                if (m == R(1)) break;
            }
        }
        mul[k++] = m;
    }
    return k;
}

template <class R>
void lascl_apply(int k, const R *mul, R *x, size_t count)
{
    for (int s = 0; s < k; s++)
        for (size_t i = 0; i < count; i++) x[i] *= mul[s];
}

// DGGES's scale decision for a norm: 0 (none), else *to = smlnum or bignum
template <class R>
bool needs_scaling(R nrm, R *to)
{
    const R smlnum = std::sqrt(Lim<R>::safmin) / Lim<R>::prec, bignum = R(1) / smlnum;
    if (nrm > R(0) && nrm < smlnum) {
        *to = smlnum;
        return true;
    }
    if (nrm > bignum) {
        *to = bignum;
        return true;
    }
    return false;
}

// DGGES's guard before the unscaling of a real pencil's eigenvalues (see the file comment).
// aii, aii1, bii: A(i, i), A(i, i + 1), B(i, i) of the scaled Schur form (n each; aii1[n-1]
// unused).
template <class R>
void pair_guard(int n, bool ilascl, R anrm, R anrmto, bool ilbscl, R bnrm, R bnrmto, const R *aii, const R *aii1,
                const R *bii, R *alphar, R *alphai, R *beta)
{
    const R safmin = Lim<R>::safmin, safmax = R(1) / safmin;
    if (ilascl)
        for (int i = 0; i < n; i++) {
            if (alphai[i] == R(0)) continue;
            R w = R(-1);
            if (alphar[i] / safmax > anrmto / anrm || safmin / alphar[i] > anrm / anrmto)
                w = std::fabs(aii[i] / alphar[i]);
            else if (alphai[i] / safmax > anrmto / anrm || safmin / alphai[i] > anrm / anrmto)
                w = std::fabs(aii1[i] / alphai[i]);
            if (w >= R(0)) {
                beta[i] *= w;
                alphar[i] *= w;
                alphai[i] *= w;
            }
        }
    if (ilbscl)
        for (int i = 0; i < n; i++) {
            if (alphai[i] == R(0)) continue;
            if (beta[i] / safmax > bnrmto / bnrm || safmin / beta[i] > bnrm / bnrmto) {
                const R w = std::fabs(bii[i] / beta[i]);
                beta[i] *= w;
                alphar[i] *= w;
                alphai[i] *= w;
            }
        }
}

}  // namespace gs
}  // namespace xtg
