// C-linkage forwarding stubs over the upstream xTGEVC3 entry points.
//
// TEST INFRASTRUCTURE ONLY: this file is compiled together with the upstream
// sources (src/{d,s,z,c}tgevc3.cpp, whose prototypes are in include/tgevc3.h:9-12)
// into oracle/_ref/libref_tgevc3.so.  The upstream functions have C++ linkage,
// so ctypes cannot name them portably; these stubs give them flat names.
// Complex arrays are passed as interleaved (re, im) pairs, which is the layout
// of std::complex<T>.
#include <complex>
#include "tgevc3.h"

extern "C" {
void scipy_openblas_set_num_threads(int);

void ref_set_num_threads(int n) { scipy_openblas_set_num_threads(n); }

void ref_dtgevc3(char side, char howmny, const int *select, int n, const double *S, int lds,
                 const double *P, int ldp, const double *alphar, const double *alphai,
                 const double *beta, double *VL, int ldvl, double *VR, int ldvr, int mm, int *m,
                 double *work, int lwork, int *info)
{
    dtgevc3(side, howmny, select, n, S, lds, P, ldp, alphar, alphai, beta, VL, ldvl, VR, ldvr, mm,
            m, work, lwork, info);
}

void ref_stgevc3(char side, char howmny, const int *select, int n, const float *S, int lds,
                 const float *P, int ldp, const float *alphar, const float *alphai,
                 const float *beta, float *VL, int ldvl, float *VR, int ldvr, int mm, int *m,
                 float *work, int lwork, int *info)
{
    stgevc3(side, howmny, select, n, S, lds, P, ldp, alphar, alphai, beta, VL, ldvl, VR, ldvr, mm,
            m, work, lwork, info);
}

void ref_ztgevc3(char side, char howmny, const int *select, int n, const double *S, int lds,
                 const double *P, int ldp, const double *alpha, const double *beta, double *VL,
                 int ldvl, double *VR, int ldvr, int mm, int *m, double *work, int lwork, int *info)
{
    using C = std::complex<double>;
    ztgevc3(side, howmny, select, n, (const C *)S, lds, (const C *)P, ldp, (const C *)alpha,
            (const C *)beta, (C *)VL, ldvl, (C *)VR, ldvr, mm, m, (C *)work, lwork, info);
}

void ref_ctgevc3(char side, char howmny, const int *select, int n, const float *S, int lds,
                 const float *P, int ldp, const float *alpha, const float *beta, float *VL,
                 int ldvl, float *VR, int ldvr, int mm, int *m, float *work, int lwork, int *info)
{
    using C = std::complex<float>;
    ctgevc3(side, howmny, select, n, (const C *)S, lds, (const C *)P, ldp, (const C *)alpha,
            (const C *)beta, (C *)VL, ldvl, (C *)VR, ldvr, mm, m, (C *)work, lwork, info);
}
}
