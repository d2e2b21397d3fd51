// Drop-in C++ interface: the same four prototypes (C++ linkage, scalars by value) as the
// upstream header include/tgevc3.h:9-12, so code written against the upstream library
// compiles and links unchanged against libxtgevc3.so.  Behaviour: see xtgevc3.h.
#pragma once

#include <complex>

#ifndef RP
#define RP(T) T *__restrict
#endif

// replaces upstream dtgevc3 (src/dtgevc3.cpp:1150)
void dtgevc3(char side, char howmny, const int *select, int n, const double *S, int lds, const double *P, int ldp,
             const double *alphar, const double *alphai, const double *beta, RP(double) VL, int ldvl, RP(double) VR,
             int ldvr, int mm, int *m, RP(double) work, int lwork, int *info);
// replaces upstream stgevc3 (src/stgevc3.cpp:1122)
void stgevc3(char side, char howmny, const int *select, int n, const float *S, int lds, const float *P, int ldp,
             const float *alphar, const float *alphai, const float *beta, RP(float) VL, int ldvl, RP(float) VR,
             int ldvr, int mm, int *m, RP(float) work, int lwork, int *info);
// replaces upstream ztgevc3 (src/ztgevc3.cpp:435)
void ztgevc3(char side, char howmny, const int *select, int n, const std::complex<double> *S, int lds,
             const std::complex<double> *P, int ldp, const std::complex<double> *alpha,
             const std::complex<double> *beta, RP(std::complex<double>) VL, int ldvl, RP(std::complex<double>) VR,
             int ldvr, int mm, int *m, RP(std::complex<double>) work, int lwork, int *info);
// replaces upstream ctgevc3 (src/ctgevc3.cpp:435)
void ctgevc3(char side, char howmny, const int *select, int n, const std::complex<float> *S, int lds,
             const std::complex<float> *P, int ldp, const std::complex<float> *alpha, const std::complex<float> *beta,
             RP(std::complex<float>) VL, int ldvl, RP(std::complex<float>) VR, int ldvr, int mm, int *m,
             RP(std::complex<float>) work, int lwork, int *info);
