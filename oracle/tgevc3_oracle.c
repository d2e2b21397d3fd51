/*
 * CPU oracle for the blocked generalized-eigenvector path (xTGEVC3).
 *
 * TEST INFRASTRUCTURE ONLY.  This restates, in plain C with no BLAS, the algorithm of
 * the upstream project's src/{d,s,z,c}tgevc3.cpp so that tests and the CPU leg of
 * bench.py can check the CUDA product against it.  Nothing in the product links it.
 * It is pinned against outputs of the upstream library itself (fixtures under
 * tests/golden/, generated by tests/golden/make_golden.py from oracle/_ref).
 *
 * Exported (C linkage):
 *   oracle_dtgevc3 / oracle_stgevc3 : real, same argument list as upstream dtgevc3
 *   oracle_ztgevc3 / oracle_ctgevc3 : complex, interleaved (re, im) arrays
 */
#include <complex.h>
#include <float.h>
#include <math.h>
#include <stddef.h>

/* ---- double ---- */
#define R double
#define FN(x) oracle_d##x
#define RABS fabs
#define SAFEMIN DBL_MIN
#define EPSILON DBL_EPSILON
#include "tgevc3_oracle_real.inc"
#undef FN

#define C double complex
#define FN(x) oracle_z##x
#define CABS cabs
#define CONJ conj
#define CREAL creal
#define CIMAG cimag
#include "tgevc3_oracle_cplx.inc"
#undef FN
#undef C
#undef CABS
#undef CONJ
#undef CREAL
#undef CIMAG
#undef R
#undef RABS
#undef SAFEMIN
#undef EPSILON

/* ---- float ---- */
#define R float
#define FN(x) oracle_s##x
#define RABS fabsf
#define SAFEMIN FLT_MIN
#define EPSILON FLT_EPSILON
#include "tgevc3_oracle_real.inc"
#undef FN

#define C float complex
#define FN(x) oracle_c##x
#define CABS cabsf
#define CONJ conjf
#define CREAL crealf
#define CIMAG cimagf
#include "tgevc3_oracle_cplx.inc"
#undef FN
