/*
 * xtgevc3 -- C ABI of the B200 (sm_100a) implementation of the blocked generalized
 * eigenvector routines xTGEVC3.
 *
 * Given an upper quasi-triangular S and upper triangular P (real), or upper triangular S
 * and P (complex), as produced by a generalized Schur factorisation (xGGES), compute some
 * or all right eigenvectors x (beta*S*x = alpha*P*x) and/or left eigenvectors y
 * (y^H*(beta*S - alpha*P) = 0), optionally multiplied by the Schur vectors Z / Q.
 *
 * Argument meaning, INFO codes and the LWORK=-1 workspace query are those of the upstream
 * library (include/tgevc3.h:9-12 of vlovero/xTGEVC3):
 *   side    'R', 'L' or 'B' (any other value computes nothing and returns INFO = 0)
 *   howmny  'A' all, 'B' all and back-transformed by VR = Z / VL = Q given on entry,
 *           'S' the eigenvalues flagged in select (a complex pair counts when either of its
 *           two flags is set; select may be NULL, which selects nothing)
 *   mm      columns available in VL/VR;  *m (may be NULL) receives the columns used
 *   work/lwork  lwork = -1 returns the upstream workspace size in work[0]; the GPU path
 *           does not use the workspace but keeps the size rule and its error code
 *   info    0 success, -2 bad howmny, -16 mm too small, -19 lwork too small,
 *           1 a CUDA call failed (text in xtgevc3_last_error()); positive codes are new:
 *           the upstream code never returns them.
 * Real pencils return a complex pair (k, k+1) as two columns (Re x, Im x) of the
 * eigenvector for alphar[k] + i*alphai[k] (alphai[k] > 0); columns are in ascending
 * eigenvalue order.  Complex arrays are interleaved (re, im) pairs, the layout of
 * std::complex / C99 _Complex.  Matrices are column-major.
 *
 * Output scale: unless XTGEVC3_NORMALIZE is set the eigenvectors carry the scale of the
 * upstream algorithm (x_k = 1 on the eigenvalue's own row); when the overflow guards fire,
 * this implementation scales single columns where the upstream code scales a 32-column
 * panel, so those columns differ from the upstream output by a positive factor.
 *
 * Host-pointer calls of real pencils upload S and P while the solve runs and compute the
 * pencil norms on up to 32 host threads of their own, joined before the call returns.
 */
#ifndef XTGEVC3_H
#define XTGEVC3_H

#ifdef __cplusplus
extern "C" {
#endif

/* Option flags. */
#define XTGEVC3_NORMALIZE 1u /* scale every eigenvector (a real pair jointly) to max_i |re|+|im| = 1 */
#define XTGEVC3_SIMT 2u      /* use the SIMT GEMM kernels instead of the FP64 tensor-core kernel */
/* Split-precision form (dtgevc3 only): the trailing updates and the back-transform run as
 * products of BF16 slices of the FP64 operands on the BF16 tensor cores, with exact FP32
 * accumulation per 128-deep K chunk and FP64 summation; the diagonal solves, scale factors
 * and 2x2 solves stay FP64.  XTGEVC3_SLICES(s) picks the slice count s in [1, 6] (default 6,
 * ~48 bits per operand). */
#define XTGEVC3_SPLIT 4u
#define XTGEVC3_SLICES(s) ((unsigned)(s) << 8)
/* With XTGEVC3_SPLIT: INT8 slices (7-bit digits, s in [1, 7], default 7, ~49 bits per
 * operand) on the INT8 tensor cores with exact INT32 accumulation over the whole K. */
#define XTGEVC3_SPLIT_INT8 8u
/* With XTGEVC3_SPLIT: residue form.  Each row of A / column of B is scaled by a power of two
 * to an integer of t bits; the product of the integers is recovered exactly from its
 * residues modulo L pairwise-coprime moduli <= 256 (Chinese remainder theorem), one INT8
 * tensor-core GEMM with exact INT32 sums per modulus.  XTGEVC3_SLICES(L) picks L in [2, 16]
 * (default 14: ~47-bit operands at K = 8192; t = floor((log2 P - ceil(log2 K) - 2) / 2)).
 * L products replace the s(s+1)/2 of the digit slices. */
#define XTGEVC3_SPLIT_CRT 32u
/* Split forms: after the split pass, each eigenvector's relative residual in Schur
 * coordinates, ||(beta S - alpha P) x||_2 / ((|beta| ||S||_1 + |alpha| ||P||_1) ||x||_2) in
 * the scaling of the solve, is estimated from a 16-row random sketch; eigenvectors whose
 * estimate exceeds a quarter of the bound (1e-12; the environment variable
 * XTGEVC3_REFINE_BOUND overrides it) are solved again with FP64 GEMMs (the refinement step)
 * and overwrite their output columns.  XTGEVC3_SPLIT_NO_REFINE skips the check. */
#define XTGEVC3_SPLIT_NO_REFINE 64u
/* Look-ahead schedule: the trailing update of each pair of row blocks runs on a second
 * stream while the next pair's diagonal solves run (guard rescaling of the rows that
 * update writes is deferred until it has finished).  Same results to rounding (the default
 * schedule sums the updates of two row blocks in one GEMM); on B200 it measured no faster
 * (the update fills the GPU), so it is off by default. */
#define XTGEVC3_LOOKAHEAD 16u

/* ---- split-precision GEMM on device operands (no upstream counterpart) ----------------
 * C (+)= A B with column-major FP64 A (M x K), B (K x N), C (M x N) on the device, through
 * the tensor-core path of a split form: kind 0 BF16 slices, 1 INT8 digit slices, 2 INT8
 * residues; slices = the slice / modulus count (0: the form's default).  K < 65536.  The
 * building block of the split forms, exposed for testing and measurement.  Synchronous on
 * `stream`; returns 0, 1 (CUDA failure, message in xtgevc3_last_error()) or -1 (bad
 * argument). */
int xtgevc3_split_gemm_dev(void *stream, int kind, int slices, int M, int N, int K, const double *A, int lda,
                           const double *B, int ldb, double *C, int ldc, int accumulate);

/* Process-wide flags used by the drop-in entry points below (default 0). */
void xtgevc3_set_flags(unsigned flags);
unsigned xtgevc3_get_flags(void);

/* Text of the last CUDA failure seen by the calling thread ("" if none). */
const char *xtgevc3_last_error(void);

/* ---- kernel trace (no upstream counterpart) -------------------------------------------
 * When enabled, every kernel the library launches is bracketed by CUDA events on its
 * stream; per kernel class the launch count, summed device time (ms) and algorithmic
 * flops / bytes (operation counts of the math, not hardware counters) accumulate until
 * reset.  Classes: 0 prep, 1 diag_solve, 2 gemm_update, 3 gemm_backtransform,
 * 4 writeback, 5 normalize.  xtgevc3_trace_get returns -1 for an unknown class.
 * xtgevc3_launch_count counts every kernel launched by the library (traced or not). */
void xtgevc3_trace_enable(int on);
void xtgevc3_trace_reset(void);
int xtgevc3_trace_get(int cls, long long *launches, double *ms, double *flops, double *bytes);
const char *xtgevc3_trace_name(int cls);
long long xtgevc3_launch_count(void);
/* Eigenvector columns that the calling thread's last split-form call solved again in FP64
 * (0 after any other call). */
int xtgevc3_split_refined(void);

/* ---- host-pointer entry points (drop-in) -------------------------------------------
 * C-linkage twins of dtgevc3/stgevc3/ztgevc3/ctgevc3 (include/tgevc3.h).  Inputs are
 * copied to the current CUDA device, results copied back before return.             */

/* replaces upstream dtgevc3, src/dtgevc3.cpp:1150 */
void xtgevc3_dtgevc3(char side, char howmny, const int *select, int n, const double *S, int lds, const double *P,
                     int ldp, const double *alphar, const double *alphai, const double *beta, double *VL, int ldvl,
                     double *VR, int ldvr, int mm, int *m, double *work, int lwork, int *info);
/* replaces upstream stgevc3, src/stgevc3.cpp:1122 */
void xtgevc3_stgevc3(char side, char howmny, const int *select, int n, const float *S, int lds, const float *P,
                     int ldp, const float *alphar, const float *alphai, const float *beta, float *VL, int ldvl,
                     float *VR, int ldvr, int mm, int *m, float *work, int lwork, int *info);
/* replaces upstream ztgevc3, src/ztgevc3.cpp:435 (complex arrays interleaved) */
void xtgevc3_ztgevc3(char side, char howmny, const int *select, int n, const double *S, int lds, const double *P,
                     int ldp, const double *alpha, const double *beta, double *VL, int ldvl, double *VR, int ldvr,
                     int mm, int *m, double *work, int lwork, int *info);
/* replaces upstream ctgevc3, src/ctgevc3.cpp:435 (complex arrays interleaved) */
void xtgevc3_ctgevc3(char side, char howmny, const int *select, int n, const float *S, int lds, const float *P,
                     int ldp, const float *alpha, const float *beta, float *VL, int ldvl, float *VR, int ldvr, int mm,
                     int *m, float *work, int lwork, int *info);

/* ---- device-pointer entry points ----------------------------------------------------
 * Same computation on matrices already resident on the current CUDA device: S, P, VL, VR
 * are device pointers; the alpha, alphai, beta and select arrays are HOST arrays of
 * length n.  Work is queued on
 * `stream` (a cudaStream_t, NULL = legacy default stream) and complete on return.
 * Scratch memory comes from the device's stream-ordered pool.  INFO as above (no
 * workspace argument, so no -19).  Returns 0, or 1 if a CUDA call failed.
 * These have no upstream counterpart (the upstream library is CPU-only).              */
int xtgevc3_dtgevc3_dev(unsigned flags, void *stream, char side, char howmny, const int *select, int n,
                        const double *S, int lds, const double *P, int ldp, const double *alphar,
                        const double *alphai, const double *beta, double *VL, int ldvl, double *VR, int ldvr, int mm,
                        int *m, int *info);
int xtgevc3_stgevc3_dev(unsigned flags, void *stream, char side, char howmny, const int *select, int n,
                        const float *S, int lds, const float *P, int ldp, const float *alphar, const float *alphai,
                        const float *beta, float *VL, int ldvl, float *VR, int ldvr, int mm, int *m, int *info);
int xtgevc3_ztgevc3_dev(unsigned flags, void *stream, char side, char howmny, const int *select, int n,
                        const double *S, int lds, const double *P, int ldp, const double *alpha, const double *beta,
                        double *VL, int ldvl, double *VR, int ldvr, int mm, int *m, int *info);
int xtgevc3_ctgevc3_dev(unsigned flags, void *stream, char side, char howmny, const int *select, int n,
                        const float *S, int lds, const float *P, int ldp, const float *alpha, const float *beta,
                        float *VL, int ldvl, float *VR, int ldvr, int mm, int *m, int *info);

/* ---- standard eigenproblem: xTREVC3 (no counterpart in the upstream library) ----------
 * Right and/or left eigenvectors of an upper quasi-triangular Schur factor T (from LAPACK
 * xHSEQR / xGEES: real T with standardised 2x2 blocks; complex T upper triangular), with
 * the argument meaning, INFO codes and results of LAPACK xTREVC3 (the upstream benchmarks
 * time LAPACK's dtrevc3 beside dtgevc3, benchmarks/bench_dtgevc3.cpp:127-149): HOWMNY 'A',
 * 'B' (VL/VR hold Q on entry) or 'S'; every eigenvector scaled so that its largest
 * component has |re| + |im| = 1; a real pair stored as (Re, Im) columns with LAPACK's
 * phase.  Eigenvalues are read from T's diagonal blocks.  Computed by the generalized
 * solver with P = I (built on the device; its zero strips are skipped).  Differences from
 * LAPACK: SELECT is read-only (LAPACK rewrites a pair's flags), WORK is not used (a query,
 * LWORK = -1, answers the minimum max(1, 3n), complex max(1, 2n) and LRWORK max(1, n)).
 * INFO: -1 SIDE, -2 HOWMNY, -4 N, -6 LDT, -8 LDVL, -10 LDVR, -11 MM < M, -14 LWORK,
 * -16 LRWORK (complex), 1 a CUDA failure.  Complex arrays interleaved.                  */
void xtgevc3_dtrevc3(char side, char howmny, const int *select, int n, const double *T, int ldt, double *VL,
                     int ldvl, double *VR, int ldvr, int mm, int *m, double *work, int lwork, int *info);
void xtgevc3_strevc3(char side, char howmny, const int *select, int n, const float *T, int ldt, float *VL, int ldvl,
                     float *VR, int ldvr, int mm, int *m, float *work, int lwork, int *info);
void xtgevc3_ztrevc3(char side, char howmny, const int *select, int n, const double *T, int ldt, double *VL,
                     int ldvl, double *VR, int ldvr, int mm, int *m, double *work, int lwork, double *rwork,
                     int lrwork, int *info);
void xtgevc3_ctrevc3(char side, char howmny, const int *select, int n, const float *T, int ldt, float *VL, int ldvl,
                     float *VR, int ldvr, int mm, int *m, float *work, int lwork, float *rwork, int lrwork, int *info);
/* device forms: T, VL, VR device pointers, select a host array; flags as the _dev forms
 * above (XTGEVC3_NORMALIZE is implied); returns 0, or 1 if a CUDA call failed           */
int xtgevc3_dtrevc3_dev(unsigned flags, void *stream, char side, char howmny, const int *select, int n,
                        const double *T, int ldt, double *VL, int ldvl, double *VR, int ldvr, int mm, int *m,
                        int *info);
int xtgevc3_strevc3_dev(unsigned flags, void *stream, char side, char howmny, const int *select, int n,
                        const float *T, int ldt, float *VL, int ldvl, float *VR, int ldvr, int mm, int *m, int *info);
int xtgevc3_ztrevc3_dev(unsigned flags, void *stream, char side, char howmny, const int *select, int n,
                        const double *T, int ldt, double *VL, int ldvl, double *VR, int ldvr, int mm, int *m,
                        int *info);
int xtgevc3_ctrevc3_dev(unsigned flags, void *stream, char side, char howmny, const int *select, int n,
                        const float *T, int ldt, float *VL, int ldvl, float *VR, int ldvr, int mm, int *m, int *info);

/* ---- condition numbers: xTGSNA (no counterpart upstream) ----------------------------------
 * LAPACK xTGSNA's arguments, INFO codes and results for the selected eigenvalues of a
 * generalized Schur pencil (A, B) (quasi-triangular A, triangular B):
 * S (JOB = 'E' or 'B'): reciprocal condition numbers of the eigenvalues,
 * S(k) = sqrt(|y^H A x|^2 + |y^H B x|^2) / (||x|| ||y||), from the left and right
 * eigenvectors VL, VR in Schur coordinates (as xtgevc3_*tgevc3 return them with HOWMNY 'A'
 * or 'S'); a real pair (A(k+1,k) != 0) gets one S for both columns; S = -1 where the
 * numerator is zero (not for a pair, as in LAPACK).
 * DIF (JOB = 'V' or 'B'): LAPACK's estimate of the reciprocal condition number of the
 * eigenvectors, as xTGSNA computes it: a copy of the pencil with the eigenvalue's block
 * reordered to the top (DIF = 0 when a swap is rejected), then xTGSYL's Frobenius-norm
 * estimate for the rest of the pencil (+-1 right-hand sides chosen by look-ahead), a real
 * pair's own 2x2 bound taken as well.  Complex pencils: the reordering is LAPACK's rotations,
 * DIF agrees with LAPACK's to rounding.  Real pencils: the look-ahead choices depend on the
 * signs of the reordered copy, which LAPACK itself leaves to rounding noise in swaps of 2x2
 * blocks; where the copy has LAPACK's signs, DIF agrees with LAPACK's to rounding,
 * elsewhere it is an estimate of the same quality (both within a small factor above the
 * true smallest singular value).
 * VL, VR are not referenced for JOB = 'V'; IWORK is not referenced and WORK is not used
 * (the query, LWORK = -1, answers LAPACK's LWORK: max(1, n) for JOB = 'E'; with DIF
 * 2 n (n + 2) + 16 for real, 2 n^2 for complex pencils).  INFO: -1 JOB, -2 HOWMNY, -4 N,
 * -6 LDA, -8 LDB, -10 LDVL, -12 LDVR (JOB 'E' or 'B'), -15 MM < M, -18 LWORK, 1 a CUDA
 * failure.  Complex arrays interleaved (S, DIF real).  Device forms: S only (JOB = 'E'; other
 * JOB values return INFO = -1), A, B, VL, VR and S device pointers; DIF on the device:
 * xtgevc3_*tgsna_dif_dev below.                                                            */
void xtgevc3_dtgsna(char job, char howmny, const int *select, int n, const double *A, int lda, const double *B,
                    int ldb, const double *VL, int ldvl, const double *VR, int ldvr, double *s, double *dif, int mm,
                    int *m, double *work, int lwork, int *iwork, int *info);
void xtgevc3_stgsna(char job, char howmny, const int *select, int n, const float *A, int lda, const float *B, int ldb,
                    const float *VL, int ldvl, const float *VR, int ldvr, float *s, float *dif, int mm, int *m,
                    float *work, int lwork, int *iwork, int *info);
void xtgevc3_ztgsna(char job, char howmny, const int *select, int n, const double *A, int lda, const double *B,
                    int ldb, const double *VL, int ldvl, const double *VR, int ldvr, double *s, double *dif, int mm,
                    int *m, double *work, int lwork, int *iwork, int *info);
void xtgevc3_ctgsna(char job, char howmny, const int *select, int n, const float *A, int lda, const float *B, int ldb,
                    const float *VL, int ldvl, const float *VR, int ldvr, float *s, float *dif, int mm, int *m,
                    float *work, int lwork, int *iwork, int *info);
int xtgevc3_dtgsna_dev(void *stream, char job, char howmny, const int *select, int n, const double *A, int lda,
                       const double *B, int ldb, const double *VL, int ldvl, const double *VR, int ldvr, double *s,
                       int mm, int *m, int *info);
int xtgevc3_stgsna_dev(void *stream, char job, char howmny, const int *select, int n, const float *A, int lda,
                       const float *B, int ldb, const float *VL, int ldvl, const float *VR, int ldvr, float *s, int mm,
                       int *m, int *info);
int xtgevc3_ztgsna_dev(void *stream, char job, char howmny, const int *select, int n, const double *A, int lda,
                       const double *B, int ldb, const double *VL, int ldvl, const double *VR, int ldvr, double *s,
                       int mm, int *m, int *info);
int xtgevc3_ctgsna_dev(void *stream, char job, char howmny, const int *select, int n, const float *A, int lda,
                       const float *B, int ldb, const float *VL, int ldvl, const float *VR, int ldvr, float *s, int mm,
                       int *m, int *info);
/* DIF alone on the device: A, B and DIF device pointers (complex A, B interleaved, DIF
 * real), SELECT / M / INFO on the host; the checks of xTGSNA with JOB = 'V' (-2 HOWMNY, -4 N,
 * -6 LDA, -8 LDB, -15 MM).  Returns 0, or 1 when a CUDA call failed (INFO = 1).           */
int xtgevc3_dtgsna_dif_dev(void *stream, char howmny, const int *select, int n, const double *A, int lda,
                           const double *B, int ldb, double *dif, int mm, int *m, int *info);
int xtgevc3_stgsna_dif_dev(void *stream, char howmny, const int *select, int n, const float *A, int lda,
                           const float *B, int ldb, float *dif, int mm, int *m, int *info);
int xtgevc3_ztgsna_dif_dev(void *stream, char howmny, const int *select, int n, const double *A, int lda,
                           const double *B, int ldb, double *dif, int mm, int *m, int *info);
int xtgevc3_ctgsna_dif_dev(void *stream, char howmny, const int *select, int n, const float *A, int lda,
                           const float *B, int ldb, float *dif, int mm, int *m, int *info);

/* ---- eigenvalue reordering, complex pencils: xTGEXC (no counterpart upstream) ---------
 * Moves the eigenvalue at row ifst of the complex generalized Schur pencil (A, B) (upper
 * triangular) to row ilst by swaps of adjacent diagonal entries, each an equivalence
 * transformation by two rotations, and applies them to Q (wantq != 0) and Z (wantz != 0):
 * LAPACK ZTGEXC / CTGEXC's arguments (Fortran references become values for inputs), INFO
 * codes and results.  ifst, *ilst are 1-based.  On return *ilst is the eigenvalue's row;
 * INFO = 1: a swap failed the stability tests, the pencil is reordered up to it and *ilst
 * is the first row of that swap (as in LAPACK); INFO = -3 N, -5 LDA, -7 LDB, -9 LDQ,
 * -11 LDZ, -12 IFST, -13 ILST.  Complex arrays interleaved.  Device forms: A, B, Q, Z
 * device pointers, the call returns once the reordering is done (0, or 1 when a CUDA call
 * failed).  Real pencils: the D/STGEXC entry points below. */
void xtgevc3_ztgexc(int wantq, int wantz, int n, double *A, int lda, double *B, int ldb, double *Q, int ldq, double *Z,
                    int ldz, int ifst, int *ilst, int *info);
void xtgevc3_ctgexc(int wantq, int wantz, int n, float *A, int lda, float *B, int ldb, float *Q, int ldq, float *Z,
                    int ldz, int ifst, int *ilst, int *info);
int xtgevc3_ztgexc_dev(void *stream, int wantq, int wantz, int n, double *A, int lda, double *B, int ldb, double *Q,
                       int ldq, double *Z, int ldz, int ifst, int *ilst, int *info);
int xtgevc3_ctgexc_dev(void *stream, int wantq, int wantz, int n, float *A, int lda, float *B, int ldb, float *Q,
                       int ldq, float *Z, int ldz, int ifst, int *ilst, int *info);

/* ---- eigenvalue reordering, real pencils: D/STGEXC (no counterpart upstream) --------------
 * LAPACK DTGEXC / STGEXC's arguments, INFO codes and results (Fortran references become
 * pointers for in/out arguments, values for inputs): the diagonal block (1x1, or 2x2 for a
 * complex pair) at row *ifst of the real generalized Schur pencil (A quasi-upper
 * triangular, B upper triangular) moves to row *ilst by swaps of adjacent diagonal blocks
 * (LAPACK D/STGEX2: two rotations for two 1x1 blocks, otherwise the direct swapping method
 * through a small generalized Sylvester equation, with each new 2x2 block standardised).
 * As in LAPACK, *ifst and *ilst move to the first row of their 2x2 blocks, *ilst is
 * adjusted for the block sizes and returns the block's row; INFO = 1 (a swap failed the
 * stability tests; the pencil is reordered up to it and *ilst is where the block is).  Q
 * and Z agree with LAPACK's to rounding for swaps of 1x1 blocks; a swap involving a 2x2
 * block has a choice between two re-triangularisations that LAPACK decides on rounding
 * noise, so there the columns of Q and Z (and the rows and columns of A and B) agree with
 * LAPACK's up to sign.  Other codes and the device forms as for the complex entry points
 * above. */
void xtgevc3_dtgexc(int wantq, int wantz, int n, double *A, int lda, double *B, int ldb, double *Q, int ldq, double *Z,
                    int ldz, int *ifst, int *ilst, int *info);
void xtgevc3_stgexc(int wantq, int wantz, int n, float *A, int lda, float *B, int ldb, float *Q, int ldq, float *Z,
                    int ldz, int *ifst, int *ilst, int *info);
int xtgevc3_dtgexc_dev(void *stream, int wantq, int wantz, int n, double *A, int lda, double *B, int ldb, double *Q,
                       int ldq, double *Z, int ldz, int *ifst, int *ilst, int *info);
int xtgevc3_stgexc_dev(void *stream, int wantq, int wantz, int n, float *A, int lda, float *B, int ldb, float *Q,
                       int ldq, float *Z, int ldz, int *ifst, int *ilst, int *info);

/* ---- generalized Schur form: Z/C/D/SGGES without ordering (no counterpart upstream, which
 * assumes this step done) ------------------------------------------------------------------
 * A = VSL S VSR^H, B = VSL T VSR^H with VSL, VSR unitary, S, T upper triangular (overwriting
 * A, B) and T's diagonal real and non-negative; alpha = diag(S), beta = diag(T) (the
 * eigenvalues alpha / beta).  LAPACK ZGGES's arguments without ordering (SORT = 'N': no
 * SELCTG, SDIM) and without workspace: JOBVSL / JOBVSR 'V' or 'N'; INFO as LAPACK numbers its
 * arguments (-1 JOBVSL, -2 JOBVSR, -5 N, -7 LDA, -9 LDB, -14 LDVSL, -16 LDVSR), or i > 0 when
 * the QZ iterations did not deflate eigenvalue i within 30 n iterations (S, T not in Schur
 * form then).  A (B) whose largest entry in modulus lies outside [sqrt(safmin) / eps, its
 * inverse] is scaled into that range first and the form and eigenvalues scaled back at the end,
 * as LAPACK's xGGES does (xLASCL's factors; real pencils with DGGES's guard of complex pairs);
 * then the pencil is balanced by permutations (xGGBAL with JOB = 'P': isolated eigenvalues
 * moved to the ends) and VSL / VSR permuted back (xGGBAK), as xGGES does.  One CTA runs the chain of rotations (B triangular, Hessenberg-
 * triangular reduction, single-shift QZ), so the call is latency-bound; its value is the
 * result staying on the device for the eigenvector solve (xtgevc3_ztgevc3_dev).  Complex
 * arrays interleaved.  Device form: every array a device pointer (alpha, beta n complex
 * values each), the call returns once the form is computed (0, or 1 when a CUDA call
 * failed).                                                                                 */
void xtgevc3_zgges(char jobvsl, char jobvsr, int n, double *A, int lda, double *B, int ldb, double *alpha,
                   double *beta, double *VSL, int ldvsl, double *VSR, int ldvsr, int *info);
void xtgevc3_cgges(char jobvsl, char jobvsr, int n, float *A, int lda, float *B, int ldb, float *alpha, float *beta,
                   float *VSL, int ldvsl, float *VSR, int ldvsr, int *info);
int xtgevc3_zgges_dev(void *stream, char jobvsl, char jobvsr, int n, double *A, int lda, double *B, int ldb,
                      double *alpha, double *beta, double *VSL, int ldvsl, double *VSR, int ldvsr, int *info);
int xtgevc3_cgges_dev(void *stream, char jobvsl, char jobvsr, int n, float *A, int lda, float *B, int ldb, float *alpha,
                      float *beta, float *VSL, int ldvsl, float *VSR, int ldvsr, int *info);
/* Real pencils: D/SGGES without ordering, the generalized real Schur form (S upper
 * quasi-triangular, 2x2 blocks for complex pairs facing diagonal blocks of T with positive
 * entries, T's diagonal non-negative) and alphar, alphai, beta as LAPACK's DHGEQZ returns them
 * (a pair: per-row alphar, alphai with alphai(j) > 0 > alphai(j+1), and its own betas).
 * INFO numbered by DGGES's argument list (-15 LDVSL, -17 LDVSR; the others as above).     */
void xtgevc3_dgges(char jobvsl, char jobvsr, int n, double *A, int lda, double *B, int ldb, double *alphar,
                   double *alphai, double *beta, double *VSL, int ldvsl, double *VSR, int ldvsr, int *info);
void xtgevc3_sgges(char jobvsl, char jobvsr, int n, float *A, int lda, float *B, int ldb, float *alphar, float *alphai,
                   float *beta, float *VSL, int ldvsl, float *VSR, int ldvsr, int *info);
int xtgevc3_dgges_dev(void *stream, char jobvsl, char jobvsr, int n, double *A, int lda, double *B, int ldb,
                      double *alphar, double *alphai, double *beta, double *VSL, int ldvsl, double *VSR, int ldvsr,
                      int *info);
int xtgevc3_sgges_dev(void *stream, char jobvsl, char jobvsr, int n, float *A, int lda, float *B, int ldb,
                      float *alphar, float *alphai, float *beta, float *VSL, int ldvsl, float *VSR, int ldvsr, int *info);

/* xGGES with ordering: LAPACK Z/C/D/SGGES's SORT, SELCTG and SDIM in its own positions
 * (replacing the LAPACK call `zgges_(jobvsl, jobvsr, sort, selctg, &n, A, &lda, B, &ldb, &sdim,
 * alpha, beta, VSL, &ldvsl, VSR, &ldvsr, work, &lwork, rwork, bwork, &info)` and its d/s/c
 * siblings; no workspace arguments).  SORT = 'N': as the calls above, SDIM = 0.  SORT = 'S':
 * after the QZ step SELCTG is called on the host for every eigenvalue (real: SELCTG(alphar(j),
 * alphai(j), beta(j)); complex: SELCTG(alpha(j), beta(j)), each a (re, im) pair; nonzero =
 * selected, a real complex pair counting as selected when either of its values is), the
 * pencil is reordered on the device so that the selected eigenvalues lead (xTGSEN with
 * IJOB = 0: the xTGEXC walks of the reordering entry points below, then the eigenvalues
 * recomputed from the reordered pencil, xLAG2 for real 2x2 blocks, and the rows normalised
 * as xTGSEN does), VSL / VSR updated, and SDIM = the number of selected eigenvalues after the
 * reordering (a pair counts 2).  INFO = n + 3 when a swap was rejected (the pencil partly
 * reordered), n + 2 when an eigenvalue selected after the reordering follows one that is not
 * (rounding changed a selection), both as LAPACK's xGGES; SELCTG null with SORT = 'S': INFO =
 * -4; SORT neither 'N' nor 'S': -3.  The device forms call SELCTG on the host too (reading the
 * 2-3 n eigenvalue numbers back), so SELCTG is a host function in every form.               */
typedef int (*xtgevc3_dselect3)(const double *alphar, const double *alphai, const double *beta);
typedef int (*xtgevc3_sselect3)(const float *alphar, const float *alphai, const float *beta);
typedef int (*xtgevc3_zselect2)(const double *alpha, const double *beta);
typedef int (*xtgevc3_cselect2)(const float *alpha, const float *beta);
void xtgevc3_zgges_sort(char jobvsl, char jobvsr, char sort, xtgevc3_zselect2 selctg, int n, double *A, int lda,
                        double *B, int ldb, int *sdim, double *alpha, double *beta, double *VSL, int ldvsl, double *VSR,
                        int ldvsr, int *info);
void xtgevc3_cgges_sort(char jobvsl, char jobvsr, char sort, xtgevc3_cselect2 selctg, int n, float *A, int lda,
                        float *B, int ldb, int *sdim, float *alpha, float *beta, float *VSL, int ldvsl, float *VSR,
                        int ldvsr, int *info);
int xtgevc3_zgges_sort_dev(void *stream, char jobvsl, char jobvsr, char sort, xtgevc3_zselect2 selctg, int n, double *A,
                           int lda, double *B, int ldb, int *sdim, double *alpha, double *beta, double *VSL, int ldvsl,
                           double *VSR, int ldvsr, int *info);
int xtgevc3_cgges_sort_dev(void *stream, char jobvsl, char jobvsr, char sort, xtgevc3_cselect2 selctg, int n, float *A,
                           int lda, float *B, int ldb, int *sdim, float *alpha, float *beta, float *VSL, int ldvsl,
                           float *VSR, int ldvsr, int *info);
void xtgevc3_dgges_sort(char jobvsl, char jobvsr, char sort, xtgevc3_dselect3 selctg, int n, double *A, int lda,
                        double *B, int ldb, int *sdim, double *alphar, double *alphai, double *beta, double *VSL,
                        int ldvsl, double *VSR, int ldvsr, int *info);
void xtgevc3_sgges_sort(char jobvsl, char jobvsr, char sort, xtgevc3_sselect3 selctg, int n, float *A, int lda,
                        float *B, int ldb, int *sdim, float *alphar, float *alphai, float *beta, float *VSL, int ldvsl,
                        float *VSR, int ldvsr, int *info);
int xtgevc3_dgges_sort_dev(void *stream, char jobvsl, char jobvsr, char sort, xtgevc3_dselect3 selctg, int n,
                           double *A, int lda, double *B, int ldb, int *sdim, double *alphar, double *alphai,
                           double *beta, double *VSL, int ldvsl, double *VSR, int ldvsr, int *info);
int xtgevc3_sgges_sort_dev(void *stream, char jobvsl, char jobvsr, char sort, xtgevc3_sselect3 selctg, int n, float *A,
                           int lda, float *B, int ldb, int *sdim, float *alphar, float *alphai, float *beta, float *VSL,
                           int ldvsl, float *VSR, int ldvsr, int *info);

/* LAPACK D/S/Z/CTGSEN: the eigenvalues that SELECT flags move to the leading rows of the
 * generalized Schur pencil (A, B) by the swaps of xTGEXC, Q and Z updated when WANTQ / WANTZ
 * (replacing `dtgsen_(&ijob, &wantq, &wantz, select, &n, A, &lda, B, &ldb, alphar, alphai,
 * beta, Q, &ldq, Z, &ldz, &m, &pl, &pr, dif, work, &lwork, iwork, &liwork, &info)`; no
 * workspace arguments).  IJOB 0 (reordering), 1 (PL, PR: the projection norms from xTGSYL's
 * solution of the Sylvester equation of the two diagonal blocks of the reordered pencil), 2
 * (DIF(1:2): xTGSYL's Frobenius-norm estimates of Difu and Difl), 3 (DIF(1:2): the 1-norm
 * estimates, xLACN2 driving solves with TRANS = 'N' and 'T' / 'C'), 4 (1 and 2), 5 (1 and 3).
 * pl, pr, dif may be NULL when not wanted.  M = 0 or n: PL = PR = 1, DIF = ||(A, B)||_F; a
 * rejected swap: PL = PR = DIF = 0.  Complex pencils: LAPACK's values to rounding (estimated
 * before the rows are normalised, as ZTGSEN does), except DIF(2) of IJOB 3, 5, estimated here
 * on the same operator as DTGSEN's and as IJOB 2, 4 (LAPACK ZTGSEN's value there changes with
 * the contents of its workspace).  Real pencils: DIF depends on the signs of the reordered
 * pencil's columns, which real swaps of 2x2 blocks choose on rounding-level quantities (as
 * LAPACK's), so it can differ from LAPACK's estimate where those signs differ; on the same
 * reordered pencil it is LAPACK's.  The eigenvalues of the reordered pencil as
 * xTGSEN returns them (real: xLAG2 on each 2x2 block, 1x1 blocks with B(k, k) made
 * non-negative by negating row k of A and B and column k of Q; complex: when 0 < M < n and
 * every swap was done, each row scaled so that B(k, k) is real and non-negative, Q's columns
 * with it; otherwise the input diagonals).  M = the dimension of the selected subspace (a real
 * 2x2 block counts 2 when either of its rows is selected).  INFO: -1 IJOB, -5 N, -7 LDA, -9 LDB,
 * -14 / -13 LDQ, -16 / -15 LDZ (real / complex); 1 when a swap was rejected (the pencil partly
 * reordered; real pencils still get the recomputed eigenvalues); n + 1 (not a LAPACK value)
 * when a CUDA call failed in the host-pointer form.  SELECT is a host array in both forms; the
 * device form's other arrays are device pointers (returns 0, or 1 when a CUDA call failed).  */
void xtgevc3_dtgsen(int ijob, int wantq, int wantz, const int *select, int n, double *A, int lda, double *B, int ldb,
                    double *alphar, double *alphai, double *beta, double *Q, int ldq, double *Z, int ldz, int *m,
                    double *pl, double *pr, double *dif, int *info);
void xtgevc3_stgsen(int ijob, int wantq, int wantz, const int *select, int n, float *A, int lda, float *B, int ldb,
                    float *alphar, float *alphai, float *beta, float *Q, int ldq, float *Z, int ldz, int *m, float *pl,
                    float *pr, float *dif, int *info);
void xtgevc3_ztgsen(int ijob, int wantq, int wantz, const int *select, int n, double *A, int lda, double *B, int ldb,
                    double *alpha, double *beta, double *Q, int ldq, double *Z, int ldz, int *m, double *pl,
                    double *pr, double *dif, int *info);
void xtgevc3_ctgsen(int ijob, int wantq, int wantz, const int *select, int n, float *A, int lda, float *B, int ldb,
                    float *alpha, float *beta, float *Q, int ldq, float *Z, int ldz, int *m, float *pl, float *pr,
                    float *dif, int *info);
int xtgevc3_dtgsen_dev(void *stream, int ijob, int wantq, int wantz, const int *select, int n, double *A, int lda,
                       double *B, int ldb, double *alphar, double *alphai, double *beta, double *Q, int ldq, double *Z,
                       int ldz, int *m, double *pl, double *pr, double *dif, int *info);
int xtgevc3_stgsen_dev(void *stream, int ijob, int wantq, int wantz, const int *select, int n, float *A, int lda,
                       float *B, int ldb, float *alphar, float *alphai, float *beta, float *Q, int ldq, float *Z,
                       int ldz, int *m, float *pl, float *pr, float *dif, int *info);
int xtgevc3_ztgsen_dev(void *stream, int ijob, int wantq, int wantz, const int *select, int n, double *A, int lda,
                       double *B, int ldb, double *alpha, double *beta, double *Q, int ldq, double *Z, int ldz, int *m,
                       double *pl, double *pr, double *dif, int *info);
int xtgevc3_ctgsen_dev(void *stream, int ijob, int wantq, int wantz, const int *select, int n, float *A, int lda,
                       float *B, int ldb, float *alpha, float *beta, float *Q, int ldq, float *Z, int ldz, int *m,
                       float *pl, float *pr, float *dif, int *info);

/* LAPACK D/S/Z/CTGSYL: the generalized Sylvester equation A R - L B = scale C, D R - L E =
 * scale F (TRANS = 'N'), or A^T R + D^T L = scale C, R B^T + L E^T = -scale F (TRANS = 'T', real;
 * 'C' with ^H, complex) of two generalized Schur pencils (A, D) m x m, (B, E) n x n; C, F
 * (m x n) overwritten by R, L (replacing `dtgsyl_(&trans, &ijob, &m, &n, A, &lda, B, &ldb, C,
 * &ldc, D, &ldd, E, &lde, F, &ldf, &scale, &dif, work, &lwork, iwork, &info)`; no workspace).
 * IJOB 0 solves, 1 solves and estimates DIF, 3 only estimates DIF (xLATDF's look-ahead, the
 * Frobenius-norm estimate; C, F zeroed), in xTGSYL's blocked order so that the solution and
 * the estimate are LAPACK's to rounding; the transposed solves ignore IJOB, as LAPACK's.  The
 * xGECON-based IJOB 2, 4 (INFO = -2) are not built.  Complex arrays interleaved.  INFO: -1 .. -16 as LAPACK numbers its arguments (M, N >= 1), >
 * 0 when a pivot of a small system was raised (the solution then perturbed, as LAPACK's),
 * m + n + 1 (not a LAPACK value) when a CUDA call failed in the host-pointer form.  One CTA;
 * device form: every array a device pointer, scale and dif host pointers.                    */
void xtgevc3_dtgsyl(char trans, int ijob, int m, int n, const double *A, int lda, const double *B, int ldb, double *C,
                    int ldc, const double *D, int ldd, const double *E, int lde, double *F, int ldf, double *scale,
                    double *dif, int *info);
void xtgevc3_stgsyl(char trans, int ijob, int m, int n, const float *A, int lda, const float *B, int ldb, float *C,
                    int ldc, const float *D, int ldd, const float *E, int lde, float *F, int ldf, float *scale,
                    float *dif, int *info);
int xtgevc3_dtgsyl_dev(void *stream, char trans, int ijob, int m, int n, const double *A, int lda, const double *B,
                       int ldb, double *C, int ldc, const double *D, int ldd, const double *E, int lde, double *F,
                       int ldf, double *scale, double *dif, int *info);
int xtgevc3_stgsyl_dev(void *stream, char trans, int ijob, int m, int n, const float *A, int lda, const float *B,
                       int ldb, float *C, int ldc, const float *D, int ldd, const float *E, int lde, float *F, int ldf,
                       float *scale, float *dif, int *info);
void xtgevc3_ztgsyl(char trans, int ijob, int m, int n, const double *A, int lda, const double *B, int ldb, double *C,
                    int ldc, const double *D, int ldd, const double *E, int lde, double *F, int ldf, double *scale,
                    double *dif, int *info);
void xtgevc3_ctgsyl(char trans, int ijob, int m, int n, const float *A, int lda, const float *B, int ldb, float *C,
                    int ldc, const float *D, int ldd, const float *E, int lde, float *F, int ldf, float *scale,
                    float *dif, int *info);
int xtgevc3_ztgsyl_dev(void *stream, char trans, int ijob, int m, int n, const double *A, int lda, const double *B,
                       int ldb, double *C, int ldc, const double *D, int ldd, const double *E, int lde, double *F,
                       int ldf, double *scale, double *dif, int *info);
int xtgevc3_ctgsyl_dev(void *stream, char trans, int ijob, int m, int n, const float *A, int lda, const float *B,
                       int ldb, float *C, int ldc, const float *D, int ldd, const float *E, int lde, float *F, int ldf,
                       float *scale, float *dif, int *info);

/* LAPACK D/S/Z/CGGBAL and xGGBAK with JOB = 'N' or 'P' (permutation balancing, the first and
 * last steps of xGGES): xGGBAL moves isolated eigenvalues to the ends of the pencil (rows with
 * at most one nonzero in the active columns to the bottom, then columns with at most one
 * nonzero in the active rows to the left; LSCALE / RSCALE record the swaps, 1 on [ILO, IHI]),
 * xGGBAK applies the row swaps back to the vectors V (n x m; SIDE 'L' with LSCALE, 'R' with
 * RSCALE).  Equal to LAPACK's bit for bit (the search rule of older LAPACK releases, which
 * also isolates a row whose one nonzero is off the diagonal).  JOB = 'S' / 'B' (the scaling)
 * are not built: INFO = -1.  INFO as LAPACK numbers its arguments; n + 1 (not a LAPACK value)
 * when a CUDA call failed in the host-pointer form.  One CTA; device forms: matrices and
 * scales on the device, ILO / IHI host values (returns 0, or 1 when a CUDA call failed).    */
void xtgevc3_dggbal(char job, int n, double *A, int lda, double *B, int ldb, int *ilo, int *ihi, double *lscale,
                    double *rscale, int *info);
void xtgevc3_sggbal(char job, int n, float *A, int lda, float *B, int ldb, int *ilo, int *ihi, float *lscale,
                    float *rscale, int *info);
void xtgevc3_zggbal(char job, int n, double *A, int lda, double *B, int ldb, int *ilo, int *ihi, double *lscale,
                    double *rscale, int *info);
void xtgevc3_cggbal(char job, int n, float *A, int lda, float *B, int ldb, int *ilo, int *ihi, float *lscale,
                    float *rscale, int *info);
int xtgevc3_dggbal_dev(void *stream, char job, int n, double *A, int lda, double *B, int ldb, int *ilo, int *ihi,
                       double *lscale, double *rscale, int *info);
int xtgevc3_sggbal_dev(void *stream, char job, int n, float *A, int lda, float *B, int ldb, int *ilo, int *ihi,
                       float *lscale, float *rscale, int *info);
int xtgevc3_zggbal_dev(void *stream, char job, int n, double *A, int lda, double *B, int ldb, int *ilo, int *ihi,
                       double *lscale, double *rscale, int *info);
int xtgevc3_cggbal_dev(void *stream, char job, int n, float *A, int lda, float *B, int ldb, int *ilo, int *ihi,
                       float *lscale, float *rscale, int *info);
void xtgevc3_dggbak(char job, char side, int n, int ilo, int ihi, const double *lscale, const double *rscale, int m,
                    double *V, int ldv, int *info);
void xtgevc3_sggbak(char job, char side, int n, int ilo, int ihi, const float *lscale, const float *rscale, int m,
                    float *V, int ldv, int *info);
void xtgevc3_zggbak(char job, char side, int n, int ilo, int ihi, const double *lscale, const double *rscale, int m,
                    double *V, int ldv, int *info);
void xtgevc3_cggbak(char job, char side, int n, int ilo, int ihi, const float *lscale, const float *rscale, int m,
                    float *V, int ldv, int *info);
int xtgevc3_dggbak_dev(void *stream, char job, char side, int n, int ilo, int ihi, const double *lscale,
                       const double *rscale, int m, double *V, int ldv, int *info);
int xtgevc3_sggbak_dev(void *stream, char job, char side, int n, int ilo, int ihi, const float *lscale,
                       const float *rscale, int m, float *V, int ldv, int *info);
int xtgevc3_zggbak_dev(void *stream, char job, char side, int n, int ilo, int ihi, const double *lscale,
                       const double *rscale, int m, double *V, int ldv, int *info);
int xtgevc3_cggbak_dev(void *stream, char job, char side, int n, int ilo, int ihi, const float *lscale,
                       const float *rscale, int m, float *V, int ldv, int *info);

/* ---- allocation-free device entry point (no counterpart in the upstream library) -----
 * Same computation and arguments as xtgevc3_dtgevc3_dev (without flags), for callers that
 * cannot allocate device memory at this point: e.g. a framework that has reserved the
 * device memory for its own pool, or a latency-critical loop where a device allocation is
 * not acceptable.  It calls no cudaMalloc/cudaFree or other allocating routine: its scratch
 * is one 8 MiB block of device memory inside the library, held on every GPU that loads
 * the library until exit, so problems are limited to what fits (SIDE='B', HOWMNY='B':
 * n <= 478); larger ones return 2 with a message in xtgevc3_last_error(), without device
 * work.  The first call on a device looks up the block's device address (a failed lookup
 * is retried by the next call).  Every call blocks the calling thread until its result is
 * complete (it synchronises its stream), so it cannot be used inside a stream capture.
 * All calls share the block: calls whose work overlaps on the GPU race and must be
 * ordered by the caller (e.g. one stream).
 * Returns 0, 1 (CUDA failure, *info = 1) or 2 (too large).                              */
int xtgevc3_dtgevc3_dev_noalloc(void *stream, char side, char howmny, const int *select, int n, const double *S,
                                int lds, const double *P, int ldp, const double *alphar, const double *alphai,
                                const double *beta, double *VL, int ldvl, double *VR, int ldvr, int mm, int *m,
                                int *info);

/* ---- adjoint of the right eigenvectors (no counterpart in the upstream library) -------
 * Reverse-mode derivative of X = the right eigenvectors computed with SIDE='R',
 * HOWMNY='A' (in the Schur basis; for HOWMNY='B', V = Z X, pass G = Z^T dL/dV) with
 * respect to S and P, the eigenvalues held fixed:  given G = dL/dX, returns dS = dL/dS and
 * dP = dL/dP.  prec 'd', 's' (real arrays; a complex pair's two columns carry dL/dRe x and
 * dL/dIm x) or 'z', 'c' (interleaved complex; gradients are dL/dRe + i dL/dIm).  S, P, X,
 * G, dS, dP are device pointers on the current device (column-major, leading dimensions
 * >= n); alpha (alphar), alphai and beta are HOST arrays as for the device entry points
 * (alphai NULL for 'z'/'c').  X must be the forward's output for these S, P, alpha, beta:
 * its per-column scale (the overflow guards of the forward) is read back from it.  The
 * derivative includes the dependence of a complex pair's scale on the pencil norms (the
 * upstream coefficient scaling) and of its 2x2 seed on S and P.  The forward reads the
 * upper Hessenberg band (i <= j + 1) of a real S, subdiagonal zeros included, and the
 * upper triangle of P and of complex pencils; every other entry gets 0.  Work is queued on `stream` and complete on return.
 * Returns 0, -1 (bad argument) or 1 (CUDA failure); message in xtgevc3_last_error(). */
int xtgevc3_adjoint(char prec, void *stream, int n, const void *S, int lds, const void *P, int ldp,
                    const void *alpha, const void *alphai, const void *beta, const void *X, int ldx, const void *G,
                    int ldg, void *dS, int ldds, void *dP, int lddp);

/* ---- batched form (no counterpart in the upstream library) ---------------------------
 * Eigenvectors of many independent real pencils of different orders in one persistent
 * kernel launch, captured once in a CUDA graph.  One pencil: every pointer is a device
 * pointer on the current device, matrices column-major with the given leading dimensions
 * (>= n); alphar/alphai/beta are device arrays of length n.  Q and Z (HOWMNY='B') are
 * read only and the eigenvectors go to VL / VR, which must not overlap Q / Z (unlike
 * the in-place upstream interface).  Computes all eigenvectors (HOWMNY 'A' or 'B'; 'S'
 * is not offered): n columns of VL and/or VR per pencil, as the single-pencil entry
 * points would return them.  Unused pointers may be NULL. */
typedef struct xtgevc3_dpencil {
    int n, lds, ldp, ldq, ldz, ldvl, ldvr;
    const double *S, *P;
    const double *alphar, *alphai, *beta;
    const double *Q, *Z;
    double *VL, *VR;
} xtgevc3_dpencil;
typedef struct xtgevc3_spencil {
    int n, lds, ldp, ldq, ldz, ldvl, ldvr;
    const float *S, *P;
    const float *alphar, *alphai, *beta;
    const float *Q, *Z;
    float *VL, *VR;
} xtgevc3_spencil;

/* A plan binds one batch: the descriptor array (copied), the tile configuration, the
 * device workspace and the captured graph.  xtgevc3_batched_run launches the graph on
 * `stream`; run it again after writing new data into the same device buffers.  The
 * result is complete when the stream reaches the end of the launch;
 * xtgevc3_batched_wait synchronises the stream and reports the kernel's status word.
 * config: XTGEVC3_BATCH_CONFIG(nt, h) = NT columns per tile (16 or 32) and row blocks of
 * H rows (32 or 64); 0 takes the process default (set by the tuner, by
 * xtgevc3_batched_set_default, or by the environment variable XTGEVC3_BATCH_CONFIG,
 * e.g. "d:16x64,s:32x64").  The largest order a configuration accepts follows from the
 * shared memory per block (n <= 512 with every configuration on B200; larger orders are
 * refused with a message).  Returns 0, -1 (bad argument: message in
 * xtgevc3_last_error()) or 1 (CUDA failure). */
typedef struct xtgevc3_batch xtgevc3_batch;
#define XTGEVC3_BATCH_CONFIG(nt, h) (((unsigned)(nt) << 8) | (unsigned)(h))
int xtgevc3_dtgevc3_batched_create(char side, char howmny, int count, const xtgevc3_dpencil *pencils,
                                   unsigned config, xtgevc3_batch **plan);
int xtgevc3_stgevc3_batched_create(char side, char howmny, int count, const xtgevc3_spencil *pencils,
                                   unsigned config, xtgevc3_batch **plan);
int xtgevc3_batched_run(xtgevc3_batch *plan, void *stream);
/* 0 ok, 1 CUDA failure, 3 a bounded wait of the kernel's work queue expired */
int xtgevc3_batched_wait(xtgevc3_batch *plan, void *stream);
void xtgevc3_batched_destroy(xtgevc3_batch *plan);
/* the plan's tile configuration, grid size (CTAs) and units of work */
int xtgevc3_batched_info(const xtgevc3_batch *plan, unsigned *config, int *grid, int *units);
/* Tuner: times every tile configuration that fits on this batch (reps launches each, after
 * one warm-up) and returns the fastest in *best (and its time in ms in *best_ms); it
 * becomes the process default for that precision.  Returns as _create. */
int xtgevc3_dtgevc3_batched_tune(char side, char howmny, int count, const xtgevc3_dpencil *pencils, int reps,
                                 unsigned *best, float *best_ms);
int xtgevc3_stgevc3_batched_tune(char side, char howmny, int count, const xtgevc3_spencil *pencils, int reps,
                                 unsigned *best, float *best_ms);
/* prec 'd' or 's'; config 0 restores the built-in default */
void xtgevc3_batched_set_default(char prec, unsigned config);
unsigned xtgevc3_batched_get_default(char prec);

#ifdef __cplusplus
}
#endif

#endif /* XTGEVC3_H */
