// Host-side driver of the device algorithm (declarations shared by engine.cu and api.cpp).
#pragma once
#include <cstdint>
#include <vector>
#include <cuda_runtime.h>
#include <functional>
#include <string>

namespace xtg {

// Options of one call (see XTGEVC3_* flags in include/xtgevc3.h).
struct Options {
    int normalize = 0;  // scale every eigenvector to max |re| + |im| = 1 (LAPACK convention)
    int simt = 0;       // force the SIMT GEMM kernels instead of the tensor-core kernel
    int split = 0;      // > 0: FP64 GEMMs (real double) as slice products with this many slices
    int split_kind = 0; // 0: BF16 slices (kind::f16), 1: INT8 slices (kind::i8), 2: INT8 residues (CRT)
    // Split forms: columns whose sketched relative residual exceeds refine_bound are solved
    // again with FP64 GEMMs (refine = 0 leaves them as they are).
    int refine = 1;
    double refine_bound = 1e-12;
    int lookahead = 0;  // trailing updates on a second stream, overlapping the next solves
    // Standard problem (xTREVC3): P is the identity and the caller passes P = nullptr.  The
    // solver builds it from scratch for the diagonal-block solves and the norms; the update
    // GEMMs skip its strips (identically zero off the diagonal).
    int p_identity = 0;
    // Real 2x2 pairs get LAPACK xTREVC3's phase: the pair's eigenvector is multiplied by the
    // unit complex number that makes its seed entry real with LAPACK's sign and ratio (one
    // entry of the 2x2 seed real, the other imaginary), before the back-transform.
    int lapack_pairs = 0;
    // When set, all device scratch of the call is carved from this buffer (nothing is
    // allocated) and the two sides run one after the other on the caller's stream.
    void *arena = nullptr;
    size_t arena_bytes = 0;
    // Real pencils on the device: read S's subdiagonal back to the host before planning the
    // row blocks (a blocking copy).  Otherwise the blocks are planned from alphai and a
    // kernel checks S against that plan; a call whose check fails is run again with this
    // set (arena mode always reads it back).
    int read_sub = 0;
    // Host-pointer path: the back-transform of a side waits for this event (the upload of
    // Z / Q on another stream), and side_done is called once a side's last kernel is
    // queued, with that side's stream (the result can be downloaded behind the other side).
    cudaEvent_t back_ready[2] = {nullptr, nullptr};  // right, left
    // Called once, with the call's stream, after every host-to-device copy of the call's own
    // (eigenvalues, column lists) is queued and before any side's kernels are: uploads that
    // only the back-transform needs start from here (an event recorded on this stream), so
    // the copy engine does not queue the small copies that start the solve behind them.
    std::function<void(cudaStream_t st)> staged;
    // Host-pointer path, real types: S and P reach the device while the call runs, column
    // panels from the right alternating with row strips from the top.  host_S (lds
    // host_lds): the caller's S, from which the subdiagonal is read instead of from the
    // device copy.  host_norms: fills {anorm, bnorm},
    // the same column sums in the same order as the device reduction (bit-identical), called
    // once after `staged`.  cols_ready(left, c, st): makes stream st wait until columns
    // [c, n) of S and P are on the device (asked by the right side before each group of row
    // blocks).  rows_ready(r, st): makes st wait until rows [0, r) of S and P are on the
    // device and returns the number of leading rows that are (>= r); the left side asks
    // before each group and transposes the rows that arrived.
    const void *host_S = nullptr;
    int host_lds = 0;
    std::function<void(double *anorm_bnorm)> host_norms;
    std::function<void(bool left, int col, cudaStream_t st)> cols_ready;
    std::function<int(int rows, cudaStream_t st)> rows_ready;
    std::function<void(bool left, cudaStream_t st)> side_done;
    // HOWMNY='B' without normalisation: the back-transform runs in column chunks and this
    // is called after each with the output columns [o0, o1) it completed.
    std::function<void(bool left, cudaStream_t st, int o0, int o1)> cols_done;
    // Host-pointer path, HOWMNY='B' without normalisation, when set: Z / Q reach the device
    // in row panels and the back-transform follows them.  back_rows_ready(left, r, st) makes
    // st wait until rows [0, r) of the side's Z / Q are on the device and returns the number
    // of leading rows that are (>= r); each panel's rows of every output column are then
    // computed (V rows = Z rows X) and rows_done(left, st, r0, r1) is called with them.
    std::function<int(bool left, int rows, cudaStream_t st)> back_rows_ready;
    std::function<void(bool left, cudaStream_t st, int r0, int r1)> rows_done;
};

// Device scratch (bytes) a call needs in arena mode: shared eigenvalue data plus the larger
// side (the sides reuse one region).  Counts each slice rounded up to 256 bytes.
size_t arena_bytes_needed(int n, int m, bool right, bool left, bool back, bool normalize, bool cplx, size_t real_size);

// One call on device-resident matrices.
//   S, P, VL, VR : device pointers, leading dimensions in elements of the scalar type
//                  (a complex number counts as one element).  VR (VL) holds Z (Q) on entry
//                  when howmny == 'B'.
//   alpha, alphai, beta, select : HOST pointers of length n.  Real: alpha = alphar (R*),
//                  alphai (R*), beta (R*).  Complex: alpha, beta interleaved, alphai unused.
//   m_total      : number of eigenvector columns (as counted by the argument check).
// Returns 0, or 1 when a CUDA call failed (message in last_error()).
template <class R, bool CPLX>
int solve_device(char side, char howmny, const int *select, int n, const void *S, int lds, const void *P,
                 int ldp, const void *alpha, const void *alphai, const void *beta, void *VL, int ldvl, void *VR,
                 int ldvr, int m_total, const Options &opt, cudaStream_t st);

// C (+)= A B (column-major FP64 device operands, M x K times K x N) through one of the
// split-precision tensor-core paths: kind 0 BF16 slices, 1 INT8 digit slices, 2 INT8 residues
// (slices = slice / modulus count).  Synchronous.  Returns 0, 1 (CUDA failure or an expired
// bounded wait; message in last_error()) or -1 (bad argument).
int split_gemm_device(int kind, int slices, int M, int N, int K, const double *A, int lda, const double *B, int ldb,
                      double *C, int ldc, int accumulate, cudaStream_t st);

// Once per device: memory-pool release threshold and the kernels' shared-memory limits.
void configure_device(int dev);

const char *last_error();
// Columns the last split-form call on this thread solved again in FP64 (0 for other calls).
int refined_columns();
void set_last_error(const std::string &s);

// Kernel trace: per kernel class, launches, CUDA-event time on the launching stream and
// algorithmic flops / bytes (the operation counts of the math, not hardware counters).
// The split forms' GEMMs are traced by part: kTSplitPrep (operand exponents and slices /
// residues), kTSplitGemm (the tensor-core kernel; flops = the FP64 product's 2MNK) and
// kTSplitCrt (reconstruction of the residue form); the rest of their update / back-transform
// work stays in kTUpdate / kTBack.
enum TraceCat { kTPrep = 0, kTDiag, kTUpdate, kTBack, kTWriteback, kTNormalize, kTSplitPrep, kTSplitGemm, kTSplitCrt,
                kTCount };
const char *trace_name(int cat);
void trace_enable(int on);
void trace_reset();
int trace_get(int cat, long long *launches, double *ms, double *flops, double *bytes);
long long launch_count();
// Adds launches made outside solve_device (the batched form's graph launches).
void count_launches(long long k);

// Eigenvalue condition numbers (LAPACK xTGSNA, JOB = 'E') of the selected eigenvalues of a
// generalized Schur pencil (A, B) from their eigenvectors VL, VR (m columns, device
// pointers): AX = A VR, BX = B VR on the tensor cores, then one warp per eigenvalue.
// items: first column of each eigenvalue; kinds: 0 real, 1 (Re, Im) pair, 2 complex;
// s_dev: device array of m condition numbers.  Returns 0, or 1 (message in last_error).
template <class R, bool CPLX>
int eig_cond_device(int n, const void *A, int lda, const void *B, int ldb, const void *VL, int ldvl, const void *VR,
                    int ldvr, int m, const std::vector<int> &items, const std::vector<uint8_t> &kinds, void *s_dev,
                    cudaStream_t st);

// Eigenvector condition estimates DIF (LAPACK D/STGSNA, JOB = 'V' / 'B') of the selected
// blocks of a real generalized Schur pencil (A, B) (device pointers): rows[i] is a block's
// first row (0-based), outs[i] the index of its DIF in dif_dev (a pair fills two), pairs[i]
// whether it is a 2x2 block.  Returns 0, or 1 (message in last_error).
template <class R>
int dif_device(int n, const R *A, int lda, const R *B, int ldb, const std::vector<int> &rows,
               const std::vector<int> &outs, const std::vector<uint8_t> &pairs, R *dif_dev, cudaStream_t st);
// The same for a complex generalized Schur pencil (A, B interleaved complex, device pointers;
// one DIF per selected eigenvalue; rows[i] its row, outs[i] its index in dif_dev).
template <class R>
int dif_device_cplx(int n, const R *A, int lda, const R *B, int ldb, const std::vector<int> &rows,
                    const std::vector<int> &outs, R *dif_dev, cudaStream_t st);

}  // namespace xtg
