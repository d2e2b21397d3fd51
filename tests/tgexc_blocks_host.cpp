// The real reordering kernel's arithmetic compiled for the CPU (test harness, not a product
// path): xtgevc3_b200/csrc/tgexc_real_blocks.cuh is host and device code, so the swaps and the
// walk that the GPU kernel runs can be compared with LAPACK D/STGEX2 and D/STGEXC on a machine
// without a GPU.  Built by tests/test_tgexc_blocks_host.py with g++ into a temporary folder.
#include "../xtgevc3_b200/csrc/tgexc_real_blocks.cuh"

using namespace xtg::rb;

namespace {

template <class R>
Pencil<R> pencil(int wantq, int wantz, int n, R *A, int lda, R *B, int ldb, R *Q, int ldq, R *Z, int ldz)
{
    return Pencil<R>{n, wantq, wantz, A, B, Q, Z, lda, ldb, ldq, ldz};
}

// one swap at j1 (1-based) of blocks n1 above n2: 0 done, 1 rejected (xTGEX2's INFO)
template <class R>
int swap_one(const Pencil<R> &p, int j1, int n1, int n2)
{
    Swap<R> s;
    s.j1 = j1 - 1;
    s.n1 = n1;
    s.n2 = n2;
    swap_prepare(p, s);
    if (s.ok == 1)
        for (int ph = 0; ph < 3; ph++) swap_apply(p, s, ph, 0, 1);
    return s.ok == 0 ? 1 : 0;
}

}  // namespace

extern "C" {

int host_dtgexc(int wantq, int wantz, int n, double *A, int lda, double *B, int ldb, double *Q, int ldq, double *Z,
                int ldz, int *ifst, int *ilst)
{
    return tgexc_serial(pencil(wantq, wantz, n, A, lda, B, ldb, Q, ldq, Z, ldz), *ifst, *ilst);
}

int host_stgexc(int wantq, int wantz, int n, float *A, int lda, float *B, int ldb, float *Q, int ldq, float *Z,
                int ldz, int *ifst, int *ilst)
{
    return tgexc_serial(pencil(wantq, wantz, n, A, lda, B, ldb, Q, ldq, Z, ldz), *ifst, *ilst);
}

int host_dtgex2(int wantq, int wantz, int n, double *A, int lda, double *B, int ldb, double *Q, int ldq, double *Z,
                int ldz, int j1, int n1, int n2)
{
    return swap_one(pencil(wantq, wantz, n, A, lda, B, ldb, Q, ldq, Z, ldz), j1, n1, n2);
}

int host_stgex2(int wantq, int wantz, int n, float *A, int lda, float *B, int ldb, float *Q, int ldq, float *Z,
                int ldz, int j1, int n1, int n2)
{
    return swap_one(pencil(wantq, wantz, n, A, lda, B, ldb, Q, ldq, Z, ldz), j1, n1, n2);
}

}  // extern "C"
