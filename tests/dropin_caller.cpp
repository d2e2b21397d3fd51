// A C++ caller of the drop-in interface, written the way the upstream LAPACK-comparison
// tests call the library (tests/test_lapack_d.cpp:278-284 of the upstream project): an
// LWORK = -1 query, a workspace of the size it returns, then the call -- through the
// C++-linkage prototypes of include/tgevc3.h, linked against libxtgevc3.so.
//
//   dropin_caller d|z SIDE HOWMNY n in.bin out.bin
//
// in.bin (column-major, native endianness):
//   d: S, P (n x n), alphar, alphai, beta (n), VL, VR (n x n; Q, Z for HOWMNY = 'B')
//   z: S, P (n x n complex), alpha, beta (n complex), VL, VR (n x n complex)
// out.bin: int32 {lwork query answer, m, info}, then VL, VR (n x n, same type).
#include <complex>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "tgevc3.h"

template <class T>
static bool read_all(FILE *f, std::vector<T> &v)
{
    return std::fread(v.data(), sizeof(T), v.size(), f) == v.size();
}

template <class T>
static int run(char side, char howmny, int n, FILE *in, FILE *out)
{
    const size_t nn = (size_t)n * n;
    std::vector<T> S(nn), P(nn), VL(nn), VR(nn);
    constexpr bool real = sizeof(T) == sizeof(double);
    std::vector<T> a(n), ai(real ? n : 0), b(n);
    if (!read_all(in, S) || !read_all(in, P) || !read_all(in, a) || (real && !read_all(in, ai)) ||
        !read_all(in, b) || !read_all(in, VL) || !read_all(in, VR)) {
        std::fprintf(stderr, "short input\n");
        return 2;
    }
    int m = 0, info = 0;
    T q{};
    // workspace query, as the upstream tests do
    if constexpr (real)
        dtgevc3(side, howmny, nullptr, n, S.data(), n, P.data(), n, a.data(), ai.data(), b.data(), VL.data(), n,
                VR.data(), n, n, &m, &q, -1, &info);
    else
        ztgevc3(side, howmny, nullptr, n, S.data(), n, P.data(), n, a.data(), b.data(), VL.data(), n, VR.data(), n,
                n, &m, &q, -1, &info);
    if (info != 0) {
        std::fprintf(stderr, "query info %d\n", info);
        return 3;
    }
    const int lwork = (int)std::real(q);
    std::vector<T> work(lwork);
    if constexpr (real)
        dtgevc3(side, howmny, nullptr, n, S.data(), n, P.data(), n, a.data(), ai.data(), b.data(), VL.data(), n,
                VR.data(), n, n, &m, work.data(), lwork, &info);
    else
        ztgevc3(side, howmny, nullptr, n, S.data(), n, P.data(), n, a.data(), b.data(), VL.data(), n, VR.data(), n,
                n, &m, work.data(), lwork, &info);
    const int head[3] = {lwork, m, info};
    std::fwrite(head, sizeof(int), 3, out);
    std::fwrite(VL.data(), sizeof(T), nn, out);
    std::fwrite(VR.data(), sizeof(T), nn, out);
    return 0;
}

int main(int argc, char **argv)
{
    if (argc != 7) {
        std::fprintf(stderr, "usage: %s d|z SIDE HOWMNY n in.bin out.bin\n", argv[0]);
        return 1;
    }
    const char prec = argv[1][0], side = argv[2][0], howmny = argv[3][0];
    const int n = std::atoi(argv[4]);
    FILE *in = std::fopen(argv[5], "rb");
    FILE *out = std::fopen(argv[6], "wb");
    if (!in || !out) {
        std::fprintf(stderr, "cannot open files\n");
        return 1;
    }
    const int rc = prec == 'd' ? run<double>(side, howmny, n, in, out)
                               : run<std::complex<double>>(side, howmny, n, in, out);
    std::fclose(in);
    std::fclose(out);
    return rc;
}
