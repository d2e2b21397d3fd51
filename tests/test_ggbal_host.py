"""Permutation balancing (xtgevc3_b200/csrc/ggbal.cuh: rb::ggbal_cta, LAPACK xGGBAL with
JOB = 'P'; rb::ggbak_cta, xGGBAK with JOB = 'P') compiled for the CPU by tests/qz_host.cpp,
against LAPACK's own DGGBAL / ZGGBAL / DGGBAK (their Fortran interfaces in SciPy's OpenBLAS),
bit for bit: the permuted A and B, ILO, IHI, LSCALE and RSCALE, on
pencils with isolated eigenvalues of every kind the search meets (rows with no or one
off-diagonal nonzero, columns likewise, chains of them, a fully triangular pencil, none), on 1
and several host threads."""
import ctypes as ct

import numpy as np
import pytest

import oracle
from test_qz_host import _p, host  # noqa: F401  (fixture)


def lapack_ggbal(A, B):
    cplx = np.iscomplexobj(A)
    f = getattr(oracle._openblas(), "scipy_zggbal_" if cplx else "scipy_dggbal_")
    n = A.shape[0]
    A, B = np.array(A, order="F"), np.array(B, order="F")
    ilo, ihi, info = ct.c_int(), ct.c_int(), ct.c_int()
    ls, rs, work = np.full(n, -7.0), np.full(n, -7.0), np.zeros(6 * n + 6)
    iv = lambda v: ct.byref(ct.c_int(v))  # noqa: E731
    f(ct.c_char_p(b"P"), iv(n), _p(A), iv(n), _p(B), iv(n), ct.byref(ilo), ct.byref(ihi), _p(ls), _p(rs), _p(work),
      ct.byref(info), ct.c_size_t(1))
    assert info.value == 0
    return A, B, ilo.value, ihi.value, ls, rs


def host_ggbal(L, A, B, nth=1):
    cplx = np.iscomplexobj(A)
    n = A.shape[0]
    A, B = np.array(A, order="F"), np.array(B, order="F")
    ls, rs = np.full(n, -7.0), np.full(n, -7.0)
    ilo, ihi = ct.c_int(), ct.c_int()
    (L.host_zggbal if cplx else L.host_dggbal)(nth, n, _p(A), _p(B), _p(ls), _p(rs), ct.byref(ilo), ct.byref(ihi))
    return A, B, ilo.value, ihi.value, ls, rs


def structured(kind, n, seed, cplx):
    rng = np.random.default_rng(seed)
    def draw():
        M = rng.standard_normal((n, n))
        return M + 1j * rng.standard_normal((n, n)) if cplx else M
    A, B = draw(), draw()
    if kind == "row_offdiag":  # a row with one off-diagonal nonzero
        A[2, :] = 0
        B[2, :] = 0
        A[2, 5] = 1.5
        B[2, 5] = 0.5
    elif kind == "row_zero_col":  # a zero row and a column with one nonzero
        A[4, :] = 0
        B[4, :] = 0
        A[:, 1] = 0
        B[:, 1] = 0
        A[6, 1] = 2.0
    elif kind == "chain":  # the first four columns triangular: the column search isolates them in turn
        for k in range(4):
            A[k + 1:, k] = 0
            B[k + 1:, k] = 0
    elif kind == "triangular":
        A, B = np.triu(A), np.triu(B)
    elif kind == "permuted_triangular":
        p = rng.permutation(n)
        A, B = np.triu(A)[np.ix_(p, p)], np.triu(B)[np.ix_(p, p)]
    return np.asfortranarray(A), np.asfortranarray(B)


KINDS = ["none", "row_offdiag", "row_zero_col", "chain", "triangular", "permuted_triangular"]


@pytest.mark.parametrize("cplx", [False, True], ids=["d", "z"])
@pytest.mark.parametrize("kind", KINDS, ids=str)
@pytest.mark.parametrize("n", [1, 2, 9, 17], ids=lambda n: f"n{n}")
def test_ggbal_matches_lapack(host, cplx, kind, n):
    if n < 9 and kind not in ("none", "triangular"):
        pytest.skip("the constructions need n >= 9")
    A, B = structured(kind, n, 5, cplx)
    r = lapack_ggbal(A, B)
    for nth in (1, 4):
        h = host_ggbal(host, A, B, nth)
        assert (h[2], h[3]) == (r[2], r[3]), (kind, h[2:4], r[2:4])
        assert np.array_equal(h[0], r[0]) and np.array_equal(h[1], r[1]), kind
        assert np.array_equal(h[4], r[4]) and np.array_equal(h[5], r[5]), (kind, h[4], r[4])


@pytest.mark.parametrize("kind", KINDS[1:], ids=str)
def test_ggbak_matches_lapack(host, kind):
    n = 17
    A, B = structured(kind, n, 6, False)
    r = lapack_ggbal(A, B)
    V = np.asfortranarray(np.random.default_rng(1).standard_normal((n, n)))
    for side, scale in ((b"L", r[4]), (b"R", r[5])):
        Vr = V.copy(order="F")
        iv = lambda v: ct.byref(ct.c_int(v))  # noqa: E731
        info = ct.c_int()
        oracle._openblas().scipy_dggbak_(ct.c_char_p(b"P"), ct.c_char_p(side), iv(n), iv(r[2]), iv(r[3]),
                                          _p(scale), _p(scale), iv(n), _p(Vr), iv(n), ct.byref(info), ct.c_size_t(1),
                                          ct.c_size_t(1))
        Vh = V.copy(order="F")
        host.host_dggbak(3, n, r[2], r[3], _p(np.ascontiguousarray(scale)), _p(Vh))
        assert np.array_equal(Vh, Vr), (kind, side)


@pytest.mark.parametrize("cplx", [False, True], ids=["d", "z"])
@pytest.mark.parametrize("kind", KINDS, ids=str)
def test_balanced_qz_flow_matches_lapack_gges(host, cplx, kind):
    """xGGES's flow with balancing on host threads (the bodies of the device kernels): xGGBAL
    'P', the QZ step on the whole balanced pencil, xGGBAK 'P' on Q and Z.  A = Q S Z^H and
    B = Q T Z^H to 1e-12 n, S, T in (quasi-)triangular form, and LAPACK xGGES's eigenvalues
    (relative 1e-9; the isolated ones exactly the diagonal entries LAPACK reads)."""
    from test_qz_host import host_qz, host_rqz
    import scipy.linalg.lapack as la
    n = 17
    A, B = structured(kind, n, 5, cplx)
    Ab, Bb, ilo, ihi, ls, rs = host_ggbal(host, A, B)
    if cplx:
        S, T, Q, Z, info = host_qz(host, Ab, Bb)
        lam = np.diag(S) / np.diag(T)
        r = la.zgges(lambda a, b: 0, A, B)
        lam_r = r[3] / r[4]
        bak = host.host_zggbak
    else:
        S, T, Q, Z, ar, ai, be, info = host_rqz(host, Ab, Bb)
        lam = (ar + 1j * ai) / be
        r = la.dgges(lambda x, y, z: 0, A, B)
        lam_r = (r[3] + 1j * r[4]) / r[5]
        bak = host.host_dggbak
    assert info == 0
    bak(2, n, ilo, ihi, _p(np.ascontiguousarray(ls)), _p(Q))
    bak(2, n, ilo, ihi, _p(np.ascontiguousarray(rs)), _p(Z))
    for M, M0 in ((S, A), (T, B)):
        assert np.abs(Q @ M @ Z.conj().T - M0).max() <= 1e-12 * n * np.abs(M0).max()
    assert np.abs(np.tril(T, -1)).max() == 0 and np.abs(np.tril(S, -2)).max() == 0
    fin = np.isfinite(lam_r) & np.isfinite(lam)
    for x, y in ((lam[fin], lam_r[fin]), (lam_r[fin], lam[fin])):
        d = np.abs(x[:, None] - y[None, :]).min(1) / np.maximum(np.abs(x), 1e-300)
        assert d.max() <= 1e-9, (kind, d.max())


def test_ggbal_ggbak_argument_checks():
    """xtgevc3_dggbal / dggbak: LAPACK's argument numbers, JOB = 'S' / 'B' refused (-1), all
    before any device work; JOB = 'N' and n = 0 answered on the host (ILO = 1, IHI = n)."""
    import xtgevc3_b200 as X
    L = X.lib()
    M = np.zeros((4, 4))
    v = np.zeros(4)
    ilo, ihi, info = ct.c_int(), ct.c_int(), ct.c_int()
    for job, n, lda, ldb, want in ((b"S", 4, 4, 4, -1), (b"B", 4, 4, 4, -1), (b"X", 4, 4, 4, -1), (b"P", -1, 4, 4, -2),
                                   (b"P", 4, 3, 4, -4), (b"P", 4, 4, 3, -6), (b"P", 0, 1, 1, 0)):
        L.xtgevc3_dggbal(job, n, _p(M), lda, _p(M), ldb, ct.byref(ilo), ct.byref(ihi), _p(v), _p(v), ct.byref(info))
        assert info.value == want, (job, n, info.value)
    assert (ilo.value, ihi.value) == (1, 0)
    for job, side, n, lo, hi, m, ldv, want in ((b"S", b"L", 4, 1, 4, 4, 4, -1), (b"P", b"X", 4, 1, 4, 4, 4, -2),
                                               (b"P", b"L", -1, 1, 4, 4, 4, -3), (b"P", b"L", 4, 0, 4, 4, 4, -4),
                                               (b"P", b"L", 4, 3, 2, 4, 4, -5), (b"P", b"L", 4, 1, 4, -1, 4, -8),
                                               (b"P", b"L", 4, 1, 4, 4, 3, -10), (b"N", b"R", 4, 1, 4, 4, 4, 0)):
        L.xtgevc3_dggbak(job, side, n, lo, hi, _p(v), _p(v), m, _p(M), ldv, ct.byref(info))
        assert info.value == want, (job, side, info.value)


@pytest.mark.parametrize("m", [1, 7, 30], ids=lambda m: f"m{m}")
def test_ggbak_rectangular_matches_lapack(host, m):
    """xGGBAK on n x m vectors (m other than n), both sides, against LAPACK DGGBAK."""
    n = 17
    A, B = structured("row_zero_col", n, 6, False)
    r = lapack_ggbal(A, B)
    V = np.asfortranarray(np.random.default_rng(2).standard_normal((n, m)))
    for side, scale in ((b"L", r[4]), (b"R", r[5])):
        Vr = V.copy(order="F")
        iv = lambda v: ct.byref(ct.c_int(v))  # noqa: E731
        info = ct.c_int()
        oracle._openblas().scipy_dggbak_(ct.c_char_p(b"P"), ct.c_char_p(side), iv(n), iv(r[2]), iv(r[3]), _p(scale),
                                          _p(scale), iv(m), _p(Vr), iv(n), ct.byref(info), ct.c_size_t(1),
                                          ct.c_size_t(1))
        Vh = V.copy(order="F")
        host.host_dggbak_m(4, n, m, r[2], r[3], _p(np.ascontiguousarray(scale)), _p(Vh))
        assert np.array_equal(Vh, Vr), side
