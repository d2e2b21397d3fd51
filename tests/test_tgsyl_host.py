"""The generalized Sylvester solver (xtgevc3_b200/csrc/tgsyl.cuh: rb::tgsyl_cta and
rb::ztgsyl_cta, LAPACK D/S/Z/CTGSYL with TRANS = 'N') and xTGSEN's estimates on it (tgsen.cuh:
rb::tgsen_real_estimates, rb::tgsen_cplx_estimates, IJOB 1, 2, 4) compiled for the CPU by
tests/qz_host.cpp, against LAPACK.

The oracles are LAPACK's own DTGSYL (its Fortran interface in SciPy's OpenBLAS) and DTGSEN
(SciPy's wrapper), on generalized Schur pencils from LAPACK DGGES of iid N(0,1) pencils.  The
solver follows xTGSYL's blocked order, so R, L, SCALE and the DIF estimate agree with LAPACK's
to rounding (1e-12 double, 2e-4 single).  xTGSEN's PL and PR do not depend on the signs the
real 2x2 swaps leave on the reordered pencil's columns and agree to rounding too; its DIF
estimates (xLATDF's look-ahead) do, and the reordering chooses those signs on rounding-level
quantities as LAPACK does, so DIF is checked exactly on LAPACK's own reordered pencil and
within a factor of 2 on ours.  Complex swaps have no such choice: ZTGSEN's PL, PR and DIF
(estimated before the rows are normalised, as ZTGSEN does) agree with LAPACK's to rounding.
"""
import ctypes as ct

import numpy as np
import pytest
import scipy.linalg.lapack as la

import oracle
from test_qz_host import _p, host  # noqa: F401  (fixture)
from test_tgsen_host import REAL_SELECTIONS, _real_schur


def _schur(k, seed, dt=np.float64):
    g = np.random.default_rng(seed)
    S, T, *_ = la.dgges(lambda x, y, z: 0, g.standard_normal((k, k)), g.standard_normal((k, k)))
    return np.asfortranarray(S.astype(dt)), np.asfortranarray(T.astype(dt))


def host_tgsyl(L, ijob, A, B, C, D, E, F, nth=1):
    dt = A.dtype.type
    m, n = C.shape
    Cw, Fw = np.array(C, order="F"), np.array(F, order="F")
    rt = ct.c_double if dt in (np.float64, np.complex128) else ct.c_float
    sc, dif = rt(0), rt(0)
    f = {np.float64: L.host_dtgsyl, np.float32: L.host_stgsyl, np.complex128: L.host_ztgsyl,
         np.complex64: L.host_ctgsyl}[dt]
    info = f(nth, ijob, m, n, _p(A), _p(B), _p(Cw), _p(D), _p(E), _p(Fw), ct.byref(sc), ct.byref(dif))
    return Cw, Fw, sc.value, dif.value, info


SIZES = [(1, 1), (2, 2), (1, 5), (5, 1), (2, 7), (3, 4), (7, 9), (20, 13), (41, 17)]


def sylv_operands(m, n, seed, dt):
    """(A, B, C, D, E, F): (A, D), (B, E) generalized Schur pencils from LAPACK xGGES of iid
    N(0,1) pencils (complex: complex N(0,1)), C, F iid N(0,1)"""
    g = np.random.default_rng(seed + 7)
    if np.dtype(dt).kind == "c":
        A, D = (M.astype(dt) for M in oracle.complex_schur_pencil(m, seed)[:2])
        B, E = (M.astype(dt) for M in oracle.complex_schur_pencil(n, seed + 100)[:2])
        C, F = (np.asfortranarray((g.standard_normal((m, n)) + 1j * g.standard_normal((m, n))).astype(dt))
                for _ in range(2))
    else:
        A, D = _schur(m, seed, dt)
        B, E = _schur(n, seed + 100, dt)
        C, F = (np.asfortranarray(g.standard_normal((m, n)).astype(dt)) for _ in range(2))
    return A, B, C, D, E, F


@pytest.mark.parametrize("dt", [np.float64, np.float32, np.complex128, np.complex64], ids=["d", "s", "z", "c"])
@pytest.mark.parametrize("mn", SIZES, ids=lambda t: f"{t[0]}x{t[1]}")
def test_tgsyl_matches_lapack(host, dt, mn):
    m, n = mn
    tol = 1e-12 if dt in (np.float64, np.complex128) else 2e-4
    for seed in range(3):
        A, B, C, D, E, F = sylv_operands(m, n, seed, dt)
        for ijob in (0, 1, 3):
            rR, rL, rs, rd, ri = oracle.lapack_tgsyl("N", ijob, A, B, C, D, E, F)
            hR, hL, hs, hd, hi = host_tgsyl(host, ijob, A, B, C, D, E, F)
            assert (hi, hs) == (ri, rs), (ijob, hi, ri, hs, rs)
            if ijob != 3:
                for M, R in ((hR, rR), (hL, rL)):
                    assert np.abs(M - R).max() <= tol * 10 * max(np.abs(R).max(), 1.0), (ijob, seed)
            if ijob != 0:
                assert abs(hd - rd) <= tol * 10 * abs(rd), (ijob, hd, rd)


def test_tgsyl_threads_bit_for_bit(host):
    """The solvers' bodies on 5 and 64 host threads give the one-thread result bit for bit."""
    for dt in (np.float64, np.complex128):
        A, B, C, D, E, F = sylv_operands(23, 19, 1, dt)
        for ijob in (0, 1, 3):
            one = host_tgsyl(host, ijob, A, B, C, D, E, F, nth=1)
            for nth in (5, 64):
                many = host_tgsyl(host, ijob, A, B, C, D, E, F, nth=nth)
                assert np.array_equal(one[0], many[0]) and np.array_equal(one[1], many[1])
                assert one[2:] == many[2:]


def test_tgsyl_scales_against_overflow(host):
    """Right-hand sides near the overflow threshold: xGESC2 scales the solution down and SCALE <
    1 reports it, as LAPACK does (same SCALE, same solution)."""
    A, D = _schur(6, 4)
    B, E = _schur(5, 5)
    A[np.diag_indices(6)] *= 1e-6
    D[np.diag_indices(6)] *= 1e-6
    g = np.random.default_rng(6)
    C, F = (np.asfortranarray(g.standard_normal((6, 5)) * 1e305) for _ in range(2))
    rR, rL, rs, _, ri = oracle.lapack_tgsyl("N", 0, A, B, C, D, E, F)
    hR, hL, hs, _, hi = host_tgsyl(host, 0, A, B, C, D, E, F)
    assert rs < 1 and (hs, hi) == (rs, ri)
    for M, R in ((hR, rR), (hL, rL)):
        assert np.all(np.isfinite(M)) and np.abs(M - R).max() <= 1e-11 * np.abs(R).max()


def host_tgsen_full(L, ijob, sel, A, B, Q, Z, nth=1):
    dt = A.dtype.type
    n = A.shape[0]
    a, b, q, z = (np.array(M, order="F") for M in (A, B, Q, Z))
    ev = [np.zeros(max(n, 1), dtype=dt) for _ in range(3)]
    est = np.zeros(4, dtype=dt)
    m = ct.c_int(-1)
    f = L.host_dtgsen if dt == np.float64 else L.host_stgsen
    s = np.ascontiguousarray(sel, dtype=np.int32)
    info = f(nth, ijob, n, _p(a), _p(b), _p(q), _p(z), _p(s), *[_p(e) for e in ev], _p(est), ct.byref(m))
    return a, b, q, z, ev, est, m.value, info


@pytest.mark.parametrize("kind", ["neg_real", "pairs", "reals", "first_of_pair", "every_third", "none", "all"],
                         ids=str)
@pytest.mark.parametrize("n,seed", [(8, 3), (30, 11), (45, 4)], ids=["8", "30", "45"])
def test_tgsen_estimates_match_lapack(host, kind, n, seed):
    S, T, Q, Z, ar, ai, be = _real_schur(n, seed, np.float64)
    sel = REAL_SELECTIONS[kind](ar, ai, be).astype(np.int32)
    lw = n * n + 64
    for ijob in (1, 2, 4):
        r = la.dtgsen(sel, S, T, Q, Z, ijob=ijob, lwork=lw, liwork=lw)
        a, b, q, z, ev, est, m, info = host_tgsen_full(host, ijob, sel, S, T, Q, Z)
        assert (m, info) == (r[7], r[8 + 3]) == (r[7], 0)
        if ijob in (1, 4):
            assert abs(est[0] - r[8]) <= 1e-10 * r[8] and abs(est[1] - r[9]) <= 1e-10 * r[9], (est, r[8], r[9])
        if ijob in (2, 4):
            d = r[10]
            if 0 < m < n:
                assert np.all(est[2:] <= 2 * d) and np.all(est[2:] >= d / 2), (est[2:], d)
            else:  # ||(A, B)||_F, no swap involved
                assert np.allclose(est[2:], d, rtol=1e-13)
    # exact on LAPACK's own reordered pencil: DIF(1), DIF(2) from the solver there
    if 0 < sel.sum() < n:
        r0 = la.dtgsen(sel, S, T, Q, Z, ijob=0, lwork=lw, liwork=lw)
        r2 = la.dtgsen(sel, S, T, Q, Z, ijob=2, lwork=lw, liwork=lw)
        A, B, m = r0[0], r0[1], r0[7]
        z0 = np.zeros((m, n - m), order="F")
        d1 = host_tgsyl(host, 3, np.asfortranarray(A[:m, :m]), np.asfortranarray(A[m:, m:]), z0,
                        np.asfortranarray(B[:m, :m]), np.asfortranarray(B[m:, m:]), z0)[3]
        z1 = np.zeros((n - m, m), order="F")
        d2 = host_tgsyl(host, 3, np.asfortranarray(A[m:, m:]), np.asfortranarray(A[:m, :m]), z1,
                        np.asfortranarray(B[m:, m:]), np.asfortranarray(B[:m, :m]), z1)[3]
        assert abs(d1 - r2[10][0]) <= 1e-12 * r2[10][0] and abs(d2 - r2[10][1]) <= 1e-12 * r2[10][1]


def test_tgsen_estimates_rejection_and_threads(host):
    """A rejected swap gives PL = PR = DIF = 0 (INFO = 1), as LAPACK; the estimates' bodies on
    7 host threads give the one-thread result bit for bit."""
    from test_tgexc_blocks_host import _twin_blocks_pencil
    A, B, Q, Z = _twin_blocks_pencil(1)
    sel = np.array([0, 0, 0, 0, 1, 0], np.int32)
    r = la.dtgsen(sel, A, B, Q, Z, ijob=4, lwork=200, liwork=200)
    h = host_tgsen_full(host, 4, sel, A, B, Q, Z)
    assert h[7] == r[11] == 1 and np.all(h[5] == 0) and r[8] == r[9] == 0 and np.all(r[10] == 0)
    S, T, Q, Z, ar, ai, be = _real_schur(30, 11, np.float64)
    sel = REAL_SELECTIONS["neg_real"](ar, ai, be).astype(np.int32)
    one = host_tgsen_full(host, 4, sel, S, T, Q, Z, nth=1)
    many = host_tgsen_full(host, 4, sel, S, T, Q, Z, nth=7)
    for x, y in zip(one[:4] + (one[5],), many[:4] + (many[5],)):
        assert np.array_equal(x, y)


def test_tgsyl_and_tgsen_argument_checks():
    """xtgevc3_dtgsyl's checks (TRANS -1, IJOB -2, M -3, N -4, LDA -6, LDB -8, LDC -10, LDD -12,
    LDE -14, LDF -16), xtgevc3_d/ztgsen's of IJOB outside 0..5, xtgevc3_ztgsyl's TRANS ('C', not
    'T'), all before any device work."""
    import xtgevc3_b200 as X
    L = X.lib()
    M = np.zeros((4, 4))
    sc, dif = ct.c_double(0), ct.c_double(0)
    cases = [(b"C", 0, 4, 4, 4, 4, 4, 4, 4, 4, -1), (b"N", 2, 4, 4, 4, 4, 4, 4, 4, 4, -2),
             (b"N", 5, 4, 4, 4, 4, 4, 4, 4, 4, -2), (b"N", 0, 0, 4, 4, 4, 4, 4, 4, 4, -3),
             (b"N", 0, 4, 0, 4, 4, 4, 4, 4, 4, -4), (b"N", 0, 4, 4, 3, 4, 4, 4, 4, 4, -6),
             (b"N", 0, 4, 4, 4, 3, 4, 4, 4, 4, -8), (b"N", 0, 4, 4, 4, 4, 3, 4, 4, 4, -10),
             (b"N", 0, 4, 4, 4, 4, 4, 3, 4, 4, -12), (b"N", 0, 4, 4, 4, 4, 4, 4, 3, 4, -14),
             (b"N", 0, 4, 4, 4, 4, 4, 4, 4, 3, -16)]
    for tr, ijob, m, n, lda, ldb, ldc, ldd, lde, ldf, want in cases:
        info = ct.c_int(99)
        L.xtgevc3_dtgsyl(tr, ijob, m, n, _p(M), lda, _p(M), ldb, _p(M), ldc, _p(M), ldd, _p(M), lde, _p(M), ldf,
                         ct.byref(sc), ct.byref(dif), ct.byref(info))
        assert info.value == want, (tr, ijob, want, info.value)
    sel = np.zeros(4, np.int32)
    v = np.zeros(8)
    m = ct.c_int(0)
    for ijob in (-1, 6):
        info = ct.c_int(99)
        L.xtgevc3_dtgsen(ijob, 1, 1, _p(sel), 4, _p(M), 4, _p(M), 4, _p(v), _p(v), _p(v), _p(M), 4, _p(M), 4,
                         ct.byref(m), _p(v), _p(v), _p(v), ct.byref(info))
        assert info.value == -1
    Mc, vc = np.zeros((4, 4), complex), np.zeros(8, complex)
    for ijob in (-1, 6):
        info = ct.c_int(99)
        L.xtgevc3_ztgsen(ijob, 1, 1, _p(sel), 4, _p(Mc), 4, _p(Mc), 4, _p(vc), _p(vc), _p(Mc), 4, _p(Mc), 4,
                         ct.byref(m), _p(v), _p(v), _p(v), ct.byref(info))
        assert info.value == -1
    for tr, mm, want in ((b"T", 4, -1), (b"C", 0, -3), (b"N", 0, -3)):  # complex: 'C', not 'T'
        info = ct.c_int(99)
        L.xtgevc3_ztgsyl(tr, 0, mm, 4, _p(Mc), 4, _p(Mc), 4, _p(Mc), 4, _p(Mc), 4, _p(Mc), 4, _p(Mc), 4,
                         ct.byref(sc), ct.byref(dif), ct.byref(info))
        assert info.value == want, (tr, info.value)


def host_ztgsen_full(L, ijob, sel, A, B, Q, Z, nth=1):
    dt = A.dtype.type
    n = A.shape[0]
    a, b, q, z = (np.array(M, order="F") for M in (A, B, Q, Z))
    ev = [np.zeros(max(n, 1), dtype=dt) for _ in range(2)]
    est = np.zeros(4, dtype=np.float64 if dt == np.complex128 else np.float32)
    m = ct.c_int(-1)
    f = L.host_ztgsen if dt == np.complex128 else L.host_ctgsen
    s = np.ascontiguousarray(sel, dtype=np.int32)
    info = f(nth, ijob, n, _p(a), _p(b), _p(q), _p(z), _p(s), *[_p(e) for e in ev], _p(est), ct.byref(m))
    return a, b, q, z, ev, est, m.value, info


@pytest.mark.parametrize("kind", ["neg_real", "every_third", "none", "all", "last", "first"], ids=str)
@pytest.mark.parametrize("n,seed", [(8, 3), (30, 12), (45, 4)], ids=["8", "30", "45"])
def test_complex_tgsen_estimates_match_lapack(host, kind, n, seed):
    """ZTGSEN IJOB 1, 2, 4: PL, PR and DIF(1:2) within 1e-12 of LAPACK's, the pencil, Q and Z
    within 1e-11, M and INFO equal."""
    from test_tgsen_host import CPLX_SELECTIONS, _cplx_schur
    S, T, Q, Z, al, be = _cplx_schur(n, seed, np.complex128)
    sel = CPLX_SELECTIONS[kind](al, be).astype(np.int32)
    lw = 2 * n * n + 64
    for ijob in (1, 2, 4):
        r = la.ztgsen(sel, S, T, Q, Z, ijob=ijob, lwork=lw, liwork=lw)
        a, b, q, z, ev, est, m, info = host_ztgsen_full(host, ijob, sel, S, T, Q, Z)
        assert (m, info) == (r[6], r[10]) == (r[6], 0)
        want = [r[7], r[8], r[9][0], r[9][1]]
        got = [est[k] for k in range(4)]
        if ijob == 1:
            want[2:] = got[2:] = [0.0, 0.0]
        if ijob == 2:
            want[:2] = got[:2] = [0.0, 0.0]
        for g_, w_ in zip(got, want):
            assert abs(g_ - w_) <= 1e-12 * abs(w_), (ijob, got, want)
        for M, R in ((a, r[0]), (b, r[1]), (q, r[4]), (z, r[5])):
            assert np.abs(M - R).max() <= 1e-11 * max(np.abs(R).max(), 1.0)


def test_complex_tgsen_estimates_threads(host):
    from test_tgsen_host import CPLX_SELECTIONS, _cplx_schur
    S, T, Q, Z, al, be = _cplx_schur(30, 12, np.complex128)
    sel = CPLX_SELECTIONS["neg_real"](al, be).astype(np.int32)
    one = host_ztgsen_full(host, 4, sel, S, T, Q, Z, nth=1)
    many = host_ztgsen_full(host, 4, sel, S, T, Q, Z, nth=7)
    for x, y in zip(one[:4] + (one[5],), many[:4] + (many[5],)):
        assert np.array_equal(x, y)


@pytest.mark.parametrize("dt", [np.float64, np.float32], ids=["d", "s"])
@pytest.mark.parametrize("mn", SIZES, ids=lambda t: f"{t[0]}x{t[1]}")
def test_tgsyl_transposed_matches_lapack(host, dt, mn):
    """TRANS = 'T': A^T R + D^T L = scale C, R B^T + L E^T = -scale F, equal to LAPACK DTGSYL's
    within 1e-12 (double) / 2e-4 (single); 1 and 5 host threads bit for bit."""
    m, n = mn
    tol = 1e-12 if dt == np.float64 else 2e-4
    rt = ct.c_double if dt == np.float64 else ct.c_float
    f = host.host_dtgsyl_t if dt == np.float64 else host.host_stgsyl_t
    for seed in range(3):
        A, B, C, D, E, F = sylv_operands(m, n, seed, dt)
        rR, rL, rs, _, ri = oracle.lapack_tgsyl("T", 0, A, B, C, D, E, F)
        outs = []
        for nth in (1, 5):
            Cw, Fw = np.array(C, order="F"), np.array(F, order="F")
            sc = rt(0)
            info = f(nth, m, n, _p(A), _p(B), _p(Cw), _p(D), _p(E), _p(Fw), ct.byref(sc))
            assert (info, sc.value) == (ri, rs)
            for M, R in ((Cw, rR), (Fw, rL)):
                assert np.abs(M - R).max() <= tol * 10 * max(np.abs(R).max(), 1.0), seed
            outs.append((Cw, Fw))
        assert np.array_equal(outs[0][0], outs[1][0]) and np.array_equal(outs[0][1], outs[1][1])


@pytest.mark.parametrize("n,seed", [(8, 3), (30, 11), (45, 4)], ids=["8", "30", "45"])
def test_tgsen_one_norm_estimates(host, n, seed):
    """IJOB 3, 5 (xLACN2 driving solves with TRANS = 'N' and 'T'): on the same pencil as LAPACK
    (its reordered output, the leading M rows selected, so that neither side swaps) PL, PR and
    DIF(1:2) equal LAPACK's within 1e-12 for every IJOB; on the full call DIF within a factor 3
    (the column signs of the real swaps, as for the Frobenius estimates)."""
    S, T, Q, Z, ar, ai, be = _real_schur(n, seed, np.float64)
    lw = 2 * n * n + 64
    for kind, f in REAL_SELECTIONS.items():
        sel = f(ar, ai, be).astype(np.int32)
        for ijob in (3, 5):
            r = la.dtgsen(sel, S, T, Q, Z, ijob=ijob, lwork=lw, liwork=lw)
            h = host_tgsen_full(host, ijob, sel, S, T, Q, Z)
            assert (h[6], h[7]) == (r[7], r[11])
            if ijob == 5:
                assert abs(h[5][0] - r[8]) <= 1e-10 * r[8] and abs(h[5][1] - r[9]) <= 1e-10 * r[9]
            assert np.all(h[5][2:] <= 3 * r[10]) and np.all(h[5][2:] >= r[10] / 3), (kind, h[5], r[10])
        r0 = la.dtgsen(sel, S, T, Q, Z, ijob=0, lwork=lw, liwork=lw)
        m = r0[7]
        A, B, Q2, Z2 = (np.asfortranarray(x) for x in (r0[0], r0[1], r0[5], r0[6]))
        sel2 = np.zeros(n, np.int32)
        sel2[:m] = 1
        for ijob in (1, 2, 3, 4, 5):
            rr = la.dtgsen(sel2, A, B, Q2, Z2, ijob=ijob, lwork=lw, liwork=lw)
            est = host_tgsen_full(host, ijob, sel2, A, B, Q2, Z2)[5]
            ref = np.array([rr[8], rr[9], rr[10][0], rr[10][1]])
            if ijob in (2, 3):
                ref[:2] = est[:2] = 0
            if ijob == 1:
                ref[2:] = est[2:] = 0
            assert np.all(np.abs(est - ref) <= 1e-12 * np.abs(ref)), (kind, ijob, est, ref)


@pytest.mark.parametrize("dt", [np.complex128, np.complex64], ids=["z", "c"])
@pytest.mark.parametrize("mn", SIZES, ids=lambda t: f"{t[0]}x{t[1]}")
def test_complex_tgsyl_conjugate_transposed_matches_lapack(host, dt, mn):
    """TRANS = 'C': A^H R + D^H L = scale C, R B^H + L E^H = -scale F, equal to LAPACK
    Z/CTGSYL's within 1e-12 (double) / 2e-4 (single); 1 and 5 host threads bit for bit."""
    m, n = mn
    tol = 1e-12 if dt == np.complex128 else 2e-4
    rt = ct.c_double if dt == np.complex128 else ct.c_float
    f = host.host_ztgsyl_c if dt == np.complex128 else host.host_ctgsyl_c
    for seed in range(3):
        A, B, C, D, E, F = sylv_operands(m, n, seed, dt)
        rR, rL, rs, _, ri = oracle.lapack_tgsyl("C", 0, A, B, C, D, E, F)
        outs = []
        for nth in (1, 5):
            Cw, Fw = np.array(C, order="F"), np.array(F, order="F")
            sc = rt(0)
            info = f(nth, m, n, _p(A), _p(B), _p(Cw), _p(D), _p(E), _p(Fw), ct.byref(sc))
            assert (info, sc.value) == (ri, rs)
            for M, R in ((Cw, rR), (Fw, rL)):
                assert np.abs(M - R).max() <= tol * 10 * max(np.abs(R).max(), 1.0), seed
            outs.append((Cw, Fw))
        assert np.array_equal(outs[0][0], outs[1][0]) and np.array_equal(outs[0][1], outs[1][1])


def _kron_inv_one_norm(A, D, B, E):
    """||Z^-1||_1 of the Sylvester operator (R, L) -> (A R - L B, D R - L E), dense"""
    m, n = A.shape[0], B.shape[0]
    Im, In = np.eye(m), np.eye(n)
    Z = np.block([[np.kron(In, A), -np.kron(B.T, Im)], [np.kron(In, D), -np.kron(E.T, Im)]])
    return np.abs(np.linalg.inv(Z)).sum(0).max()


@pytest.mark.parametrize("kind", ["neg_real", "every_third", "none", "all", "last", "first"], ids=str)
@pytest.mark.parametrize("n,seed", [(8, 3), (12, 5), (30, 12)], ids=["8", "12", "30"])
def test_complex_tgsen_one_norm_estimates(host, kind, n, seed):
    """ZTGSEN IJOB 3, 5: PL, PR and DIF(1) (Difu) equal to LAPACK's within 1e-12.  LAPACK's own
    DIF(2) there is not reproducible (it changes with the contents of the workspace before the
    call), so DIF(2) is checked against the operator it estimates, (A22, B22 | A11, B11) of the
    reordered pencil before its normalisation (the operator of DTGSEN's Difl and of ZTGSEN's
    IJOB 2, 4): a 1-norm estimate never exceeds ||Z^-1||_1, so DIF(2) >= 1 / ||Z^-1||_1, and
    xLACN2 is exact or close on these orders (within a factor 3)."""
    from test_tgsen_host import CPLX_SELECTIONS, _cplx_schur
    S, T, Q, Z, al, be = _cplx_schur(n, seed, np.complex128)
    sel = CPLX_SELECTIONS[kind](al, be).astype(np.int32)
    lw = 2 * n * n + 64
    m = int(sel.sum())
    for ijob in (3, 5):
        r = la.ztgsen(sel, S, T, Q, Z, ijob=ijob, lwork=lw, liwork=lw)
        a, b, q, z, ev, est, mm, info = host_ztgsen_full(host, ijob, sel, S, T, Q, Z)
        assert (mm, info) == (r[6], r[10]) == (m, 0)
        if ijob == 5:
            assert abs(est[0] - r[7]) <= 1e-12 * r[7] and abs(est[1] - r[8]) <= 1e-12 * r[8]
        if m in (0, n):
            assert np.allclose(est[2:], r[9], rtol=1e-13)
            continue
        assert abs(est[2] - r[9][0]) <= 1e-12 * r[9][0], (est, r[9])
        if n <= 12:  # the dense operator of Difl on the reordered pencil (LAPACK's moves, before normalisation)
            A, B = S.copy(order="F"), T.copy(order="F")
            ks = 0
            for k in range(1, n + 1):
                if sel[k - 1]:
                    ks += 1
                    if k != ks:
                        A, B = oracle.lapack_tgexc(A, B, None, None, k, ks)[:2]
            nrm = _kron_inv_one_norm(A[m:, m:], B[m:, m:], A[:m, :m], B[:m, :m])
            assert 1 / nrm * (1 - 1e-10) <= est[3] <= 3 / nrm, (est[3], 1 / nrm)


@pytest.mark.parametrize("cplx", [False, True], ids=["d", "z"])
@pytest.mark.parametrize("n", [1, 2, 3, 4], ids=lambda n: f"n{n}")
def test_tgsen_small_orders_every_selection(host, cplx, n):
    """Orders 1 to 4, every selection pattern, IJOB 0 and 4: M, INFO, the eigenvalues and (complex
    pencils, no sign choice) PL, PR, DIF equal to LAPACK's; real PL, PR too."""
    import itertools
    from test_tgsen_host import _cplx_schur
    if cplx:
        S, T, Q, Z, al, be = _cplx_schur(n, 40 + n, np.complex128)
    else:
        S, T, Q, Z, ar, ai, be = _real_schur(n, 40 + n, np.float64)
    lw = 2 * n * n + 64
    for bits in itertools.product((0, 1), repeat=n):
        sel = np.array(bits, np.int32)
        for ijob in (0, 4):
            if cplx:
                r = la.ztgsen(sel, S, T, Q, Z, ijob=ijob, lwork=lw, liwork=lw)
                h = host_ztgsen_full(host, ijob, sel, S, T, Q, Z)
                assert (h[6], h[7]) == (r[6], r[10]), (bits, ijob)
                for v, w in zip(h[4], (r[2], r[3])):
                    assert np.abs(v[:n] - w).max() <= 1e-12 * max(np.abs(w).max(), 1.0)
                if ijob == 4:
                    ref = np.array([r[7], r[8], r[9][0], r[9][1]])
                    assert np.all(np.abs(h[5] - ref) <= 1e-12 * np.abs(ref)), (bits, h[5], ref)
            else:
                r = la.dtgsen(sel, S, T, Q, Z, ijob=ijob, lwork=lw, liwork=lw)
                h = host_tgsen_full(host, ijob, sel, S, T, Q, Z)
                assert (h[6], h[7]) == (r[7], r[11]), (bits, ijob)
                lam = (h[4][0][:n] + 1j * h[4][1][:n]) / h[4][2][:n]
                lam_r = (r[2] + 1j * r[3]) / r[4]
                assert np.abs(lam - lam_r).max() <= 1e-10 * max(np.abs(lam_r).max(), 1.0), bits
                if ijob == 4:
                    assert abs(h[5][0] - r[8]) <= 1e-12 * r[8] and abs(h[5][1] - r[9]) <= 1e-12 * r[9]
