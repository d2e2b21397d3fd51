"""The reordering step of xGGES with SORT = 'S' (xtgevc3_b200/csrc/tgsen.cuh: rb::tgsen_real_cta,
rb::tgsen_cplx_cta, the kernels' bodies, and rb::gges_sdim_real / _cplx, xGGES's check of the
reordered eigenvalues) compiled for the CPU by tests/qz_host.cpp, against LAPACK.

The oracle is LAPACK's own D/Z/S/CTGSEN with IJOB = 0 from SciPy's OpenBLAS, given the same
generalized Schur pencil (LAPACK xGGES of iid N(0,1) pencils, real and complex) and the same
selection; xGGES with SORT = 'S' is that call on the QZ output with SELECT = SELCTG of the QZ
eigenvalues (checked bit for bit against SciPy's xGGES in test_gges_sort_is_qz_then_tgsen).
Complex swaps apply LAPACK's rotations, so A, B, Q, Z and the eigenvalues agree to rounding;
real swaps involving 2x2 blocks agree up to the sign of each column of Q and Z (the choice
between two re-triangularisations is made on rounding-level quantities), so those are
compared after giving each column the reference's sign.  Tolerances: 1e-12 (double) / 2e-4
(single) of the matrix's largest entry; eigenvalues 1e-12 / 2e-4 relative.
"""
import ctypes as ct

import numpy as np
import pytest
import scipy.linalg.lapack as la

import oracle
from test_qz_host import _p, host, host_qz, host_rqz, pencil, rpencil  # noqa: F401  (fixture)
from test_tgexc_blocks_host import _twin_blocks_pencil, sign_aligned

TOL = {np.float64: 1e-12, np.float32: 2e-4, np.complex128: 1e-12, np.complex64: 2e-4}


def _rel(M, R):
    return float(np.abs(M - R).max() / max(np.abs(R).max(), 1e-300))


def host_tgsen(L, sel, A, B, Q, Z, nth=1):
    """rb::tgsen_*_cta on nth host threads on copies; returns (A, B, eigenvalue arrays..., Q, Z,
    info) in the order of oracle.lapack_tgsen0 (without m)."""
    dt = A.dtype.type
    n = A.shape[0]
    a, b, q, z = (np.array(M, order="F", dtype=dt) for M in (A, B, Q, Z))
    s = np.ascontiguousarray(sel, dtype=np.int32)
    if dt in (np.float64, np.float32):
        ev = [np.zeros(max(n, 1), dtype=dt) for _ in range(3)]
        f = L.host_dtgsen0 if dt == np.float64 else L.host_stgsen0
    else:
        ev = [np.zeros(max(n, 1), dtype=dt) for _ in range(2)]
        f = L.host_ztgsen0 if dt == np.complex128 else L.host_ctgsen0
    info = f(nth, 1, 1, n, _p(a), _p(b), _p(q), _p(z), _p(s), *[_p(e) for e in ev])
    return (a, b, *[e[:n] for e in ev], q, z, info)


def _real_schur(n, seed, dt):
    A, B = rpencil(n, seed, dt)
    S, T, _, ar, ai, be, Q, Z, _, info = la.dgges(lambda x, y, z: 0, A.astype(np.float64), B.astype(np.float64))
    assert info == 0
    return [np.asfortranarray(M.astype(dt)) for M in (S, T, Q, Z)] + [ar, ai, be]


REAL_SELECTIONS = {
    "neg_real": lambda ar, ai, be: ar * be < 0,
    "pairs": lambda ar, ai, be: ai != 0,
    "reals": lambda ar, ai, be: ai == 0,
    "first_of_pair": lambda ar, ai, be: ai > 0,
    "every_third": lambda ar, ai, be: np.arange(ar.size) % 3 == 2,
    "none": lambda ar, ai, be: np.zeros(ar.size, bool),
    "all": lambda ar, ai, be: np.ones(ar.size, bool),
    "last": lambda ar, ai, be: np.arange(ar.size) == ar.size - 1,
}


@pytest.mark.parametrize("dt", [np.float64, np.float32], ids=["d", "s"])
@pytest.mark.parametrize("kind", list(REAL_SELECTIONS), ids=str)
def test_real_reordering_matches_lapack(host, dt, kind):
    n = 30
    S, T, Q, Z, ar, ai, be = _real_schur(n, 11, dt)
    sel = REAL_SELECTIONS[kind](ar, ai, be).astype(np.int32)
    r = oracle.lapack_tgsen0(sel, S, T, Q, Z)
    h = host_tgsen(host, sel, S, T, Q, Z)
    assert h[-1] == r[-1] == 0
    a, b, q, z = sign_aligned(h[0], h[1], h[5], h[6], r[5], r[6])
    tol = TOL[dt]
    for M, R in ((a, r[0]), (b, r[1]), (q, r[5]), (z, r[6])):
        assert _rel(M, R) < tol * 10, kind
    # eigenvalues: the same complex numbers in the same rows, and the same betas
    lam = (h[2] + 1j * h[3]) / h[4]
    lam_r = (r[2] + 1j * r[3]) / r[4]
    assert np.abs(lam - lam_r).max() <= tol * 10 * np.abs(lam_r).max(), kind
    assert np.abs(h[4] - r[4]).max() <= tol * 10 * np.abs(r[4]).max(), kind
    # the selected eigenvalues lead
    m = r[7]
    assert m == int(sel.sum() + sum(1 for k in range(n - 1) if ai[k] > 0 and sel[k] != sel[k + 1]))
    assert np.isclose(np.sort_complex(lam[:m]), np.sort_complex(lam_r[:m]), rtol=tol * 100).all()


def _cplx_schur(n, seed, dt):
    A, B, Q, Z = oracle.complex_schur_pencil(n, seed, np.complex128)
    al, be = np.diag(A).copy(), np.diag(B).copy()
    return [np.asfortranarray(M.astype(dt)) for M in (A, B, Q, Z)] + [al.astype(dt), be.astype(dt)]


CPLX_SELECTIONS = {
    "neg_real": lambda al, be: (al * np.conj(be)).real < 0,
    "every_third": lambda al, be: np.arange(al.size) % 3 == 2,
    "none": lambda al, be: np.zeros(al.size, bool),
    "all": lambda al, be: np.ones(al.size, bool),
    "last": lambda al, be: np.arange(al.size) == al.size - 1,
    "first": lambda al, be: np.arange(al.size) == 0,
}


@pytest.mark.parametrize("dt", [np.complex128, np.complex64], ids=["z", "c"])
@pytest.mark.parametrize("kind", list(CPLX_SELECTIONS), ids=str)
def test_complex_reordering_matches_lapack(host, dt, kind):
    n = 30
    S, T, Q, Z, al, be = _cplx_schur(n, 12, dt)
    sel = CPLX_SELECTIONS[kind](al, be).astype(np.int32)
    r = oracle.lapack_tgsen0(sel, S, T, Q, Z)
    h = host_tgsen(host, sel, S, T, Q, Z)
    assert h[-1] == r[-1] == 0
    tol = TOL[dt]
    for M, R in ((h[0], r[0]), (h[1], r[1]), (h[4], r[4]), (h[5], r[5])):
        assert _rel(M, R) < tol * 10, kind
    if 0 < sel.sum() < n:  # ZTGSEN sets alpha, beta only then (otherwise its own copies)
        for v, w in ((h[2], r[2]), (h[3], r[3])):
            assert _rel(v, w) < tol * 10, kind
        assert np.all(np.diag(h[1]).imag == 0) and np.all(np.diag(h[1]).real >= 0)
    else:
        assert np.array_equal(h[2], np.diag(S)) and np.array_equal(h[3], np.diag(T))


def test_bodies_on_host_threads(host):
    """The kernels' bodies on 7 and 64 host threads (std::barrier for the CTA barrier) give the
    one-thread results bit for bit."""
    for dt, mk, sels in ((np.float64, _real_schur, REAL_SELECTIONS), (np.complex128, _cplx_schur, CPLX_SELECTIONS)):
        parts = mk(40, 13, dt)
        S, T, Q, Z = parts[:4]
        for kind in ("neg_real", "every_third", "last"):
            sel = sels[kind](*parts[4:]).astype(np.int32)
            one = host_tgsen(host, sel, S, T, Q, Z, nth=1)
            for nth in (7, 64):
                many = host_tgsen(host, sel, S, T, Q, Z, nth=nth)
                assert all(np.array_equal(x, y) for x, y in zip(one[:-1], many[:-1])), (dt, kind, nth)
                assert one[-1] == many[-1]


@pytest.mark.parametrize("sel", [[0, 0, 0, 1, 0, 0], [0, 0, 0, 0, 1, 0], [0, 0, 0, 0, 0, 1], [1, 0, 0, 1, 1, 0]],
                         ids=lambda s: "".join(map(str, s)))
def test_real_rejection_matches_lapack(host, sel):
    """Two identical 2x2 blocks: moving the second past the first is a singular Sylvester
    equation; DTGSEN stops at the rejected swap (INFO = 1) and still recomputes the
    eigenvalues of the pencil as the accepted swaps left it."""
    A, B, Q, Z = _twin_blocks_pencil(1)
    sel = np.array(sel, np.int32)
    r = oracle.lapack_tgsen0(sel, A, B, Q, Z)
    h = host_tgsen(host, sel, A, B, Q, Z)
    assert h[-1] == r[-1]
    a, b, q, z = sign_aligned(h[0], h[1], h[5], h[6], r[5], r[6])
    for M, R in ((a, r[0]), (b, r[1]), (q, r[5]), (z, r[6])):
        assert _rel(M, R) < 1e-12
    for v, w in zip(h[2:5], r[2:5]):
        assert np.abs(v - w).max() < 1e-12 * max(np.abs(w).max(), 1.0)


def test_complex_rejection_matches_lapack(host):
    """A badly scaled 3 x 3 pencil on which ZTGEXC rejects the first swap (fixture of the
    complex reordering tests): ZTGSEN returns INFO = 1 with the pencil unchanged and alpha,
    beta the diagonals of the input."""
    import os
    d = np.load(os.path.join(os.path.dirname(__file__), "golden", "tgexc", "z_rejections.npz"))
    A, B = d["A1"], d["B1"]
    I = np.eye(3, dtype=np.complex128, order="F")
    sel = np.array([0, 0, 1], np.int32)
    r = oracle.lapack_tgsen0(sel, A, B, I, I)
    h = host_tgsen(host, sel, A, B, I, I)
    assert h[-1] == r[-1] == 1
    for M, R in ((h[0], r[0]), (h[1], r[1]), (h[4], r[4]), (h[5], r[5])):
        den = np.abs(R).max(0)
        den[den == 0] = 1.0
        assert float((np.abs(M - R).max(0) / den).max()) < 1e-12
    assert np.array_equal(h[2], np.diag(A)) and np.array_equal(h[3], np.diag(B))
    assert np.array_equal(r[2], np.diag(A)) and np.array_equal(r[3], np.diag(B))


def test_gges_sort_is_qz_then_tgsen():
    """The oracle's premise: LAPACK xGGES with SORT = 'S' equals its SORT = 'N' output followed
    by xTGSEN (IJOB = 0) with SELECT = SELCTG of the QZ eigenvalues, bit for bit."""
    rng = np.random.default_rng(3)
    for n in (8, 33):
        A, B = rng.standard_normal((n, n)), rng.standard_normal((n, n))
        f = lambda ar, ai, be: ar * be < 0  # noqa: E731
        S, T, _, ar, ai, be, Q, Z, _, _ = la.dgges(lambda x, y, z: 0, A, B)
        r1 = oracle.lapack_gges_sort(A, B, f)
        r2 = oracle.lapack_tgsen0(f(ar, ai, be), S, T, Q, Z)
        assert r1[2] == r2[7] and r1[-1] == r2[-1] == 0
        for x, y in zip((r1[0], r1[1], r1[3], r1[4], r1[5], r1[6], r1[7]), (r2[0], r2[1], r2[2], r2[3], r2[4], r2[5],
                                                                         r2[6])):
            assert np.array_equal(x, y)
        Ac, Bc = A + 1j * rng.standard_normal((n, n)), B + 1j * rng.standard_normal((n, n))
        g = lambda a, b: (a * np.conj(b)).real < 0  # noqa: E731
        S, T, _, al, be, Q, Z, _, _ = la.zgges(lambda x, y: 0, Ac, Bc)
        r1 = oracle.lapack_gges_sort(Ac, Bc, g)
        r2 = oracle.lapack_tgsen0(g(al, be), S, T, Q, Z)
        assert r1[2] == r2[6] and r1[-1] == r2[-1] == 0
        for x, y in zip((r1[0], r1[1], r1[3], r1[4], r1[5], r1[6]), (r2[0], r2[1], r2[2], r2[3], r2[4], r2[5])):
            assert np.array_equal(x, y)


def _sdim(L, flags, ar, ai=None, be=None):
    n = len(flags)
    f = np.ascontiguousarray(flags, dtype=np.int32)
    info = ct.c_int(0)
    if ai is not None:
        ar, ai, be = (np.ascontiguousarray(v, dtype=np.float64) for v in (ar, ai, be))
        return L.host_dgges_sdim(n, _p(f), _p(ar), _p(ai), _p(be), ct.byref(info)), info.value
    al, be = (np.ascontiguousarray(v, dtype=np.complex128) for v in (ar, be))
    return L.host_zgges_sdim(n, _p(f), _p(al), _p(be), ct.byref(info)), info.value


def test_sdim_check_matches_lapack(host):
    """xGGES's SDIM (and INFO 0) from its check of the reordered eigenvalues, on LAPACK's own
    sorted output, with the selection that SELCTG makes there."""
    rng = np.random.default_rng(5)
    for n in (9, 40):
        A, B = rng.standard_normal((n, n)), rng.standard_normal((n, n))
        for f in REAL_SELECTIONS.values():
            if f is REAL_SELECTIONS["every_third"] or f is REAL_SELECTIONS["last"]:
                continue  # by position: not a predicate of the eigenvalue
            r = oracle.lapack_gges_sort(A, B, lambda x, y, z: bool(f(np.array([x]), np.array([y]), np.array([z]))[0]))
            ar, ai, be = r[3], r[4], r[5]
            flags = f(ar, ai, be).astype(np.int32)
            assert _sdim(host, flags, ar, ai, be) == (r[2], r[-1]) == (r[2], 0)
        Ac, Bc = A + 1j * rng.standard_normal((n, n)), B + 1j * rng.standard_normal((n, n))
        g = CPLX_SELECTIONS["neg_real"]
        r = oracle.lapack_gges_sort(Ac, Bc, lambda x, y: bool(g(np.array([x]), np.array([y]))[0]))
        flags = g(r[3], r[4]).astype(np.int32)
        assert _sdim(host, flags, r[3], None, r[4]) == (r[2], 0)


def test_sdim_check_flags_changed_selections(host):
    """INFO = n + 2 when a selected eigenvalue follows one that is not; a complex pair counts
    2 when either of its values is selected (DGGES's rule)."""
    z = np.zeros(4)
    assert _sdim(host, [1, 0, 1, 0], z + 1, z, z + 1) == (2, 6)
    assert _sdim(host, [1, 1, 0, 0], z + 1, z, z + 1) == (2, 0)
    ai = np.array([0.0, 1.0, -1.0, 0.0])
    assert _sdim(host, [1, 0, 1, 0], z + 1, ai, z + 1) == (3, 0)
    assert _sdim(host, [0, 1, 0, 0], z + 1, ai, z + 1) == (2, 6)  # the pair, after an unselected value
    assert _sdim(host, [0, 0, 1, 1], z + 1, ai, z + 1) == (3, 6)
    c = np.ones(4, dtype=np.complex128)
    assert _sdim(host, [1, 1, 0, 1], c, None, c) == (3, 6)
    assert _sdim(host, [1, 1, 1, 0], c, None, c) == (3, 0)


def _pencil(n, seed, dt):
    """iid N(0,1) pencil (complex: N(0,1) real and imaginary parts) of the xGGES tests"""
    rng = np.random.default_rng(seed)
    A, B = rng.standard_normal((n, n)), rng.standard_normal((n, n))
    if np.dtype(dt).kind == "c":
        A, B = A + 1j * rng.standard_normal((n, n)), B + 1j * rng.standard_normal((n, n))
    return A.astype(dt), B.astype(dt)


@pytest.mark.parametrize("dt", [np.float64, np.float32, np.complex128, np.complex64], ids=["d", "s", "z", "c"])
@pytest.mark.parametrize("n,seed", [(48, 31), (40, 32)], ids=["48", "40"])
def test_qz_then_reordering_on_host(host, dt, n, seed):
    """The device chain of xtgevc3_*gges_sort on the CPU (on the pencils of the GPU tests of
    xGGES with ordering): the QZ bodies, SELCTG on their eigenvalues, the reordering bodies;
    the pencil stays equivalent to (A, B), the selected eigenvalues lead, and they are the
    eigenvalues LAPACK's xGGES with SORT = 'S' puts there."""
    A, B = _pencil(n, seed, dt)
    single = dt in (np.float32, np.complex64)
    if np.dtype(dt).kind == "f":
        S, T, Q, Z, ar, ai, be, info = host_rqz(host, A, B)
        assert info == 0
        f = REAL_SELECTIONS["neg_real"]
        sel = f(ar, ai, be).astype(np.int32)
        a, b, ar2, ai2, be2, q, z, info = host_tgsen(host, sel, S, T, Q, Z)
        lam = (ar2 + 1j * ai2) / be2
        r = oracle.lapack_gges_sort(A.astype(np.float64), B.astype(np.float64), lambda x, y, w: x * w < 0)
        lam_r = (r[3] + 1j * r[4]) / r[5]
        flags = f(ar2, ai2, be2).astype(np.int32)
        sdim, info2 = _sdim(host, flags, ar2, ai2, be2)
    else:
        S, T, Q, Z, info = host_qz(host, A, B)
        assert info == 0
        g = CPLX_SELECTIONS["neg_real"]
        sel = g(np.diag(S), np.diag(T)).astype(np.int32)
        a, b, al2, be2, q, z, info = host_tgsen(host, sel, S, T, Q, Z)
        lam = al2 / be2
        r = oracle.lapack_gges_sort(A.astype(np.complex128), B.astype(np.complex128),
                                    lambda x, y: (x * np.conj(y)).real < 0)
        lam_r = r[3] / r[4]
        sdim, info2 = _sdim(host, g(al2, be2).astype(np.int32), al2.astype(np.complex128), None,
                            be2.astype(np.complex128))
    assert info == 0 and info2 == 0 and sdim == r[2] > 0
    scale = max(np.abs(A).max(), np.abs(B).max())
    tol = 2e-5 if single else 1e-12
    assert np.abs(q @ a @ z.conj().T - A).max() < tol * n * scale
    assert np.abs(q @ b @ z.conj().T - B).max() < tol * n * scale
    assert np.abs(np.tril(b, -1)).max() == 0
    assert np.abs(np.tril(a, -2)).max() == 0
    rt = 1e-3 if single else 1e-8
    assert np.allclose(np.sort_complex(lam[:sdim]), np.sort_complex(lam_r[:sdim]), rtol=rt)
    assert np.allclose(np.sort_complex(lam[sdim:]), np.sort_complex(lam_r[sdim:]), rtol=rt)


def test_gges_sort_argument_checks():
    """xtgevc3_*gges_sort's argument checks (no device work): SORT (-3), SELCTG null with
    SORT = 'S' (-4), then xGGES's own order (-5 N, -7 LDA, -9 LDB, -15 / -14 LDVSL, -17 / -16
    LDVSR)."""
    import xtgevc3_b200 as X
    L = X.lib()
    M = np.zeros((4, 4))
    v = np.zeros(8)
    sd = ct.c_int(-1)
    null3, null2 = X._SELECT["d"](), X._SELECT["z"]()
    keep = X._SELECT["d"](lambda a, b, c: 0)
    cases = [(b"V", b"V", b"X", keep, 4, 4, 4, 4, 4, -3), (b"V", b"V", b"S", null3, 4, 4, 4, 4, 4, -4),
             (b"V", b"V", b"S", keep, -1, 4, 4, 4, 4, -5), (b"V", b"V", b"S", keep, 4, 3, 4, 4, 4, -7),
             (b"V", b"V", b"S", keep, 4, 4, 3, 4, 4, -9), (b"V", b"V", b"S", keep, 4, 4, 4, 3, 4, -15),
             (b"V", b"V", b"S", keep, 4, 4, 4, 4, 3, -17), (b"Q", b"V", b"S", keep, 4, 4, 4, 4, 4, -1)]
    for jl, jr, so, sel, nn, lda, ldb, ldl, ldr, want in cases:
        info = ct.c_int(99)
        L.xtgevc3_dgges_sort(jl, jr, so, sel, nn, _p(M), lda, _p(M), ldb, ct.byref(sd), _p(v), _p(v), _p(v), _p(M), ldl,
                             _p(M), ldr, ct.byref(info))
        assert info.value == want, (so, want, info.value)
    Mc = np.zeros((4, 4), dtype=np.complex128)
    vc = np.zeros(8, dtype=np.complex128)
    keep2 = X._SELECT["z"](lambda a, b: 0)
    for so, sel, ldl, want in ((b"X", keep2, 4, -3), (b"S", null2, 4, -4), (b"S", keep2, 3, -14)):
        info = ct.c_int(99)
        L.xtgevc3_zgges_sort(b"V", b"V", so, sel, 4, _p(Mc), 4, _p(Mc), 4, ct.byref(sd), _p(vc), _p(vc), _p(Mc), ldl,
                             _p(Mc), 4, ct.byref(info))
        assert info.value == want, (so, want, info.value)


@pytest.mark.parametrize("dt", [np.float64, np.complex128], ids=["d", "z"])
@pytest.mark.parametrize("n", [1, 2, 3, 5], ids=lambda n: f"n{n}")
def test_qz_then_reordering_small_orders(host, dt, n):
    """The chain of xtgevc3_*gges_sort on orders 1 to 5 (several seeds): LAPACK's SDIM and INFO,
    the selected eigenvalues leading, A = Q S Z^H."""
    for seed in range(4):
        A, B = _pencil(n, 60 + seed, dt)
        if np.dtype(dt).kind == "f":
            S, T, Q, Z, ar, ai, be, info = host_rqz(host, A, B)
            f = REAL_SELECTIONS["neg_real"]
            sel = f(ar, ai, be).astype(np.int32)
            a, b, ar2, ai2, be2, q, z, info2 = host_tgsen(host, sel, S, T, Q, Z)
            sdim, info3 = _sdim(host, f(ar2, ai2, be2).astype(np.int32), ar2, ai2, be2)
            r = oracle.lapack_gges_sort(A, B, lambda x, y, w: x * w < 0)
        else:
            S, T, Q, Z, info = host_qz(host, A, B)
            g = CPLX_SELECTIONS["neg_real"]
            sel = g(np.diag(S), np.diag(T)).astype(np.int32)
            a, b, al2, be2, q, z, info2 = host_tgsen(host, sel, S, T, Q, Z)
            sdim, info3 = _sdim(host, g(al2, be2).astype(np.int32), al2, None, be2)
            r = oracle.lapack_gges_sort(A, B, lambda x, y: (x * np.conj(y)).real < 0)
        assert (info, info2, info3) == (0, 0, 0) and sdim == r[2], (n, seed, sdim, r[2])
        scale = max(np.abs(A).max(), np.abs(B).max())
        assert np.abs(q @ a @ z.conj().T - A).max() < 1e-12 * max(n, 2) * scale
        assert np.abs(q @ b @ z.conj().T - B).max() < 1e-12 * max(n, 2) * scale
