"""The complex QZ kernel's body (xtgevc3_b200/csrc/qz_cplx.cuh: rb::zgges_cta, the code the GPU
kernel runs) compiled for the CPU by tests/qz_host.cpp, on one thread and on host threads with
a std::barrier for the CTA barrier.

The form is not compared entry by entry with LAPACK ZGGES (which balances the pencil first and
runs its own QZ variant); what must hold, for random complex N(0,1) pencils and pencils with
a rank-deficient B:
  * A = Q S Z^H and B = Q T Z^H to 1e-13 n relative (single: 1e-5 n), Q and Z unitary;
  * S and T exactly upper triangular, T's diagonal real and non-negative;
  * the eigenvalues alpha / beta equal LAPACK's (SciPy) to 1e-8 relative (single: 1e-3), and a
    B of rank n - k gives exactly k zero betas (infinite eigenvalues);
  * INFO = 0;
  * the same body on 1 to 512 host threads gives the same arrays bit for bit.
Runs without a GPU."""
import ctypes as ct
import os
import shutil
import subprocess

import numpy as np
import pytest
import scipy.linalg

import xtgevc3_b200 as X
from conftest import ROOT


@pytest.fixture(scope="module")
def host():
    if shutil.which("g++") is None:
        pytest.skip("g++ not available")
    out = os.path.join(ROOT, "tests", "_build")
    os.makedirs(out, exist_ok=True)
    lib = os.path.join(out, "libqz_host.so")
    src = os.path.join(ROOT, "tests", "qz_host.cpp")
    hdrs = [os.path.join(ROOT, "xtgevc3_b200", "csrc", h)
            for h in ("qz_cplx.cuh", "qz_real.cuh", "tgsen.cuh", "tgsyl.cuh", "ggbal.cuh", "gges_scale.h",
                      "tgsna_dif_cplx.cuh", "tgsna_dif.cuh",
                      "tgexc_real_blocks.cuh")]
    if not os.path.exists(lib) or os.path.getmtime(lib) < max(os.path.getmtime(f) for f in [src] + hdrs):
        r = subprocess.run(["g++", "-O2", "-std=c++20", "-pthread", "-shared", "-fPIC", "-ffp-contract=off", "-o", lib,
                            src], capture_output=True, text=True)
        assert r.returncode == 0, r.stderr
    return ct.CDLL(lib)


def _p(a):
    return a.ctypes.data_as(ct.c_void_p)


def host_qz(L, A, B, nth=1):
    dt = A.dtype
    n = A.shape[0]
    a, b = np.asfortranarray(A).copy(order="F"), np.asfortranarray(B).copy(order="F")
    q, z = np.zeros((n, n), dtype=dt, order="F"), np.zeros((n, n), dtype=dt, order="F")
    f = L.host_zgges if dt == np.complex128 else L.host_cgges
    info = f(nth, 1, 1, n, _p(a), _p(b), _p(q), _p(z))
    return a, b, q, z, info


def pencil(n, seed, dt=np.complex128, rank_drop=0):
    r = np.random.default_rng(seed)
    A = r.standard_normal((n, n)) + 1j * r.standard_normal((n, n))
    B = r.standard_normal((n, n)) + 1j * r.standard_normal((n, n))
    if rank_drop:
        k = rank_drop
        if seed % 2 == 0 or 2 * k > n:
            B[:, :k] = 0
        else:
            B[:, :k] = B[:, k:2 * k]
    return A.astype(dt), B.astype(dt)


def check_form(A, B, S, T, Q, Z, single=False):
    """the invariants above; returns the alpha / beta pairs"""
    n = A.shape[0]
    tol = (1e-5 if single else 1e-13) * max(n, 1)
    for M, M0 in ((S, A), (T, B)):
        assert np.abs(Q @ M @ Z.conj().T - M0).max() <= tol * max(np.abs(M0).max(), 1e-300)
    for W in (Q, Z):
        assert np.abs(W.conj().T @ W - np.eye(n)).max() <= tol
    if n > 1:
        assert np.abs(np.tril(S, -1)).max() == 0 and np.abs(np.tril(T, -1)).max() == 0
    d = np.diag(T)
    assert np.all(d.imag == 0) and np.all(d.real >= 0)
    return np.diag(S), d


def eig_match(alpha, beta, A, B, single=False):
    """finite eigenvalues alpha / beta against LAPACK's, each matched to its nearest"""
    big = np.abs(B).max()
    fin = np.abs(beta) > (1e-5 if single else 1e-12) * max(big, 1)
    ev = alpha[fin] / beta[fin]
    ref = scipy.linalg.eigvals(A.astype(np.complex128), B.astype(np.complex128))
    ref = ref[np.isfinite(ref)]
    for e in ev:
        assert np.min(np.abs(ref - e)) <= (1e-3 if single else 1e-8) * max(1, abs(e)), e
    return int((~fin).sum())


@pytest.mark.parametrize("dt", [np.complex128, np.complex64], ids=["z", "c"])
def test_schur_form_of_random_pencils(host, dt):
    single = dt == np.complex64
    for n in (1, 2, 3, 5, 8, 17, 40, 64):
        for seed in range(4):
            A, B = pencil(n, 1000 * n + seed, dt)
            S, T, Q, Z, info = host_qz(host, A, B)
            assert info == 0
            alpha, beta = check_form(A, B, S, T, Q, Z, single)
            assert eig_match(alpha, beta, A, B, single) == 0


def test_infinite_eigenvalues(host):
    """B of rank n - k (zero or repeated columns): exactly k zero betas, the finite eigenvalues
    LAPACK's (the form's zero-splitting and zero-chasing steps)."""
    for n in (3, 6, 12, 30):
        for k in (1, 2, 3):
            if k >= n:
                continue
            for seed in range(4):
                A, B = pencil(n, 5000 + 100 * n + 10 * k + seed, rank_drop=k)
                S, T, Q, Z, info = host_qz(host, A, B)
                assert info == 0
                alpha, beta = check_form(A, B, S, T, Q, Z)
                assert eig_match(alpha, beta, A, B) == k, (n, k, seed)


@pytest.mark.timeout(300)
def test_kernel_body_on_host_threads(host):
    """1 to 512 threads: every thread reaches every barrier (the timeout fails a mismatch) and
    the arrays equal the one-thread run bit for bit."""
    for n, k in ((5, 0), (33, 0), (14, 2)):
        A, B = pencil(n, 77 + n, rank_drop=k)
        ref = host_qz(host, A, B, 1)
        for nth in (3, 64, 512):
            got = host_qz(host, A, B, nth)
            assert got[4] == ref[4]
            for x, y in zip(got[:4], ref[:4]):
                np.testing.assert_array_equal(x, y)


def test_gges_argument_checks():
    """xtgevc3_zgges: LAPACK ZGGES's INFO codes (numbered by its argument list), answered
    before any CUDA call, and the N = 0 quick return."""
    n = 4
    M = np.zeros((n, n), dtype=np.complex128, order="F")
    v = np.zeros(n, dtype=np.complex128)
    L = X.lib()

    def call(jl=b"V", jr=b"V", nn=n, lda=n, ldb=n, ldl=n, ldr=n):
        info = ct.c_int(99)
        L.xtgevc3_zgges(jl, jr, nn, _p(M), lda, _p(M), ldb, _p(v), _p(v), _p(M), ldl, _p(M), ldr, ct.byref(info))
        return info.value
    assert call(jl=b"X") == -1
    assert call(jr=b"X") == -2
    assert call(nn=-1) == -5
    assert call(lda=n - 1) == -7
    assert call(ldb=n - 1) == -9
    assert call(ldl=n - 1) == -14 and call(jl=b"N", ldl=0) == -14
    assert call(ldr=n - 1) == -16
    assert call(nn=0, lda=1, ldb=1, ldl=1, ldr=1) == 0
    assert call(jl=b"N", jr=b"N", nn=0, lda=1, ldb=1, ldl=1, ldr=1) == 0


# ---- real pencils (rb::dgges_cta) ------------------------------------------------------------
def host_rqz(L, A, B, nth=1):
    dt = A.dtype
    n = A.shape[0]
    a, b = np.asfortranarray(A).copy(order="F"), np.asfortranarray(B).copy(order="F")
    q, z = np.zeros((n, n), dtype=dt, order="F"), np.zeros((n, n), dtype=dt, order="F")
    ar, ai, be = (np.zeros(max(n, 1), dtype=dt) for _ in range(3))
    f = L.host_dgges if dt == np.float64 else L.host_sgges
    info = f(nth, 1, 1, n, *(_p(x) for x in (a, b, q, z, ar, ai, be)))
    return a, b, q, z, ar[:n], ai[:n], be[:n], info


def rpencil(n, seed, dt=np.float64, rank_drop=0):
    r = np.random.default_rng(seed)
    A, B = r.standard_normal((n, n)), r.standard_normal((n, n))
    if rank_drop:
        k = rank_drop
        if seed % 2 == 0 or 2 * k > n:
            B[:, :k] = 0
        else:
            B[:, :k] = B[:, k:2 * k]
    return A.astype(dt), B.astype(dt)


def check_real_form(A, B, S, T, Q, Z, ar, ai, be, single=False):
    """A = Q S Z^T, B = Q T Z^T, Q, Z orthogonal; S quasi-triangular with non-overlapping 2x2
    blocks, each facing a diagonal block of T with positive entries; T triangular with
    non-negative diagonal; a 1x1 block's (alphar, alphai, beta) = (S_kk, 0, T_kk), a pair's
    alphai of opposite signs."""
    n = A.shape[0]
    tol = (1e-5 if single else 1e-13) * max(n, 1)
    for M, M0 in ((S, A), (T, B)):
        assert np.abs(Q @ M @ Z.T - M0).max() <= tol * max(np.abs(M0).max(), 1e-300)
    for W in (Q, Z):
        assert np.abs(W.T @ W - np.eye(n)).max() <= tol
    if n > 1:
        assert np.abs(np.tril(S, -2)).max() == 0 and np.abs(np.tril(T, -1)).max() == 0
    k = 0
    while k < n:
        if k + 1 < n and S[k + 1, k] != 0:
            assert T[k, k + 1] == 0 and T[k, k] > 0 and T[k + 1, k + 1] > 0
            assert k + 2 >= n or S[k + 2, k + 1] == 0
            assert ai[k] > 0 > ai[k + 1] and be[k] > 0 and be[k + 1] > 0
            k += 2
        else:
            assert T[k, k] >= 0 and (ar[k], ai[k], be[k]) == (S[k, k], 0, T[k, k])
            k += 1


def real_eig_match(A, B, ar, ai, be, single=False):
    fin = np.abs(be) > (1e-5 if single else 1e-12) * max(np.abs(B).max(), 1)
    ev = (ar[fin] + 1j * ai[fin]) / be[fin]
    ref = scipy.linalg.eigvals(A.astype(np.float64), B.astype(np.float64))
    ref = ref[np.isfinite(ref)]
    for e in ev:
        assert np.min(np.abs(ref - e)) <= (1e-3 if single else 1e-8) * max(1, abs(e)), e
    return int((~fin).sum())


@pytest.mark.parametrize("dt", [np.float64, np.float32], ids=["d", "s"])
def test_real_schur_form_of_random_pencils(host, dt):
    single = dt == np.float32
    for n in (1, 2, 3, 4, 5, 8, 17, 40, 64):
        for seed in range(4):
            A, B = rpencil(n, 3000 * n + seed, dt)
            S, T, Q, Z, ar, ai, be, info = host_rqz(host, A, B)
            assert info == 0
            check_real_form(A, B, S, T, Q, Z, ar, ai, be, single)
            assert real_eig_match(A, B, ar, ai, be, single) == 0


def test_real_infinite_eigenvalues(host):
    for n in (3, 6, 12, 30):
        for k in (1, 2, 3):
            if k >= n:
                continue
            for seed in range(4):
                A, B = rpencil(n, 7000 + 100 * n + 10 * k + seed, rank_drop=k)
                S, T, Q, Z, ar, ai, be, info = host_rqz(host, A, B)
                assert info == 0
                check_real_form(A, B, S, T, Q, Z, ar, ai, be)
                assert real_eig_match(A, B, ar, ai, be) == k, (n, k, seed)


@pytest.mark.timeout(300)
def test_real_kernel_body_on_host_threads(host):
    for n, k in ((7, 0), (33, 0), (16, 2)):
        A, B = rpencil(n, n, rank_drop=k)
        ref = host_rqz(host, A, B, 1)
        for nth in (3, 64, 512):
            got = host_rqz(host, A, B, nth)
            for x, y in zip(got, ref):
                np.testing.assert_array_equal(x, y)


def test_real_form_feeds_the_eigenvector_solve(host):
    """The real form and its alphar / alphai / beta taken by xTGEVC3 (the oracle's C
    restatement, HOWMNY = 'B' with Q, Z): the eigenvectors of the original pencil, by their
    residuals beta A x - alpha B x and y^H (beta A - alpha B)."""
    import oracle
    n = 80
    A, B = rpencil(n, 5)
    S, T, Q, Z, ar, ai, be, info = host_rqz(host, A, B)
    VL, VR, m, info2 = oracle.tgevc3("B", "B", S, T, ar, be, alphai=ai, VL=Q.copy(order="F"), VR=Z.copy(order="F"))
    assert (info, info2, m) == (0, 0, n)
    na, nb = np.abs(A).max(), np.abs(B).max()
    k = 0
    while k < n:
        if ai[k] == 0:
            x, y, a, w = VR[:, k], VL[:, k], ar[k], 1
        else:
            x, y, a, w = VR[:, k] + 1j * VR[:, k + 1], VL[:, k] + 1j * VL[:, k + 1], ar[k] + 1j * ai[k], 2
        b = be[k]
        scale = (abs(b) * na + abs(a) * nb) * n
        assert np.abs(b * (A @ x) - a * (B @ x)).max() <= 1e-12 * scale * np.abs(x).max()
        assert np.abs(b * (y.conj() @ A) - a * (y.conj() @ B)).max() <= 1e-12 * scale * np.abs(y).max()
        k += w


def test_real_gges_argument_checks():
    """xtgevc3_dgges: DGGES's INFO numbering (ALPHAR, ALPHAI shift LDVSL / LDVSR to -15 / -17)."""
    n = 4
    M = np.zeros((n, n), order="F")
    v = np.zeros(n)
    L = X.lib()

    def call(jl=b"V", jr=b"V", nn=n, lda=n, ldb=n, ldl=n, ldr=n):
        info = ct.c_int(99)
        L.xtgevc3_dgges(jl, jr, nn, _p(M), lda, _p(M), ldb, _p(v), _p(v), _p(v), _p(M), ldl, _p(M), ldr, ct.byref(info))
        return info.value
    assert call(jl=b"X") == -1 and call(jr=b"X") == -2 and call(nn=-1) == -5
    assert call(lda=n - 1) == -7 and call(ldb=n - 1) == -9
    assert call(ldl=n - 1) == -15 and call(ldr=n - 1) == -17
    assert call(nn=0, lda=1, ldb=1, ldl=1, ldr=1) == 0
