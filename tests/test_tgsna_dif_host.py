"""DIF of the real xTGSNA kernel (xtgevc3_b200/csrc/tgsna_dif.cuh with the reordering of
tgexc_real_blocks.cuh) compiled for the CPU by tests/tgsna_dif_host.cpp and compared with
LAPACK D/STGSNA (JOB = 'V') from SciPy's OpenBLAS on real xGGES pencils.

DTGSNA's DIF is an estimate: it reorders a copy of the pencil so that the eigenvalue comes
first, then solves xTGSYL's block substitution for right-hand sides of +-1 entries chosen by
look-ahead.  Those choices follow the signs of the reordered copy, and in swaps of 2x2 blocks
LAPACK leaves the signs to rounding noise (its RQ-versus-QR choice), so:
  * the estimate step is checked exactly: on LAPACK's own reordered copy the estimate (and a
    pair's bound) must equal LAPACK's DIF to rounding (1e-12 relative);
  * whole DIFs: equal to LAPACK's (1e-12) for most eigenvalues (at least 85 %; those whose
    reordered copy has LAPACK's signs), and every estimate, ours and LAPACK's, lies between
    the true value (the smallest singular value of the Kronecker operator, by a dense SVD)
    and ten times it, ours within a factor of two of LAPACK's;
  * a rejected reordering gives DIF = 0, as in LAPACK.
Complex pencils (ZTGSNA): the reordering is LAPACK's rotations (no sign freedom), so every DIF
must equal LAPACK's to rounding (1e-12 double, 1e-4 single).
The GPU kernels' bodies themselves (written against a CTA context) also run here on host
threads with a barrier and must give the serial build's values bit for bit.
Runs without a GPU."""
import ctypes as ct
import os
import shutil
import subprocess

import numpy as np
import pytest

import oracle
from conftest import ROOT
from xtgevc3_b200 import pencils


@pytest.fixture(scope="module")
def host():
    if shutil.which("g++") is None:
        pytest.skip("g++ not available")
    out = os.path.join(ROOT, "tests", "_build")
    os.makedirs(out, exist_ok=True)
    lib = os.path.join(out, "libtgsna_dif_host.so")
    src = os.path.join(ROOT, "tests", "tgsna_dif_host.cpp")
    hdrs = [os.path.join(ROOT, "xtgevc3_b200", "csrc", h)
            for h in ("tgsna_dif.cuh", "tgsna_dif_cplx.cuh", "tgexc_real_blocks.cuh")]
    if not os.path.exists(lib) or os.path.getmtime(lib) < max(os.path.getmtime(f) for f in [src] + hdrs):
        r = subprocess.run(["g++", "-O2", "-std=c++20", "-pthread", "-shared", "-fPIC", "-ffp-contract=off", "-o", lib,
                            src], capture_output=True, text=True)
        assert r.returncode == 0, r.stderr
    L = ct.CDLL(lib)
    L.host_ddif_reordered.restype = ct.c_double
    L.host_dpair_cond.restype = ct.c_double
    return L


def _p(a):
    return a.ctypes.data_as(ct.c_void_p)


def host_dif(L, A, B, howmny="A", select=None):
    n = A.shape[0]
    pfx = "d" if A.dtype == np.float64 else "s"
    A, B = np.asfortranarray(A), np.asfortranarray(B)
    dif = np.zeros(max(n, 1), dtype=A.dtype)
    sel = np.zeros(max(n, 1), dtype=np.int32) if select is None else np.ascontiguousarray(select, dtype=np.int32)
    m = ct.c_int()
    rc = getattr(L, f"host_{pfx}dif")(ct.c_char(howmny.encode()), _p(sel), n, _p(A), n, _p(B), n, _p(dif), n,
                                      ct.byref(m))
    assert rc == 0
    return dif[:m.value]


def blocks(A):
    n, k, out = A.shape[0], 0, []
    while k < n:
        pair = k + 1 < n and A[k + 1, k] != 0
        out.append((k, pair))
        k += 2 if pair else 1
    return out


def true_dif(A, B, k):
    """smallest singular value of the Sylvester operator of the block at row k, from
    LAPACK's reordering of (A, B)"""
    r = oracle.lapack_tgexc_real(A, B, None, None, k + 1, 1)
    a, b = r[0], r[1]
    n1 = 2 if a[1, 0] != 0 else 1
    n2 = A.shape[0] - n1
    I1, I2 = np.eye(n1), np.eye(n2)
    K = np.block([[np.kron(I1, a[n1:, n1:]), -np.kron(a[:n1, :n1].T, I2)],
                  [np.kron(I1, b[n1:, n1:]), -np.kron(b[:n1, :n1].T, I2)]])
    return np.linalg.svd(K, compute_uv=False)[-1]


@pytest.mark.parametrize("n", [6, 13, 30])
def test_estimate_step_matches_lapack(host, n):
    """On LAPACK's reordered copy the estimate is LAPACK's DIF to rounding (pairs: the min
    with the pair's own bound, taken from the original block as DTGSNA does)."""
    for seed in range(6):
        S, T = pencils.gen_gges(n, 40 + seed)[:2]
        _, d, m, info = oracle.lapack_tgsna("A", S, T, None, None, job="V")
        assert info == 0 and m == n
        ks = 0
        for k, pair in blocks(S):
            r = oracle.lapack_tgexc_real(S, T, None, None, k + 1, 1)
            assert r[6] == 0
            a, b = np.asfortranarray(r[0]), np.asfortranarray(r[1])
            est = host.host_ddif_reordered(n, _p(a), _p(b))
            if pair:
                blk_a = np.asfortranarray(S[k:k + 2, k:k + 2])
                blk_b = np.asfortranarray(T[k:k + 2, k:k + 2])
                cond = host.host_dpair_cond(_p(blk_a), _p(blk_b))
                est = cond if n == 2 else min(est, cond)
            assert abs(est - d[ks]) <= 1e-12 * abs(d[ks]), (seed, k, est, d[ks])
            ks += 2 if pair else 1


@pytest.mark.parametrize("dt", [np.float64, np.float32], ids=["d", "s"])
def test_dif_matches_lapack(host, dt):
    tol = {np.float64: 1e-12, np.float32: 1e-4}[dt]
    same = total = 0
    for seed in range(8):
        for n in (7, 16, 28):
            S, T = pencils.gen_gges(n, 60 + seed + n, dtype=dt)[:2]
            _, d, m, info = oracle.lapack_tgsna("A", S, T, None, None, job="V")
            h = host_dif(host, S, T)
            assert info == 0 and len(h) == m == n
            for (k, pair), ks in zip(blocks(S), np.cumsum([0] + [2 if p else 1 for _, p in blocks(S)])[:-1]):
                total += 1
                if abs(h[ks] - d[ks]) <= tol * abs(d[ks]):
                    same += 1
                    continue
                assert 0.5 <= h[ks] / d[ks] <= 2.0, (seed, n, k, h[ks], d[ks])
                if dt == np.float64:
                    t = true_dif(S, T, k)
                    assert t * (1 - 1e-10) <= h[ks] <= 10 * t and t * (1 - 1e-10) <= d[ks] <= 10 * t
    assert same >= 0.85 * total, (same, total)


def _twin_blocks_pencil(seed, n=6):
    rng = np.random.default_rng(seed)
    A = np.triu(rng.standard_normal((n, n)))
    B = np.triu(rng.standard_normal((n, n)))
    B[np.diag_indices(n)] = np.abs(B[np.diag_indices(n)]) + 0.5
    for k in (1, 3):
        A[k:k + 2, k:k + 2] = [[0.7, 1.3], [-0.9, 0.7]]
        B[k:k + 2, k:k + 2] = np.diag([1.2, 0.8])
    return np.asfortranarray(A), np.asfortranarray(B)


def test_dif_selection_rejection_and_n1(host):
    """HOWMNY = 'S' (a pair selected by its second row fills two entries), a rejected
    reordering (the second of two identical 2x2 blocks cannot pass the first: DIF = 0) and
    n = 1 (|(a, b)|): LAPACK's values."""
    S, T = pencils.gen_gges(14, 77)[:2]
    sel = np.zeros(14, dtype=np.int32)
    pair_rows = [k for k, p in blocks(S) if p]
    sel[pair_rows[0] + 1] = 1
    sel[[k for k, p in blocks(S) if not p][:1]] = 1
    _, d, m, _ = oracle.lapack_tgsna("S", S, T, None, None, select=sel, job="V")
    h = host_dif(host, S, T, "S", sel)
    assert len(h) == m == 3
    np.testing.assert_allclose(h, d, rtol=1e-12)
    A, B = _twin_blocks_pencil(2)
    _, d, m, _ = oracle.lapack_tgsna("A", A, B, None, None, job="V")
    h = host_dif(host, A, B)
    assert d[3] == 0 and d[4] == 0  # the second twin's reordering is rejected
    np.testing.assert_array_equal(h[3:5], d[3:5])
    one_a, one_b = np.array([[3.0]], order="F"), np.array([[-4.0]], order="F")
    _, d, m, _ = oracle.lapack_tgsna("A", one_a, one_b, None, None, job="V")
    np.testing.assert_allclose(host_dif(host, one_a, one_b), d, rtol=1e-15)


def host_zdif(L, A, B, howmny="A", select=None):
    n = A.shape[0]
    pfx = "z" if A.dtype == np.complex128 else "c"
    rdt = np.float64 if pfx == "z" else np.float32
    A, B = np.asfortranarray(A), np.asfortranarray(B)
    dif = np.zeros(max(n, 1), dtype=rdt)
    sel = np.zeros(max(n, 1), dtype=np.int32) if select is None else np.ascontiguousarray(select, dtype=np.int32)
    m = ct.c_int()
    rc = getattr(L, f"host_{pfx}dif")(ct.c_char(howmny.encode()), _p(sel), n, _p(A), _p(B), _p(dif), n, ct.byref(m))
    assert rc == 0
    return dif[:m.value]


@pytest.mark.parametrize("dt", [np.complex128, np.complex64], ids=["z", "c"])
def test_complex_dif_matches_lapack(host, dt):
    """ZTGSNA / CTGSNA JOB = 'V' on complex generalized Schur forms of iid complex N(0,1)
    pencils, n = 1 .. 30, every eigenvalue; and HOWMNY = 'S'."""
    tol = {np.complex128: 1e-12, np.complex64: 1e-4}[dt]
    for seed in range(6):
        for n in (1, 2, 5, 13, 30):
            A, B = oracle.complex_schur_pencil(n, 200 + seed, dt)[:2]
            _, d, m, info = oracle.lapack_tgsna("A", A, B, None, None, job="V")
            h = host_zdif(host, A, B)
            assert info == 0 and len(h) == m == n
            np.testing.assert_allclose(h, d, rtol=tol)
    A, B = oracle.complex_schur_pencil(20, 9, dt)[:2]
    sel = np.zeros(20, dtype=np.int32)
    sel[[2, 11, 19]] = 1
    _, d, m, _ = oracle.lapack_tgsna("S", A, B, None, None, select=sel, job="V")
    np.testing.assert_allclose(host_zdif(host, A, B, "S", sel), d, rtol=tol)


def test_estimate_step_every_small_order(host):
    """The estimate step on LAPACK's reordered copies for every block of 25 pencils of each
    order n = 2 .. 12 (xTGSYL's block cuts next to 2x2 blocks, n2 = 1 .. 4, the unblocked
    case): LAPACK's DIF to 1e-12."""
    for n in range(2, 13):
        for seed in range(25):
            S, T = pencils.gen_gges(n, 5000 + 100 * n + seed)[:2]
            _, d, m, info = oracle.lapack_tgsna("A", S, T, None, None, job="V")
            ks = 0
            for k, pair in blocks(S):
                r = oracle.lapack_tgexc_real(S, T, None, None, k + 1, 1)
                if r[6] == 0:
                    a, b = np.asfortranarray(r[0]), np.asfortranarray(r[1])
                    n1 = 2 if a[1, 0] != 0 else 1
                    est = host.host_ddif_reordered(n, _p(a), _p(b)) if n > n1 else None
                    if pair:
                        cond = host.host_dpair_cond(_p(np.asfortranarray(S[k:k + 2, k:k + 2])),
                                                    _p(np.asfortranarray(T[k:k + 2, k:k + 2])))
                        est = cond if est is None else min(est, cond)
                    assert abs(est - d[ks]) <= 1e-12 * abs(d[ks]), (n, seed, k, est, d[ks])
                ks += 2 if pair else 1


@pytest.mark.parametrize("dt", [np.complex128, np.complex64], ids=["z", "c"])
def test_complex_dif_every_small_order(host, dt):
    """Every eigenvalue of 20 complex Schur pencils of each order n = 1 .. 12."""
    tol = {np.complex128: 1e-12, np.complex64: 1e-4}[dt]
    for n in range(1, 13):
        for seed in range(20):
            A, B = oracle.complex_schur_pencil(n, 7000 + 100 * n + seed, dt)[:2]
            _, d, m, info = oracle.lapack_tgsna("A", A, B, None, None, job="V")
            np.testing.assert_allclose(host_zdif(host, A, B), d, rtol=tol, err_msg=f"n={n} seed={seed}")


def _threads_dif(L, fn, nth, grid, A, B):
    n = A.shape[0]
    dif = np.zeros(max(n, 1))
    sel = np.zeros(max(n, 1), dtype=np.int32)
    m = ct.c_int()
    A, B = np.asfortranarray(A), np.asfortranarray(B)
    err = getattr(L, fn)(nth, grid, ct.c_char(b"A"), _p(sel), n, _p(A), _p(B), _p(dif), ct.byref(m))
    return dif[:m.value], err


@pytest.mark.timeout(300)
def test_kernel_bodies_on_host_threads(host):
    """The DIF kernels' bodies (rb::dif_cta, rb::zdif_cta: the code the GPU kernels run) on host
    threads, one std::thread per GPU thread and a std::barrier for the CTA barrier, several
    CTAs: every thread reaches every barrier (a mismatch would hang: the timeout fails it), and
    the DIFs equal the serial build's bit for bit whatever the thread and CTA counts (each
    entry is updated by one thread with the same arithmetic)."""
    for seed, n in ((1, 1), (2, 2), (3, 9), (4, 24), (5, 37)):
        S, T = pencils.gen_gges(n, 60 + seed)[:2]
        ref = host_dif(host, S, T)
        for nth, grid in ((1, 1), (3, 2), (32, 5), (256, 3)):
            h, err = _threads_dif(host, "threads_ddif", nth, grid, S, T)
            assert err == 0
            np.testing.assert_array_equal(h, ref, err_msg=f"real n={n} threads={nth} ctas={grid}")
        A, B = oracle.complex_schur_pencil(n, 80 + seed)[:2]
        zref = host_zdif(host, A, B)
        for nth, grid in ((1, 1), (5, 2), (64, 4)):
            h, _ = _threads_dif(host, "threads_zdif", nth, grid, A, B)
            np.testing.assert_array_equal(h, zref, err_msg=f"complex n={n} threads={nth} ctas={grid}")
