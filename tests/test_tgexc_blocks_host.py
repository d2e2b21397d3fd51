"""The real reordering kernel's arithmetic (xtgevc3_b200/csrc/tgexc_real_blocks.cuh: the swaps
of 1x1 and 2x2 diagonal blocks and the walk of a block from IFST to ILST) compiled for the CPU
by tests/tgexc_blocks_host.cpp and compared with LAPACK D/STGEX2 and D/STGEXC from SciPy's
OpenBLAS on real generalized Schur pencils (LAPACK xGGES of iid N(0,1) pencils).

What must agree:
  * INFO and, for whole moves, IFST and ILST on exit: exactly;
  * swaps of two 1x1 blocks: A, B, Q, Z to rounding (the same two rotations as LAPACK);
  * swaps involving a 2x2 block: A, B, Q, Z to rounding up to the sign of each column of Q
    and Z (and the matching rows and columns of A and B).  LAPACK re-triangularises the
    swapped pencil both by an RQ and by a QR factorisation and keeps the one whose S21 block
    is smaller; both blocks are rounding noise (about 1e-15 against a threshold of 20 eps
    ||S||), so which one it keeps depends on its GEMM's rounding, and the two differ by
    those signs after the 2x2 standardisation;
  * a moving 2x2 block whose complex pair is a rounding-level perturbation of a double real
    eigenvalue may split on the way (LAPACK's walk then moves the two 1x1 blocks one after
    the other); whether it splits is decided by rounding too, so those moves are checked by
    INFO, ILST, the backward error and the eigenvalues at the destination.
Tolerances (relative to the matrix's largest entry): double 1e-12 per swap, 1e-11 per move;
single 1e-4.  Runs without a GPU (the GPU kernel's own tests are in test_gpu_tgexc.py)."""
import ctypes as ct
import os
import shutil
import subprocess

import numpy as np
import pytest

import oracle
from conftest import ROOT
from xtgevc3_b200 import pencils

TOL_SWAP = {np.float64: 1e-12, np.float32: 1e-4}
TOL_MOVE = {np.float64: 1e-11, np.float32: 1e-4}


@pytest.fixture(scope="module")
def host():
    if shutil.which("g++") is None:
        pytest.skip("g++ not available")
    out = os.path.join(ROOT, "tests", "_build")
    os.makedirs(out, exist_ok=True)
    lib = os.path.join(out, "libtgexc_blocks_host.so")
    src = os.path.join(ROOT, "tests", "tgexc_blocks_host.cpp")
    hdr = os.path.join(ROOT, "xtgevc3_b200", "csrc", "tgexc_real_blocks.cuh")
    if not os.path.exists(lib) or os.path.getmtime(lib) < max(os.path.getmtime(src), os.path.getmtime(hdr)):
        r = subprocess.run(["g++", "-O2", "-std=c++20", "-pthread", "-shared", "-fPIC", "-ffp-contract=off", "-o", lib,
                            src], capture_output=True, text=True)
        assert r.returncode == 0, r.stderr
    return ct.CDLL(lib)


def _p(a):
    return a.ctypes.data_as(ct.c_void_p)


def _copies(*Ms):
    return [None if M is None else np.asfortranarray(M).copy(order="F") for M in Ms]


def host_tgexc(L, A, B, Q, Z, ifst, ilst):
    pfx = "d" if A.dtype == np.float64 else "s"
    A, B, Q, Z = _copies(A, B, Q, Z)
    n = A.shape[0]
    f, l_ = ct.c_int(ifst), ct.c_int(ilst)
    wq, wz = Q is not None, Z is not None
    info = getattr(L, f"host_{pfx}tgexc")(int(wq), int(wz), n, _p(A), n, _p(B), n, _p(Q) if wq else None, n,
                                          _p(Z) if wz else None, n, ct.byref(f), ct.byref(l_))
    return A, B, Q, Z, f.value, l_.value, info


def host_tgex2(L, A, B, Q, Z, j1, n1, n2):
    pfx = "d" if A.dtype == np.float64 else "s"
    A, B, Q, Z = _copies(A, B, Q, Z)
    n = A.shape[0]
    info = getattr(L, f"host_{pfx}tgex2")(1, 1, n, _p(A), n, _p(B), n, _p(Q), n, _p(Z), n, j1, n1, n2)
    return A, B, Q, Z, info


def rel(M, R):
    return float(np.abs(M - R).max() / max(np.abs(R).max(), 1e-300))


def sign_aligned(A, B, Q, Z, RQ, RZ):
    """A, B, Q, Z with each column of Q and Z (and the matching row / column of A and B)
    given the sign of the reference's."""
    dq = np.where(np.einsum("ij,ij->j", Q, RQ) < 0, -1.0, 1.0).astype(Q.dtype)
    dz = np.where(np.einsum("ij,ij->j", Z, RZ) < 0, -1.0, 1.0).astype(Z.dtype)
    return dq[:, None] * A * dz[None, :], dq[:, None] * B * dz[None, :], Q * dq[None, :], Z * dz[None, :]


def blocks_of(A):
    """(first row 0-based, size) of each diagonal block of the quasi-triangular A"""
    n, k, out = A.shape[0], 0, []
    while k < n:
        s = 2 if k + 1 < n and A[k + 1, k] != 0 else 1
        out.append((k, s))
        k += s
    return out


@pytest.mark.parametrize("dt", [np.float64, np.float32], ids=["d", "s"])
def test_block_swaps_match_lapack_tgex2(host, dt):
    """Every pair of adjacent diagonal blocks of 20 pencils (n = 12): each swap (1x1/1x1,
    1x1/2x2, 2x2/1x1, 2x2/2x2) against LAPACK xTGEX2."""
    kinds = {}
    for seed in range(20):
        S, T, _, _, _, Q, Z = pencils.gen_gges(12, seed, dtype=dt)
        bl = blocks_of(S)
        for (k, s1), (_, s2) in zip(bl, bl[1:]):
            ra, rb, rq, rz, rinfo = oracle.lapack_tgex2_real(S, T, Q, Z, k + 1, s1, s2)
            a, b, q, z, info = host_tgex2(host, S, T, Q, Z, k + 1, s1, s2)
            assert info == rinfo, (seed, k, s1, s2)
            kinds[(s1, s2)] = kinds.get((s1, s2), 0) + 1
            if s1 + s2 == 2:  # two rotations, LAPACK's own conventions: no sign freedom
                assert max(rel(a, ra), rel(b, rb), rel(q, rq), rel(z, rz)) < TOL_SWAP[dt], (seed, k)
            a, b, q, z = sign_aligned(a, b, q, z, rq, rz)
            assert max(rel(a, ra), rel(b, rb), rel(q, rq), rel(z, rz)) < TOL_SWAP[dt], (seed, k, s1, s2)
    assert all(kinds.get(kd, 0) >= 10 for kd in ((1, 1), (1, 2), (2, 1), (2, 2))), kinds


@pytest.mark.parametrize("dt", [np.float64, np.float32], ids=["d", "s"])
def test_moves_match_lapack_tgexc(host, dt):
    """Random moves (forward and backward, from and to 2x2 blocks or their second rows) on
    n = 30 pencils: IFST, ILST and INFO exactly as LAPACK xTGEXC, the arrays to rounding up
    to column signs; the moved eigenvalues sit at ILST."""
    for seed in range(10):
        S, T, _, _, _, Q, Z = pencils.gen_gges(30, 100 + seed, dtype=dt)
        rng = np.random.default_rng(seed)
        for _ in range(5):
            ifst, ilst = (int(x) for x in rng.integers(1, 31, 2))
            r = oracle.lapack_tgexc_real(S, T, Q, Z, ifst, ilst)
            h = host_tgexc(host, S, T, Q, Z, ifst, ilst)
            assert h[4:] == r[4:], (seed, ifst, ilst, h[4:], r[4:])
            a, b, q, z = sign_aligned(h[0], h[1], h[2], h[3], r[2], r[3])
            for M, R in ((a, r[0]), (b, r[1]), (q, r[2]), (z, r[3])):
                assert rel(M, R) < TOL_MOVE[dt], (seed, ifst, ilst)


def test_without_q_and_z_same_pencil(host):
    """WANTQ = WANTZ = 0: A and B are the arrays of the call that updates Q and Z."""
    S, T, _, _, _, Q, Z = pencils.gen_gges(24, 7)
    full = host_tgexc(host, S, T, Q, Z, 20, 2)
    bare = host_tgexc(host, S, T, None, None, 20, 2)
    assert bare[4:] == full[4:]
    np.testing.assert_array_equal(bare[0], full[0])
    np.testing.assert_array_equal(bare[1], full[1])


def _twin_blocks_pencil(seed, n=6):
    """A real generalized Schur pencil with two identical 2x2 blocks (rows 2-3 and 4-5,
    1-based) between 1x1 blocks: their swap is a singular generalized Sylvester equation."""
    rng = np.random.default_rng(seed)
    A = np.triu(rng.standard_normal((n, n)))
    B = np.triu(rng.standard_normal((n, n)))
    B[np.diag_indices(n)] = np.abs(B[np.diag_indices(n)]) + 0.5
    for k in (1, 3):
        A[k:k + 2, k:k + 2] = [[0.7, 1.3], [-0.9, 0.7]]
        B[k:k + 2, k:k + 2] = np.diag([1.2, 0.8])
    Q = np.linalg.qr(rng.standard_normal((n, n)))[0]
    Z = np.linalg.qr(rng.standard_normal((n, n)))[0]
    return [np.asfortranarray(M) for M in (A, B, Q, Z)]


@pytest.mark.parametrize("move", [(4, 2), (2, 5), (5, 1), (6, 1), (1, 6)], ids=lambda m: f"{m[0]}to{m[1]}")
def test_rejected_swaps_match_lapack(host, move):
    """Swapping the two identical blocks is rejected (INFO = 1) with the pencil as it was and
    ILST where the block stopped (IFST moved to its block's first row, 5 -> 4); moves of the
    1x1 blocks across both pairs go through.  All as LAPACK DTGEXC."""
    for seed in range(3):
        A, B, Q, Z = _twin_blocks_pencil(seed)
        r = oracle.lapack_tgexc_real(A, B, Q, Z, *move)
        h = host_tgexc(host, A, B, Q, Z, *move)
        assert h[4:] == r[4:], (seed, move, h[4:], r[4:])
        a, b, q, z = sign_aligned(h[0], h[1], h[2], h[3], r[2], r[3])
        for M, R in ((a, r[0]), (b, r[1]), (q, r[2]), (z, r[3])):
            assert rel(M, R) < 1e-12
        if r[6] == 1 and move in ((4, 2), (2, 5)):  # rejected at the first swap: nothing changed
            for M, M0 in zip(h[:4], (A, B, Q, Z)):
                np.testing.assert_array_equal(M, M0)


def _near_double_pencil(seed, n=8):
    """1x1 blocks with a 2x2 block at rows 3-4 (1-based) whose complex pair has an imaginary
    part at rounding level (a double real eigenvalue, perturbed) and a regular 2x2 block at
    rows 6-7."""
    rng = np.random.default_rng(seed)
    A = np.triu(rng.standard_normal((n, n)))
    B = np.triu(rng.standard_normal((n, n)))
    B[np.diag_indices(n)] = np.abs(B[np.diag_indices(n)]) + 0.5
    g = 10.0 ** rng.uniform(-17, -12)
    for k, disc in ((2, g), (5, 1.0)):
        B[k, k + 1] = 0.0
        a, b = rng.standard_normal(2)
        A[k, k], A[k + 1, k + 1] = a * B[k, k], a * B[k + 1, k + 1]
        A[k, k + 1], A[k + 1, k] = b * B[k + 1, k + 1], -disc / b * B[k, k]
    Q = np.linalg.qr(rng.standard_normal((n, n)))[0]
    Z = np.linalg.qr(rng.standard_normal((n, n)))[0]
    return [np.asfortranarray(M) for M in (A, B, Q, Z)]


def _eigs(A, B):
    import scipy.linalg
    return scipy.linalg.eigvals(A, B)


def test_splitting_block_moves(host):
    """Moves of a near-double 2x2 block that LAPACK's walk splits into two 1x1 blocks on the
    way: INFO and ILST as LAPACK, the pencil (Q A Z^T, Q B Z^T) kept to rounding, A
    quasi-triangular and B triangular, and the block's two eigenvalues at rows ILST, ILST+1
    (to 1e-6: a double eigenvalue is perturbed by sqrt(eps))."""
    done = 0
    for seed in range(400):
        A, B, Q, Z = _near_double_pencil(seed)
        move = (3, 8) if seed % 2 == 0 else (3, 1)
        r = oracle.lapack_tgexc_real(A, B, Q, Z, *move)
        if r[6] != 0 or len(blocks_of(r[0])) == len(blocks_of(A)):
            continue  # LAPACK did not split this one
        a, b, q, z, f, l_, info = host_tgexc(host, A, B, Q, Z, *move)
        assert (f, l_, info) == r[4:], (seed, move)
        for M, M0 in ((a, A), (b, B)):
            assert np.abs(q @ M @ z.T - Q @ M0 @ Z.T).max() < 1e-13 * np.abs(M0).max() * 8
        assert np.abs(np.tril(b, -1)).max() == 0 and np.abs(np.tril(a, -2)).max() == 0
        sub = [k for k in range(7) if a[k + 1, k] != 0]
        assert all(k + 1 not in sub for k in sub)  # 2x2 blocks do not overlap
        moved = np.sort_complex(_eigs(A[2:4, 2:4], B[2:4, 2:4]))
        here = np.sort_complex(_eigs(a[l_ - 1:l_ + 1, l_ - 1:l_ + 1], b[l_ - 1:l_ + 1, l_ - 1:l_ + 1]))
        assert np.abs(moved - here).max() < 1e-6 * max(1.0, np.abs(moved).max()), (seed, moved, here)
        done += 1
        if done == 12:
            break
    assert done >= 8


def _gges_rank_deficient(n, seed):
    """LAPACK DGGES of a Gaussian pencil whose B repeats (or zeroes) its first columns:
    infinite eigenvalues among the finite ones."""
    import scipy.linalg.lapack as la
    rng = np.random.default_rng(seed)
    A, B = rng.standard_normal((n, n)), rng.standard_normal((n, n))
    k = 1 + seed % 3
    B[:, :k] = B[:, k:2 * k]
    S, T, _, _, _, _, Q, Z, _, info = la.dgges(lambda *a: 0, np.asfortranarray(A), np.asfortranarray(B), sort_t=0)
    assert info == 0
    return [np.asfortranarray(M) for M in (S, T, Q, Z)]


@pytest.mark.parametrize("kind", ["graded", "infinite"])
def test_hard_pencils_keep_lapack_control_flow(host, kind):
    """Graded pencils (eigenvalues over 16 orders of magnitude) and pencils with infinite
    eigenvalues: IFST, ILST and INFO exactly as LAPACK DTGEXC on 120 random moves, and every
    result a valid reordering (Q A Z^T, Q B Z^T kept to 1e-14 relative, Q and Z orthogonal,
    A quasi-triangular, B triangular).  Elementwise agreement is not asked here: an
    infinite eigenvalue's B entry becomes rounding noise on the way, differently in LAPACK."""
    n = 14
    for seed in range(20):
        if kind == "graded":
            S, T, _, _, _, Q, Z = pencils.gen_gges(n, 900 + seed, graded=True)
        else:
            S, T, Q, Z = _gges_rank_deficient(n, seed)
        rng = np.random.default_rng(seed)
        for _ in range(6):
            ifst, ilst = (int(x) for x in rng.integers(1, n + 1, 2))
            r = oracle.lapack_tgexc_real(S, T, Q, Z, ifst, ilst)
            a, b, q, z, f, l_, info = host_tgexc(host, S, T, Q, Z, ifst, ilst)
            assert (f, l_, info) == r[4:], (seed, ifst, ilst)
            for M, M0 in ((a, S), (b, T)):
                assert np.abs(q @ M @ z.T - Q @ M0 @ Z.T).max() <= 1e-14 * n * np.abs(M0).max()
            for W in (q, z):
                assert np.abs(W.T @ W - np.eye(n)).max() < 1e-13
            assert np.abs(np.tril(b, -1)).max() == 0 and np.abs(np.tril(a, -2)).max() == 0


@pytest.mark.timeout(300)
def test_kernel_body_on_host_threads(host):
    """The reordering kernel's body (rb::walk_cta, the code the GPU kernel runs) on host
    threads, one std::thread per GPU thread and a std::barrier for the CTA barrier: every
    thread reaches every barrier (a mismatch would hang: the timeout fails it), and A, B, Q,
    Z, IFST, ILST and INFO equal the serial build's bit for bit for 1 to 512 threads."""
    cases = [(pencils.gen_gges(40, 31)[:2] + pencils.gen_gges(40, 31)[5:7], (40, 1)),
             (pencils.gen_gges(40, 31)[:2] + pencils.gen_gges(40, 31)[5:7], (2, 39)),
             (pencils.gen_gges(25, 5)[:2] + pencils.gen_gges(25, 5)[5:7], (13, 14)),
             (_twin_blocks_pencil(1), (4, 2))]
    for (S, T, Q, Z), (f0, l0) in cases:
        ref = host_tgexc(host, S, T, Q, Z, f0, l0)
        n = S.shape[0]
        for nth in (1, 5, 64, 512):
            A, B, Qc, Zc = _copies(S, T, Q, Z)
            f, l_ = ct.c_int(f0), ct.c_int(l0)
            info = host.threads_dtgexc(nth, 1, 1, n, _p(A), n, _p(B), n, _p(Qc), n, _p(Zc), n, ct.byref(f), ct.byref(l_))
            assert (f.value, l_.value, info) == ref[4:], (n, f0, l0, nth)
            for M, R in zip((A, B, Qc, Zc), ref[:4]):
                np.testing.assert_array_equal(M, R)
