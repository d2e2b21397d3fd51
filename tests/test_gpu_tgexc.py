"""xtgevc3_{z,c,d,s}tgexc (eigenvalue reordering of a generalized Schur pencil) against LAPACK
Z/C/D/STGEXC.

The oracle is LAPACK's own xTGEXC from SciPy, given the same pencil (complex: the generalized
Schur form of a pencil with iid complex N(0,1) entries, LAPACK xGGES through SciPy's qz; real:
LAPACK DGGES of iid N(0,1) pencils, and constructed pencils for rejected and splitting
swaps) and the same move.  Swaps of 1x1 blocks apply the same rotations as LAPACK, so A, B, Q
and Z agree to rounding; swaps involving a real 2x2 block agree up to the sign of each
column of Q and Z (see the block tests below).  Tolerance: elementwise difference relative
to the matrix's largest entry, 1e-12 (double) / 2e-4 (single) per move, 1e-11 / 1e-10 for
long block moves.
"""
import numpy as np
import pytest

import oracle
import xtgevc3_b200 as X

pytestmark = pytest.mark.gpu

TOL = {np.complex128: 1e-12, np.complex64: 2e-4}


def _rel(M, R):
    return float(np.abs(M - R).max() / max(np.abs(R).max(), 1e-300))


MOVES = [(4, 31), (36, 3), (1, 40), (40, 1), (11, 12), (12, 11)]


@pytest.mark.parametrize("dt", [np.complex128, np.complex64], ids=["z", "c"])
@pytest.mark.parametrize("move", MOVES, ids=lambda m: f"{m[0]}to{m[1]}")
def test_tgexc_matches_lapack(cuda_ok, dt, move):
    ifst, ilst = move
    A, B, Q, Z = oracle.complex_schur_pencil(40, 3, dt)
    ra, rb, rq, rz, rinfo = oracle.lapack_tgexc(A, B, Q, Z, ifst, ilst)
    a, b, q, z, il, info = X.tgexc(A, B, Q, Z, ifst, ilst)
    assert (info, il) == (rinfo, ilst) == (0, ilst)
    tol = TOL[dt]
    for M, R in ((a, ra), (b, rb), (q, rq), (z, rz)):
        assert _rel(M, R) < tol
    # the moved eigenvalue sits at ilst, the pencil is still triangular
    k = ilst - 1
    assert abs(a[k, k] / b[k, k] - A[ifst - 1, ifst - 1] / B[ifst - 1, ifst - 1]) < 1e3 * tol * abs(A[ifst - 1, ifst - 1] / B[ifst - 1, ifst - 1])
    assert (np.tril(a, -1) == 0).all() and (np.tril(b, -1) == 0).all()


def test_tgexc_without_q_z(cuda_ok):
    """wantq = wantz = 0: A and B as LAPACK's, Q and Z not referenced."""
    A, B, Q, Z = oracle.complex_schur_pencil(60, 8)
    ra, rb, _, _, rinfo = oracle.lapack_tgexc(A, B, None, None, 50, 2)
    a, b, q, z, il, info = X.tgexc(A, B, None, None, 50, 2)
    assert (info, il, q, z) == (0, 2, None, None)
    assert _rel(a, ra) < 1e-12 and _rel(b, rb) < 1e-12


def test_tgexc_long_move_and_invariants(cuda_ok):
    """n = 400, the last eigenvalue to the top (399 swaps): LAPACK's result to rounding, and
    Q A Z^H, Q B Z^H unchanged."""
    A, B, Q, Z = oracle.complex_schur_pencil(400, 5)
    ra, rb, rq, rz, _ = oracle.lapack_tgexc(A, B, Q, Z, 400, 1)
    a, b, q, z, il, info = X.tgexc(A, B, Q, Z, 400, 1)
    assert (info, il) == (0, 1)
    for M, R in ((a, ra), (b, rb), (q, rq), (z, rz)):
        assert _rel(M, R) < 1e-11
    for M, M0 in ((a, A), (b, B)):
        assert np.abs(q @ M @ z.conj().T - Q @ M0 @ Z.conj().T).max() < 1e-12 * np.abs(M0).max() * 400


def test_tgexc_device_form_matches_host_form(cuda_ok):
    """xtgevc3_ztgexc_dev on column-major CUDA tensors gives the host form's arrays bit for bit."""
    import torch
    A, B, Q, Z = oracle.complex_schur_pencil(120, 9)
    a, b, q, z, il, info = X.tgexc(A, B, Q, Z, 100, 5)

    def dev(M):
        return torch.from_numpy(np.ascontiguousarray(M.T)).cuda().t()

    dA, dB, dQ, dZ = dev(A), dev(B), dev(Q), dev(Z)
    il2, info2 = X.tgexc_dev(dA, dB, dQ, dZ, 100, 5)
    torch.cuda.synchronize()
    assert (il2, info2) == (il, info) == (5, 0)
    for D, H in ((dA, a), (dB, b), (dQ, q), (dZ, z)):
        np.testing.assert_array_equal(D.cpu().numpy(), H)


def test_tgexc_rejected_swap_matches_lapack(cuda_ok):
    """Badly scaled 3 x 3 pencils on which LAPACK ZTGEXC rejects a swap (fixture made by
    tests/golden/make_tgexc_rejections.py): forward and backward moves where swaps were
    applied before the rejection, and one more.  INFO = 1, the returned ILST (the row the
    eigenvalue had reached) and A, B, Q, Z (the accepted swaps kept) must equal LAPACK's;
    entries span hundreds of orders of magnitude, so each matrix is compared column by
    column relative to that column's largest entry."""
    import os
    d = np.load(os.path.join(os.path.dirname(__file__), "golden", "tgexc", "z_rejections.npz"))
    for i in range(3):
        A, B, mv = d[f"A{i}"], d[f"B{i}"], d[f"move{i}"]
        ifst, ilst = int(mv[0]), int(mv[1])
        I = np.eye(3, dtype=np.complex128, order="F")
        ra, rb, rq, rz, ril, rinfo = oracle.lapack_tgexc_ilst(A, B, I, I, ifst, ilst)
        assert rinfo == 1
        a, b, q, z, il, info = X.tgexc(A, B, I.copy(order="F"), I.copy(order="F"), ifst, ilst)
        assert (info, il) == (rinfo, ril), (i, info, il, rinfo, ril)
        for M, R in ((a, ra), (b, rb), (q, rq), (z, rz)):
            den = np.abs(R).max(0)
            den[den == 0] = 1.0
            assert float((np.abs(M - R).max(0) / den).max()) < 1e-12, i


# ---- real pencils: D/STGEXC over 1x1 blocks --------------------------------------------
TOL_R = {np.float64: 1e-12, np.float32: 2e-4}


def _real_triangular_pencil(n, seed, dt):
    """A real generalized Schur pencil with only 1x1 blocks: A, B upper triangular (N(0,1)
    parts, |B_kk| kept away from 0), Q and Z orthogonal."""
    rng = np.random.default_rng(seed)
    A = np.triu(rng.standard_normal((n, n)))
    B = np.triu(rng.standard_normal((n, n)))
    B[np.diag_indices(n)] = np.abs(B[np.diag_indices(n)]) + 0.5
    Q = np.linalg.qr(rng.standard_normal((n, n)))[0]
    Z = np.linalg.qr(rng.standard_normal((n, n)))[0]
    return tuple(np.asfortranarray(M.astype(dt)) for M in (A, B, Q, Z))


@pytest.mark.parametrize("dt", [np.float64, np.float32], ids=["d", "s"])
@pytest.mark.parametrize("move", MOVES, ids=lambda m: f"{m[0]}to{m[1]}")
def test_real_tgexc_matches_lapack(cuda_ok, dt, move):
    """Moves across real eigenvalues: LAPACK D/STGEXC's swaps (two rotations each, the real
    routine's sign conventions), so A, B, Q and Z agree with LAPACK's to rounding."""
    ifst, ilst = move
    A, B, Q, Z = _real_triangular_pencil(40, 5, dt)
    ra, rb, rq, rz, rinfo = oracle.lapack_tgexc(A, B, Q, Z, ifst, ilst)
    a, b, q, z, il, info = X.tgexc(A, B, Q, Z, ifst, ilst)
    assert (info, il) == (rinfo, ilst) == (0, ilst)
    for M, R in ((a, ra), (b, rb), (q, rq), (z, rz)):
        assert _rel(M, R) < TOL_R[dt]
    k = ilst - 1
    assert abs(a[k, k] / b[k, k] - A[ifst - 1, ifst - 1] / B[ifst - 1, ifst - 1]) < 1e-6 * max(
        1.0, abs(A[ifst - 1, ifst - 1] / B[ifst - 1, ifst - 1]))
    assert np.allclose(np.tril(a, -1), 0) and np.allclose(np.tril(b, -1), 0)


def test_real_tgexc_device_form_and_no_qz(cuda_ok):
    """Device form (column-major CUDA tensors, in place), and WANTQ = WANTZ = 0: the same A
    and B as LAPACK with Q, Z not referenced."""
    import torch
    A, B, Q, Z = _real_triangular_pencil(64, 9, np.float64)
    ra, rb, _, _, rinfo = oracle.lapack_tgexc(A, B, None, None, 50, 3)

    def dev(M):
        return torch.from_numpy(np.ascontiguousarray(M.T)).cuda().t()

    da, db = dev(A), dev(B)
    il, info = X.tgexc_dev(da, db, None, None, 50, 3)
    torch.cuda.synchronize()
    assert (info, il) == (rinfo, 3) == (0, 3)
    assert _rel(da.t().cpu().numpy().T, ra) < 1e-12 and _rel(db.t().cpu().numpy().T, rb) < 1e-12


# ---- real pencils with 2x2 blocks: the block kernel ---------------------------------------
# Parity rules as for the CPU build of the same arithmetic (test_tgexc_blocks_host.py): IFST,
# ILST and INFO exactly as LAPACK D/STGEXC, the arrays to rounding up to the sign of each
# column of Q and Z (LAPACK's choice between its RQ and QR re-triangularisation of a swapped
# 2x2 block is decided by rounding noise), splitting blocks by invariants.
from test_tgexc_blocks_host import (_near_double_pencil, _twin_blocks_pencil, blocks_of,  # noqa: E402
                                    sign_aligned)

BLOCK_MOVES = [(1, 40), (40, 1), (7, 33), (33, 7), (20, 21), (21, 20), (2, 39), (39, 2)]


@pytest.mark.parametrize("dt", [np.float64, np.float32], ids=["d", "s"])
@pytest.mark.parametrize("move", BLOCK_MOVES, ids=lambda m: f"{m[0]}to{m[1]}")
@pytest.mark.late(1)
def test_real_tgexc_blocks_match_lapack(cuda_ok, dt, move):
    """Moves through a real xGGES pencil (n = 40, most eigenvalues complex pairs)."""
    from xtgevc3_b200 import pencils
    S, P, _, _, _, Q, Z = pencils.gen_gges(40, 31, dtype=dt)
    assert len(blocks_of(S)) < 40  # 2x2 blocks present
    r = oracle.lapack_tgexc_real(S, P, Q, Z, *move)
    a, b, q, z, f, il, info = X.tgexc(S, P, Q, Z, *move, with_ifst=True)
    assert (f, il, info) == r[4:], (move, (f, il, info), r[4:])
    a, b, q, z = sign_aligned(a, b, q, z, r[2], r[3])
    for M, R in ((a, r[0]), (b, r[1]), (q, r[2]), (z, r[3])):
        assert _rel(M, R) < {np.float64: 1e-11, np.float32: 1e-4}[dt]


@pytest.mark.late(1)
def test_real_tgexc_blocks_long_move(cuda_ok):
    """n = 400, the last block to the top and back: LAPACK's IFST / ILST / INFO, its arrays
    up to column signs, and Q A Z^T, Q B Z^T unchanged."""
    from xtgevc3_b200 import pencils
    S, P, _, _, _, Q, Z = pencils.gen_gges(400, 5)
    for move in ((400, 1), (1, 400)):
        r = oracle.lapack_tgexc_real(S, P, Q, Z, *move)
        a, b, q, z, f, il, info = X.tgexc(S, P, Q, Z, *move, with_ifst=True)
        assert (f, il, info) == r[4:], move
        for M, M0 in ((a, S), (b, P)):
            assert np.abs(q @ M @ z.T - Q @ M0 @ Z.T).max() < 1e-12 * np.abs(M0).max() * 400
        a, b, q, z = sign_aligned(a, b, q, z, r[2], r[3])
        for M, R in ((a, r[0]), (b, r[1]), (q, r[2]), (z, r[3])):
            assert _rel(M, R) < 1e-10


@pytest.mark.parametrize("move", [(4, 2), (2, 5), (5, 1), (6, 1), (1, 6)], ids=lambda m: f"{m[0]}to{m[1]}")
@pytest.mark.late(1)
def test_real_tgexc_blocks_rejections(cuda_ok, move):
    """Two identical 2x2 blocks: their swap is rejected (INFO = 1, the pencil as LAPACK
    leaves it, ILST where the block stopped, IFST moved to its block's first row)."""
    A, B, Q, Z = _twin_blocks_pencil(1)
    r = oracle.lapack_tgexc_real(A, B, Q, Z, *move)
    a, b, q, z, f, il, info = X.tgexc(A, B, Q, Z, *move, with_ifst=True)
    assert (f, il, info) == r[4:], (move, (f, il, info), r[4:])
    a, b, q, z = sign_aligned(a, b, q, z, r[2], r[3])
    for M, R in ((a, r[0]), (b, r[1]), (q, r[2]), (z, r[3])):
        assert _rel(M, R) < 1e-12


@pytest.mark.late(1)
def test_real_tgexc_blocks_splitting(cuda_ok):
    """Near-double 2x2 blocks that LAPACK's walk splits: INFO and ILST as LAPACK, the pencil
    kept, the two eigenvalues at rows ILST, ILST + 1 (to 1e-6)."""
    import scipy.linalg
    done = 0
    for seed in range(200):
        A, B, Q, Z = _near_double_pencil(seed)
        move = (3, 8) if seed % 2 == 0 else (3, 1)
        r = oracle.lapack_tgexc_real(A, B, Q, Z, *move)
        if r[6] != 0 or len(blocks_of(r[0])) == len(blocks_of(A)):
            continue
        a, b, q, z, f, il, info = X.tgexc(A, B, Q, Z, *move, with_ifst=True)
        assert (f, il, info) == r[4:], seed
        for M, M0 in ((a, A), (b, B)):
            assert np.abs(q @ M @ z.T - Q @ M0 @ Z.T).max() < 1e-13 * np.abs(M0).max() * 8
        moved = np.sort_complex(scipy.linalg.eigvals(A[2:4, 2:4], B[2:4, 2:4]))
        here = np.sort_complex(scipy.linalg.eigvals(a[il - 1:il + 1, il - 1:il + 1], b[il - 1:il + 1, il - 1:il + 1]))
        assert np.abs(moved - here).max() < 1e-6 * max(1.0, np.abs(moved).max()), seed
        done += 1
        if done == 6:
            break
    assert done >= 4


@pytest.mark.late(1)
def test_real_tgexc_blocks_device_form(cuda_ok):
    """xtgevc3_dtgexc_dev on column-major CUDA tensors: the host form's arrays and IFST /
    ILST bit for bit; without Q and Z the same A and B."""
    import torch
    from xtgevc3_b200 import pencils
    S, P, _, _, _, Q, Z = pencils.gen_gges(96, 12)
    a, b, q, z, f, il, info = X.tgexc(S, P, Q, Z, 90, 4, with_ifst=True)

    def dev(M):
        return torch.from_numpy(np.ascontiguousarray(M.T)).cuda().t()

    dA, dB, dQ, dZ = dev(S), dev(P), dev(Q), dev(Z)
    assert X.tgexc_dev(dA, dB, dQ, dZ, 90, 4, with_ifst=True) == (f, il, info)
    torch.cuda.synchronize()
    for D, H in ((dA, a), (dB, b), (dQ, q), (dZ, z)):
        np.testing.assert_array_equal(D.cpu().numpy(), H)
    dA, dB = dev(S), dev(P)
    assert X.tgexc_dev(dA, dB, None, None, 90, 4, with_ifst=True) == (f, il, info)
    np.testing.assert_array_equal(dA.cpu().numpy(), a)
    np.testing.assert_array_equal(dB.cpu().numpy(), b)
