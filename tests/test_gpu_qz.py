"""xtgevc3_{z,c}gges (the generalized Schur form of a complex pencil, computed on the GPU)
under the rules of test_qz_host.py (the same kernel body checked on the CPU): A = Q S Z^H,
B = Q T Z^H, Q and Z unitary, S and T upper triangular with T's diagonal real and
non-negative, LAPACK's eigenvalues, k zero betas for a B of rank n - k.  And the chain this
step exists for: the form computed on the device, then the eigenvectors of (A, B) from it
(xtgevc3_ztgevc3_dev, HOWMNY = 'B' back-transformed by Q and Z), checked by their residuals
beta A x - alpha B x and y^H (beta A - alpha B) against the original pencil."""
import numpy as np
import pytest

import xtgevc3_b200 as X
from test_qz_host import check_form, eig_match, pencil

pytestmark = [pytest.mark.gpu, pytest.mark.late(5)]


def _dev(M):
    import torch
    return torch.from_numpy(np.ascontiguousarray(M.T)).cuda().t()


@pytest.mark.parametrize("dt", [np.complex128, np.complex64], ids=["z", "c"])
def test_gges_random_pencils(cuda_ok, dt):
    single = dt == np.complex64
    for n in (1, 5, 40, 100):
        A, B = pencil(n, 300 + n, dt)
        S, T, alpha, beta, Q, Z, info = X.gges(A, B)
        assert info == 0
        a2, b2 = check_form(A, B, S, T, Q, Z, single)
        np.testing.assert_array_equal(alpha, a2)
        np.testing.assert_array_equal(beta, b2)
        assert eig_match(alpha, beta, A, B, single) == 0


def test_gges_infinite_eigenvalues(cuda_ok):
    for n, k in ((6, 1), (12, 2), (30, 3)):
        A, B = pencil(n, 900 + n, rank_drop=k)
        S, T, alpha, beta, Q, Z, info = X.gges(A, B)
        assert info == 0
        check_form(A, B, S, T, Q, Z)
        assert eig_match(alpha, beta, A, B) == k


def test_gges_device_form_matches_host_form(cuda_ok):
    import torch
    A, B = pencil(48, 4)
    S, T, alpha, beta, Q, Z, info = X.gges(A, B)
    dA, dB = _dev(A), _dev(B)
    dQ = torch.empty((48, 48), dtype=torch.complex128, device="cuda").t()
    dZ = torch.empty((48, 48), dtype=torch.complex128, device="cuda").t()
    da, db, dinfo = X.gges_dev(dA, dB, dQ, dZ)
    torch.cuda.synchronize()
    assert dinfo == info == 0
    for D, H in ((dA, S), (dB, T), (dQ, Q), (dZ, Z), (da, alpha), (db, beta)):
        np.testing.assert_array_equal(D.cpu().numpy(), H)


def test_schur_form_then_eigenvectors_on_the_device(cuda_ok):
    """The QZ step and the eigenvector solve chained on device memory (only alpha and beta,
    2 n numbers, cross to the host, as the eigenvector entry point takes them there)."""
    import torch
    n = 96
    A, B = pencil(n, 11)
    dA, dB = _dev(A), _dev(B)
    dQ = torch.empty((n, n), dtype=torch.complex128, device="cuda").t()
    dZ = torch.empty((n, n), dtype=torch.complex128, device="cuda").t()
    alpha, beta, info = X.gges_dev(dA, dB, dQ, dZ)
    assert info == 0
    al, be = alpha.cpu().numpy(), beta.cpu().numpy()
    m, info = X.tgevc3_dev("B", "B", dA, dB, al, be, VL=dQ, VR=dZ)
    torch.cuda.synchronize()
    assert (m, info) == (n, 0)
    VL, VR = dQ.cpu().numpy(), dZ.cpu().numpy()
    na, nb = np.abs(A).max(), np.abs(B).max()
    for k in range(n):
        x, y = VR[:, k], VL[:, k]
        scale = (abs(be[k]) * na + abs(al[k]) * nb) * n
        assert np.abs(be[k] * (A @ x) - al[k] * (B @ x)).max() <= 1e-12 * scale * np.abs(x).max()
        assert np.abs(be[k] * (y.conj() @ A) - al[k] * (y.conj() @ B)).max() <= 1e-12 * scale * np.abs(y).max()


# ---- real pencils -------------------------------------------------------------------------
from test_qz_host import check_real_form, real_eig_match, rpencil  # noqa: E402


@pytest.mark.parametrize("dt", [np.float64, np.float32], ids=["d", "s"])
def test_real_gges_random_pencils(cuda_ok, dt):
    single = dt == np.float32
    for n in (1, 4, 40, 100):
        A, B = rpencil(n, 600 + n, dt)
        S, T, ar, ai, be, Q, Z, info = X.gges(A, B)
        assert info == 0
        check_real_form(A, B, S, T, Q, Z, ar, ai, be, single)
        assert real_eig_match(A, B, ar, ai, be, single) == 0


def test_real_gges_infinite_eigenvalues(cuda_ok):
    for n, k in ((6, 1), (12, 2), (30, 3)):
        A, B = rpencil(n, 800 + n, rank_drop=k)
        S, T, ar, ai, be, Q, Z, info = X.gges(A, B)
        assert info == 0
        check_real_form(A, B, S, T, Q, Z, ar, ai, be)
        assert real_eig_match(A, B, ar, ai, be) == k


def test_real_schur_form_then_eigenvectors_on_the_device(cuda_ok):
    """DGGES then DTGEVC3 on device memory (alphar, alphai, beta: 3 n numbers to the host)."""
    import torch
    n = 96
    A, B = rpencil(n, 12)
    dA, dB = _dev(A), _dev(B)
    dQ = torch.empty((n, n), dtype=torch.float64, device="cuda").t()
    dZ = torch.empty((n, n), dtype=torch.float64, device="cuda").t()
    ar, ai, be, info = X.gges_dev(dA, dB, dQ, dZ)
    assert info == 0
    ar, ai, be = ar.cpu().numpy(), ai.cpu().numpy(), be.cpu().numpy()
    m, info = X.tgevc3_dev("B", "B", dA, dB, ar, be, alphai=ai, VL=dQ, VR=dZ)
    torch.cuda.synchronize()
    assert (m, info) == (n, 0)
    VL, VR = dQ.cpu().numpy(), dZ.cpu().numpy()
    na, nb = np.abs(A).max(), np.abs(B).max()
    k = 0
    while k < n:
        if ai[k] == 0:
            x, y, a, w = VR[:, k], VL[:, k], ar[k], 1
        else:
            x, y, a, w = VR[:, k] + 1j * VR[:, k + 1], VL[:, k] + 1j * VL[:, k + 1], ar[k] + 1j * ai[k], 2
        scale = (abs(be[k]) * na + abs(a) * nb) * n
        assert np.abs(be[k] * (A @ x) - a * (B @ x)).max() <= 1e-12 * scale * np.abs(x).max()
        assert np.abs(be[k] * (y.conj() @ A) - a * (y.conj() @ B)).max() <= 1e-12 * scale * np.abs(y).max()
        k += w


@pytest.mark.parametrize("sa,sb", [(1e200, 1.0), (1e-200, 1.0), (1.0, 1e200), (1e200, 1e-200)],
                         ids=["A_huge", "A_tiny", "B_huge", "both"])
@pytest.mark.parametrize("cplx", [False, True], ids=["d", "z"])
def test_gges_scales_badly_scaled_pencils(cuda_ok, sa, sb, cplx):
    """xGGES's scaling on the device (the pencils of tests/test_gges_scale_host.py, where the same
    flow runs on host arrays): LAPACK's eigenvalues (relative 1e-9, compared as (alpha / sa) /
    (beta / sb)), A = Q S Z^H and B = Q T Z^H to 1e-12 n, everything finite."""
    import scipy.linalg.lapack as la
    n = 24
    rng = np.random.default_rng(9)
    A0, B0 = rng.standard_normal((n, n)), rng.standard_normal((n, n))
    if cplx:
        A0, B0 = A0 + 1j * rng.standard_normal((n, n)), B0 + 1j * rng.standard_normal((n, n))
    A, B = A0 * sa, B0 * sb
    out = X.gges(A, B)
    if cplx:
        S, T, al, be, Q, Z, info = out
        r = la.zgges(lambda a, b: 0, A, B)
        lam, lam_r = (al / sa) / (be / sb), (r[3] / sa) / (r[4] / sb)
        ev = (al, be)
    else:
        S, T, ar, ai, be, Q, Z, info = out
        r = la.dgges(lambda x, y, z: 0, A, B)
        lam, lam_r = ((ar + 1j * ai) / sa) / (be / sb), ((r[3] + 1j * r[4]) / sa) / (r[5] / sb)
        ev = (ar, ai, be)
    assert info == 0
    for M in (S, T, Q, Z, *ev):
        assert np.all(np.isfinite(M))
    for x, y in ((lam, lam_r), (lam_r, lam)):
        d = np.abs(x[:, None] - y[None, :]).min(1) / np.abs(x)
        assert d.max() <= 1e-9, d.max()
    for M, M0 in ((S, A), (T, B)):
        assert np.abs(Q @ M @ Z.conj().T - M0).max() <= 1e-12 * n * np.abs(M0).max()


@pytest.mark.parametrize("kind", ["none", "row_offdiag", "row_zero_col", "chain", "triangular", "permuted_triangular"],
                         ids=str)
@pytest.mark.parametrize("cplx", [False, True], ids=["d", "z"])
def test_gges_balances_structured_pencils(cuda_ok, kind, cplx):
    """xGGES's permutation balancing on the device (the pencils of tests/test_ggbal_host.py, where
    the same flow runs on host threads and xGGBAL equals LAPACK's bit for bit): A = VSL S VSR^H,
    B = VSL T VSR^H to 1e-12 n, LAPACK xGGES's eigenvalues (relative 1e-9)."""
    import scipy.linalg.lapack as la
    from test_ggbal_host import structured
    n = 17
    A, B = structured(kind, n, 5, cplx)
    out = X.gges(A, B)
    if cplx:
        S, T, al, be, Q, Z, info = out
        lam = al / be
        r = la.zgges(lambda a, b: 0, A, B)
        lam_r = r[3] / r[4]
    else:
        S, T, ar, ai, be, Q, Z, info = out
        lam = (ar + 1j * ai) / be
        r = la.dgges(lambda x, y, z: 0, A, B)
        lam_r = (r[3] + 1j * r[4]) / r[5]
    assert info == 0
    for M, M0 in ((S, A), (T, B)):
        assert np.abs(Q @ M @ Z.conj().T - M0).max() <= 1e-12 * n * np.abs(M0).max()
    fin = np.isfinite(lam_r) & np.isfinite(lam)
    for x, y in ((lam[fin], lam_r[fin]), (lam_r[fin], lam[fin])):
        d = np.abs(x[:, None] - y[None, :]).min(1) / np.maximum(np.abs(x), 1e-300)
        assert d.max() <= 1e-9, (kind, d.max())


@pytest.mark.late(2)  # the balancing kernels alone, not the QZ step
@pytest.mark.parametrize("kind", ["none", "row_offdiag", "row_zero_col", "chain", "triangular", "permuted_triangular"],
                         ids=str)
@pytest.mark.parametrize("cplx", [False, True], ids=["d", "z"])
def test_ggbal_ggbak_entry_points_match_lapack(cuda_ok, kind, cplx):
    """xtgevc3_*ggbal / *ggbak (JOB = 'P') against LAPACK DGGBAL / ZGGBAL / DGGBAK, bit for bit (the
    pencils and the oracle calls of tests/test_ggbal_host.py)."""
    from test_ggbal_host import lapack_ggbal, structured
    import ctypes as ct
    import oracle
    n = 17
    A, B = structured(kind, n, 5, cplx)
    r = lapack_ggbal(A, B)
    a, b, ilo, ihi, ls, rs, info = X.ggbal(A, B)
    assert info == 0 and (ilo, ihi) == (r[2], r[3])
    assert np.array_equal(a, r[0]) and np.array_equal(b, r[1])
    assert np.array_equal(ls, r[4]) and np.array_equal(rs, r[5])
    if not cplx:
        V = np.asfortranarray(np.random.default_rng(1).standard_normal((n, 7)))
        for side, scale in (("L", ls), ("R", rs)):
            Vr = V.copy(order="F")
            iv = lambda v: ct.byref(ct.c_int(v))  # noqa: E731
            inf = ct.c_int()
            oracle._openblas().scipy_dggbak_(ct.c_char_p(b"P"), ct.c_char_p(side.encode()), iv(n), iv(ilo), iv(ihi),
                                              scale.ctypes.data_as(ct.c_void_p), scale.ctypes.data_as(ct.c_void_p),
                                              iv(7), Vr.ctypes.data_as(ct.c_void_p), iv(n), ct.byref(inf),
                                              ct.c_size_t(1), ct.c_size_t(1))
            Vh, info = X.ggbak(V, ilo, ihi, ls, rs, side=side)
            assert info == 0 and np.array_equal(Vh, Vr), side
