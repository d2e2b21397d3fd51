"""xtgevc3_{d,s,z,c}tgsna (JOB = 'E': eigenvalue condition numbers; JOB = 'V' / 'B': the
eigenvector condition estimates DIF) against LAPACK xTGSNA.

The oracle is LAPACK's own xTGSNA from SciPy's bundled OpenBLAS, given the same Schur
pencil and the same eigenvectors (LAPACK xTGEVC's, in Schur coordinates).  S does not
depend on how an eigenvector is scaled, so the condition numbers computed from this
library's own eigenvectors (xtgevc3_*tgevc3, HOWMNY='A') must match too.  Tolerance:
relative difference 1e-10 (double) / 1e-3 (single).
"""
import numpy as np
import pytest

import oracle
import xtgevc3_b200 as X
from xtgevc3_b200 import pencils

pytestmark = pytest.mark.gpu

TOL = {np.float64: 1e-10, np.complex128: 1e-10, np.float32: 1e-3, np.complex64: 1e-3}


def _pencil(dt, n, seed):
    if np.issubdtype(dt, np.complexfloating):
        S, P, a, b, Q, Z = pencils.gen_gges(n, seed, dtype=dt)
        return S, P, a, None, b
    S, P, ar, ai, be, Q, Z = pencils.gen_gges(n, seed, dtype=dt)
    return S, P, ar, ai, be


def _rel(a, b):
    return float(np.max(np.abs(a - b) / np.maximum(np.abs(b), np.finfo(np.float64).tiny)))


CASES = [(np.float64, 150, "A"), (np.float64, 131, "S"), (np.float32, 120, "A"), (np.complex128, 110, "A"),
         (np.complex128, 97, "S"), (np.complex64, 90, "A")]


@pytest.mark.parametrize("case", CASES, ids=lambda c: f"{np.dtype(c[0]).name}-{c[1]}-{c[2]}")
def test_tgsna_matches_lapack(cuda_ok, case):
    dt, n, howmny = case
    S, P, al, ai, be = _pencil(dt, n, 40 + n)
    VL, VR = oracle.lapack_tgevc(S, P)
    sel = None
    if howmny == "S":
        sel = (np.random.default_rng(n).random(n) < 0.4).astype(np.int32)
        items = oracle.selected_items(n, "S", sel, ai if ai is not None else np.zeros(n))
        cols = []
        for k, pair in items:
            cols += [k, k + 1] if pair else [k]
        VL, VR = np.asfortranarray(VL[:, cols]), np.asfortranarray(VR[:, cols])
    ref, rm, rinfo = oracle.lapack_tgsna(howmny, S, P, VL, VR, select=sel)
    got, m, info = X.tgsna(howmny, S, P, VL, VR, select=sel)
    assert (m, info) == (rm, rinfo) == (len(ref), 0)
    assert _rel(got, ref) < TOL[dt], _rel(got, ref)


@pytest.mark.parametrize("dt", [np.float64, np.complex128], ids=["d", "z"])
def test_tgsna_from_own_eigenvectors(cuda_ok, dt):
    """tgevc3 on the GPU, then tgsna on the GPU: the same S as LAPACK from LAPACK's vectors."""
    n = 300
    S, P, al, ai, be = _pencil(dt, n, 7)
    VL0, VR0 = oracle.lapack_tgevc(S, P)
    ref, _, _ = oracle.lapack_tgsna("A", S, P, VL0, VR0)
    VL, VR, m, info = X.tgevc3("B", "A", S, P, al, be, alphai=ai)
    got, m2, info2 = X.tgsna("A", S, P, VL, VR)
    assert info == info2 == 0 and m2 == n
    assert _rel(got, ref) < 1e-9, _rel(got, ref)


def test_tgsna_schur_like_700(cuda_ok):
    """A larger, ill-conditioned Schur-form stand-in pencil (condition numbers spread over
    many orders of magnitude)."""
    n = 700
    S, P, ar, ai, be = pencils.gen_schur_like(n, 25)
    VL, VR = oracle.lapack_tgevc(S, P)
    ref, _, _ = oracle.lapack_tgsna("A", S, P, VL, VR)
    got, m, info = X.tgsna("A", S, P, VL, VR)
    assert (m, info) == (n, 0)
    assert _rel(got, ref) < 1e-8, _rel(got, ref)


# ---- DIF (JOB = 'V' / 'B') ----------------------------------------------------------------
# DTGSNA's estimate, from a copy reordered per eigenvalue and xTGSYL's +-1 look-ahead; the
# look-ahead follows the reordered copy's signs, which LAPACK leaves to rounding in swaps of
# 2x2 blocks (test_tgsna_dif_host.py checks the estimate step exactly on LAPACK's own
# reordered copies).  Here: most DIFs equal LAPACK's to rounding, every one within a factor
# of two of LAPACK's, JOB = 'B' gives JOB = 'E''s S and JOB = 'V''s DIF, the device form
# the host form's values.
from test_tgsna_dif_host import _twin_blocks_pencil, blocks  # noqa: E402


@pytest.mark.parametrize("dt", [np.float64, np.float32], ids=["d", "s"])
@pytest.mark.late(4)
def test_dif_matches_lapack(cuda_ok, dt):
    tol = {np.float64: 1e-12, np.float32: 1e-4}[dt]
    same = total = 0
    for seed, n in ((1, 9), (2, 24), (3, 40)):
        S, T = pencils.gen_gges(n, 90 + seed, dtype=dt)[:2]
        _, d, m, info = oracle.lapack_tgsna("A", S, T, None, None, job="V")
        s_, h, m2, info2 = X.tgsna("A", S, T, None, None, job="V")
        assert s_ is None and (m2, info2) == (m, info) == (n, 0)
        for ks in range(n):
            total += 1
            if abs(h[ks] - d[ks]) <= tol * abs(d[ks]):
                same += 1
            else:
                assert 0.5 <= h[ks] / d[ks] <= 2.0, (seed, ks, h[ks], d[ks])
    assert same >= 0.8 * total, (same, total)


@pytest.mark.late(4)
def test_dif_job_b_and_device_form(cuda_ok):
    import torch
    S, P, ar, ai, be = _pencil(np.float64, 30, 17)
    VL, VR = oracle.lapack_tgevc(S, P)
    s_e, m_e, _ = X.tgsna("A", S, P, VL, VR, job="E")
    _, d_v, m_v, _ = X.tgsna("A", S, P, None, None, job="V")
    s_b, d_b, m_b, info = X.tgsna("A", S, P, VL, VR, job="B")
    assert info == 0 and m_e == m_v == m_b == 30
    np.testing.assert_array_equal(s_b, s_e)
    np.testing.assert_array_equal(d_b, d_v)

    def dev(M):
        return torch.from_numpy(np.ascontiguousarray(M.T)).cuda().t()

    d_dev, m, info = X.tgsna_dif_dev(dev(S), dev(P))
    assert (m, info) == (30, 0)
    np.testing.assert_array_equal(d_dev.cpu().numpy(), d_v)


@pytest.mark.late(4)
def test_dif_selection_and_rejection(cuda_ok):
    """HOWMNY = 'S' (a pair selected by its second row), and a rejected reordering (the
    second of two identical 2x2 blocks: DIF = 0), as LAPACK."""
    S, T = pencils.gen_gges(14, 77)[:2]
    sel = np.zeros(14, dtype=np.int32)
    sel[[k for k, p in blocks(S) if p][0] + 1] = 1
    sel[[k for k, p in blocks(S) if not p][:1]] = 1
    _, d, m, _ = oracle.lapack_tgsna("S", S, T, None, None, select=sel, job="V")
    _, h, m2, info = X.tgsna("S", S, T, None, None, select=sel, job="V")
    assert (m2, info) == (m, 0) == (3, 0)
    assert h[1] == h[2]  # the pair's two entries (the real block at row 0 comes first)
    assert all(abs(x - y) <= 1e-12 * y or 0.5 <= x / y <= 2.0 for x, y in zip(h, d)), (h, d)
    A, B = _twin_blocks_pencil(2)
    _, d, m, _ = oracle.lapack_tgsna("A", A, B, None, None, job="V")
    _, h, m2, _ = X.tgsna("A", A, B, None, None, job="V")
    assert d[3] == d[4] == 0
    np.testing.assert_array_equal(h[3:5], d[3:5])


@pytest.mark.parametrize("dt", [np.complex128, np.complex64], ids=["z", "c"])
@pytest.mark.late(4)
def test_complex_dif_matches_lapack(cuda_ok, dt):
    """Z/CTGSNA JOB = 'V': the reordering is LAPACK's rotations, so every DIF equals LAPACK's
    to rounding (1e-10 double, 1e-3 single); the device form gives the host form's values."""
    import torch
    tol = {np.complex128: 1e-10, np.complex64: 1e-3}[dt]
    for seed, n in ((1, 1), (2, 7), (3, 33)):
        A, B = oracle.complex_schur_pencil(n, 300 + seed, dt)[:2]
        _, d, m, info = oracle.lapack_tgsna("A", A, B, None, None, job="V")
        s_, h, m2, info2 = X.tgsna("A", A, B, None, None, job="V")
        assert s_ is None and (m2, info2) == (m, info) == (n, 0)
        np.testing.assert_allclose(h, d, rtol=tol)
    dA = torch.from_numpy(np.ascontiguousarray(A.T)).cuda().t()
    dB = torch.from_numpy(np.ascontiguousarray(B.T)).cuda().t()
    d_dev, m, info = X.tgsna_dif_dev(dA, dB)
    assert (m, info) == (33, 0)
    np.testing.assert_array_equal(d_dev.cpu().numpy(), h)
