"""xtgevc3_d/s/z/ctgsyl (TRANS = 'N', IJOB 0, 1, 3; one CTA) against LAPACK xTGSYL, and
xtgevc3_dtgsen / ztgsen's estimates (IJOB 1, 2, 4: PL, PR, DIF) against LAPACK xTGSEN, on the
GPU.

Inputs and tolerances as in tests/test_tgsyl_host.py, where the same kernel bodies run on host
threads: R, L, SCALE and the DIF estimate of xTGSYL within 1e-11 (double) / 2e-3 (single) of
LAPACK's; PL and PR within 1e-9; xTGSEN's DIF within a factor of 2 (it depends on the column
signs that the real 2x2 swaps choose on rounding-level quantities, as LAPACK's do); complex
PL, PR, DIF within 1e-10 of LAPACK's.
"""
import numpy as np
import pytest

import oracle
import xtgevc3_b200 as X
from test_tgsen_host import REAL_SELECTIONS, _real_schur
from test_tgsyl_host import _schur, sylv_operands

pytestmark = [pytest.mark.gpu, pytest.mark.late(2)]


@pytest.mark.parametrize("dt", [np.float64, np.float32], ids=["d", "s"])
@pytest.mark.parametrize("mn", [(1, 1), (2, 2), (1, 5), (5, 1), (3, 4), (20, 13), (41, 17)],
                         ids=lambda t: f"{t[0]}x{t[1]}")
def test_tgsyl_matches_lapack(cuda_ok, dt, mn):
    m, n = mn
    tol = 1e-11 if dt == np.float64 else 2e-3
    A, D = _schur(m, 0, dt)
    B, E = _schur(n, 100, dt)
    g = np.random.default_rng(7)
    C, F = (np.asfortranarray(g.standard_normal((m, n)).astype(dt)) for _ in range(2))
    for ijob in (0, 1, 3):
        rR, rL, rs, rd, ri = oracle.lapack_tgsyl("N", ijob, A, B, C, D, E, F)
        hR, hL, hs, hd, hi = X.tgsyl(ijob, A, B, C, D, E, F)
        assert (hi, hs) == (ri, rs), (ijob, hi, ri, hs, rs)
        if ijob != 3:
            for M, R in ((hR, rR), (hL, rL)):
                assert np.abs(M - R).max() <= tol * max(np.abs(R).max(), 1.0), ijob
        if ijob != 0:
            assert abs(hd - rd) <= tol * abs(rd), (ijob, hd, rd)


def test_tgsyl_scales_against_overflow(cuda_ok):
    A, D = _schur(6, 4)
    B, E = _schur(5, 5)
    A[np.diag_indices(6)] *= 1e-6
    D[np.diag_indices(6)] *= 1e-6
    g = np.random.default_rng(6)
    C, F = (np.asfortranarray(g.standard_normal((6, 5)) * 1e305) for _ in range(2))
    rR, rL, rs, _, ri = oracle.lapack_tgsyl("N", 0, A, B, C, D, E, F)
    hR, hL, hs, _, hi = X.tgsyl(0, A, B, C, D, E, F)
    assert rs < 1 and hi == ri and abs(hs - rs) <= 1e-12 * rs
    for M, R in ((hR, rR), (hL, rL)):
        assert np.all(np.isfinite(M)) and np.abs(M - R).max() <= 1e-10 * np.abs(R).max()


@pytest.mark.parametrize("kind", ["neg_real", "pairs", "every_third", "none"], ids=str)
def test_tgsen_estimates_match_lapack(cuda_ok, kind):
    import scipy.linalg.lapack as la
    n = 30
    S, T, Q, Z, ar, ai, be = _real_schur(n, 11, np.float64)
    sel = REAL_SELECTIONS[kind](ar, ai, be).astype(np.int32)
    r = la.dtgsen(sel, S, T, Q, Z, ijob=4, lwork=n * n + 64, liwork=n * n + 64)
    h = X.tgsen(sel, S, T, Q, Z, ijob=4)
    m, pl, pr, dif, info = h[-5:]
    assert (m, info) == (r[7], r[11]) == (r[7], 0)
    assert abs(pl - r[8]) <= 1e-9 * r[8] and abs(pr - r[9]) <= 1e-9 * r[9]
    if 0 < m < n:
        assert np.all(dif <= 2 * r[10]) and np.all(dif >= r[10] / 2), (dif, r[10])
    else:
        assert np.allclose(dif, r[10], rtol=1e-12)


def test_tgsen_estimates_device_form_matches_host_form(cuda_ok):
    import torch
    S, T, Q, Z, ar, ai, be = _real_schur(30, 11, np.float64)
    sel = REAL_SELECTIONS["neg_real"](ar, ai, be).astype(np.int32)
    h = X.tgsen(sel, S, T, Q, Z, ijob=4)
    dev = [torch.from_numpy(np.ascontiguousarray(M.T)).cuda().t() for M in (S, T, Q, Z)]
    d = X.tgsen_dev(sel, *dev, ijob=4)
    torch.cuda.synchronize()
    for M, R in zip(dev, (h[0], h[1], h[5], h[6])):
        assert np.array_equal(M.cpu().numpy(), R)
    assert (d[3], d[4], d[5], d[7]) == (h[7], h[8], h[9], h[11]) and np.array_equal(d[6], h[10])


@pytest.mark.parametrize("dt", [np.complex128, np.complex64], ids=["z", "c"])
@pytest.mark.parametrize("mn", [(1, 1), (2, 2), (1, 5), (3, 4), (20, 13), (41, 17)], ids=lambda t: f"{t[0]}x{t[1]}")
def test_complex_tgsyl_matches_lapack(cuda_ok, dt, mn):
    m, n = mn
    tol = 1e-11 if dt == np.complex128 else 2e-3
    A, B, C, D, E, F = sylv_operands(m, n, 0, dt)
    for ijob in (0, 1, 3):
        rR, rL, rs, rd, ri = oracle.lapack_tgsyl("N", ijob, A, B, C, D, E, F)
        hR, hL, hs, hd, hi = X.tgsyl(ijob, A, B, C, D, E, F)
        assert (hi, hs) == (ri, rs), (ijob, hi, ri, hs, rs)
        if ijob != 3:
            for M, R in ((hR, rR), (hL, rL)):
                assert np.abs(M - R).max() <= tol * max(np.abs(R).max(), 1.0), ijob
        if ijob != 0:
            assert abs(hd - rd) <= tol * abs(rd), (ijob, hd, rd)


@pytest.mark.parametrize("kind", ["neg_real", "every_third", "none", "last"], ids=str)
def test_complex_tgsen_estimates_match_lapack(cuda_ok, kind):
    import scipy.linalg.lapack as la
    from test_tgsen_host import CPLX_SELECTIONS, _cplx_schur
    n = 30
    S, T, Q, Z, al, be = _cplx_schur(n, 12, np.complex128)
    sel = CPLX_SELECTIONS[kind](al, be).astype(np.int32)
    r = la.ztgsen(sel, S, T, Q, Z, ijob=4, lwork=2 * n * n + 64, liwork=2 * n * n + 64)
    h = X.tgsen(sel, S, T, Q, Z, ijob=4)
    m, pl, pr, dif, info = h[-5:]
    assert (m, info) == (r[6], r[10]) == (r[6], 0)
    assert abs(pl - r[7]) <= 1e-10 * r[7] and abs(pr - r[8]) <= 1e-10 * r[8]
    assert np.all(np.abs(dif - r[9]) <= 1e-10 * r[9]), (dif, r[9])
    for M, R in ((h[0], r[0]), (h[1], r[1]), (h[4], r[4]), (h[5], r[5])):
        assert np.abs(M - R).max() <= 1e-11 * max(np.abs(R).max(), 1.0)


@pytest.mark.parametrize("dt", [np.float64, np.float32], ids=["d", "s"])
@pytest.mark.parametrize("mn", [(1, 1), (2, 2), (5, 1), (3, 4), (20, 13), (41, 17)], ids=lambda t: f"{t[0]}x{t[1]}")
def test_tgsyl_transposed_matches_lapack(cuda_ok, dt, mn):
    m, n = mn
    tol = 1e-11 if dt == np.float64 else 2e-3
    A, B, C, D, E, F = sylv_operands(m, n, 0, dt)
    rR, rL, rs, _, ri = oracle.lapack_tgsyl("T", 0, A, B, C, D, E, F)
    hR, hL, hs, _, hi = X.tgsyl(0, A, B, C, D, E, F, trans="T")
    assert (hi, hs) == (ri, rs)
    for M, R in ((hR, rR), (hL, rL)):
        assert np.abs(M - R).max() <= tol * max(np.abs(R).max(), 1.0)


@pytest.mark.parametrize("ijob", [3, 5])
def test_tgsen_one_norm_estimates(cuda_ok, ijob):
    """On LAPACK's reordered pencil with its leading M rows selected (no swaps on either side):
    PL, PR, DIF(1:2) within 1e-10 of LAPACK's; on the full call DIF within a factor 3."""
    import scipy.linalg.lapack as la
    n = 30
    S, T, Q, Z, ar, ai, be = _real_schur(n, 11, np.float64)
    lw = 2 * n * n + 64
    sel = REAL_SELECTIONS["neg_real"](ar, ai, be).astype(np.int32)
    r = la.dtgsen(sel, S, T, Q, Z, ijob=ijob, lwork=lw, liwork=lw)
    h = X.tgsen(sel, S, T, Q, Z, ijob=ijob)
    assert (h[7], h[11]) == (r[7], r[11])
    assert np.all(h[10] <= 3 * r[10]) and np.all(h[10] >= r[10] / 3)
    r0 = la.dtgsen(sel, S, T, Q, Z, ijob=0, lwork=lw, liwork=lw)
    m = r0[7]
    A, B, Q2, Z2 = (np.asfortranarray(x) for x in (r0[0], r0[1], r0[5], r0[6]))
    sel2 = np.zeros(n, np.int32)
    sel2[:m] = 1
    rr = la.dtgsen(sel2, A, B, Q2, Z2, ijob=ijob, lwork=lw, liwork=lw)
    h = X.tgsen(sel2, A, B, Q2, Z2, ijob=ijob)
    assert np.all(np.abs(h[10] - rr[10]) <= 1e-10 * rr[10]), (h[10], rr[10])
    if ijob == 5:
        assert abs(h[8] - rr[8]) <= 1e-10 * rr[8] and abs(h[9] - rr[9]) <= 1e-10 * rr[9]


@pytest.mark.parametrize("dt", [np.complex128, np.complex64], ids=["z", "c"])
@pytest.mark.parametrize("mn", [(1, 1), (2, 2), (5, 1), (3, 4), (20, 13), (41, 17)], ids=lambda t: f"{t[0]}x{t[1]}")
def test_complex_tgsyl_conjugate_transposed_matches_lapack(cuda_ok, dt, mn):
    m, n = mn
    tol = 1e-11 if dt == np.complex128 else 2e-3
    A, B, C, D, E, F = sylv_operands(m, n, 0, dt)
    rR, rL, rs, _, ri = oracle.lapack_tgsyl("C", 0, A, B, C, D, E, F)
    hR, hL, hs, _, hi = X.tgsyl(0, A, B, C, D, E, F, trans="C")
    assert (hi, hs) == (ri, rs)
    for M, R in ((hR, rR), (hL, rL)):
        assert np.abs(M - R).max() <= tol * max(np.abs(R).max(), 1.0)


@pytest.mark.parametrize("ijob", [3, 5])
def test_complex_tgsen_one_norm_estimates(cuda_ok, ijob):
    """PL, PR (IJOB 5) and DIF(1) within 1e-10 of LAPACK ZTGSEN's; DIF(2) within a factor 3 of
    the host build's bound (LAPACK's own DIF(2) is not reproducible; tests/test_tgsyl_host.py)."""
    import scipy.linalg.lapack as la
    from test_tgsen_host import CPLX_SELECTIONS, _cplx_schur
    n = 30
    S, T, Q, Z, al, be = _cplx_schur(n, 12, np.complex128)
    sel = CPLX_SELECTIONS["neg_real"](al, be).astype(np.int32)
    r = la.ztgsen(sel, S, T, Q, Z, ijob=ijob, lwork=2 * n * n + 64, liwork=2 * n * n + 64)
    h = X.tgsen(sel, S, T, Q, Z, ijob=ijob)
    m, pl, pr, dif, info = h[-5:]
    assert (m, info) == (r[6], r[10]) == (r[6], 0)
    assert abs(dif[0] - r[9][0]) <= 1e-10 * r[9][0]
    if ijob == 5:
        assert abs(pl - r[7]) <= 1e-10 * r[7] and abs(pr - r[8]) <= 1e-10 * r[8]
    assert np.isfinite(dif[1]) and dif[1] > 0
