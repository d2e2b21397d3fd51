"""xGGES with ordering on the GPU: xtgevc3_{d,s,z,c}tgsen (IJOB = 0, the reordering kernel on
one CTA) against LAPACK D/S/Z/CTGSEN, and xtgevc3_*gges_sort (QZ, SELCTG on the host, the
reordering kernel, xGGES's SDIM check) against LAPACK xGGES with SORT = 'S'.

The reordering is checked on LAPACK's own generalized Schur forms (xGGES of iid N(0,1)
pencils) with the selections of tests/test_tgsen_host.py, where the same kernel bodies run on
host threads: complex results agree with LAPACK's to rounding, real ones up to the sign of
each column of Q and Z (see that file).  Tolerances 1e-12 (double) / 2e-4 (single) of the
matrix's largest entry.  The full xGGES with SORT = 'S' starts from our QZ step, whose Schur
form differs from LAPACK's by rounding, so it is checked by SDIM, INFO, the factorisation
residual and the set of leading eigenvalues.
"""
import numpy as np
import pytest

import oracle
import xtgevc3_b200 as X
from test_tgexc_blocks_host import _twin_blocks_pencil, sign_aligned
from test_tgsen_host import CPLX_SELECTIONS, REAL_SELECTIONS, TOL, _cplx_schur, _pencil, _real_schur, _rel

pytestmark = [pytest.mark.gpu, pytest.mark.late(3)]


@pytest.mark.parametrize("dt", [np.float64, np.float32], ids=["d", "s"])
@pytest.mark.parametrize("kind", ["neg_real", "pairs", "first_of_pair", "every_third", "none", "all"], ids=str)
def test_real_tgsen_matches_lapack(cuda_ok, dt, kind):
    S, T, Q, Z, ar, ai, be = _real_schur(30, 11, dt)
    sel = REAL_SELECTIONS[kind](ar, ai, be).astype(np.int32)
    r = oracle.lapack_tgsen0(sel, S, T, Q, Z)
    h = X.tgsen(sel, S, T, Q, Z)
    assert (h[-2], h[-1]) == (r[7], r[8]) == (r[7], 0)
    a, b, q, z = sign_aligned(h[0], h[1], h[5], h[6], r[5], r[6])
    tol = TOL[dt]
    for M, R in ((a, r[0]), (b, r[1]), (q, r[5]), (z, r[6])):
        assert _rel(M, R) < tol * 10, kind
    lam, lam_r = (h[2] + 1j * h[3]) / h[4], (r[2] + 1j * r[3]) / r[4]
    assert np.abs(lam - lam_r).max() <= tol * 10 * np.abs(lam_r).max(), kind


@pytest.mark.parametrize("dt", [np.complex128, np.complex64], ids=["z", "c"])
@pytest.mark.parametrize("kind", ["neg_real", "every_third", "none", "all", "last"], ids=str)
def test_complex_tgsen_matches_lapack(cuda_ok, dt, kind):
    S, T, Q, Z, al, be = _cplx_schur(30, 12, dt)
    sel = CPLX_SELECTIONS[kind](al, be).astype(np.int32)
    r = oracle.lapack_tgsen0(sel, S, T, Q, Z)
    h = X.tgsen(sel, S, T, Q, Z)
    assert (h[-2], h[-1]) == (r[6], r[7]) == (r[6], 0)
    tol = TOL[dt]
    for M, R in ((h[0], r[0]), (h[1], r[1]), (h[4], r[4]), (h[5], r[5])):
        assert _rel(M, R) < tol * 10, kind
    if 0 < sel.sum() < 30:
        for v, w in ((h[2], r[2]), (h[3], r[3])):
            assert _rel(v, w) < tol * 10, kind


def test_tgsen_device_form_matches_host_form(cuda_ok):
    import torch
    for dt, mk, sels, kind in ((np.float64, _real_schur, REAL_SELECTIONS, "neg_real"),
                               (np.complex128, _cplx_schur, CPLX_SELECTIONS, "every_third")):
        parts = mk(40, 13, dt)  # the pencils of test_tgsen_host.py::test_bodies_on_host_threads
        S, T, Q, Z = parts[:4]
        sel = sels[kind](*parts[4:]).astype(np.int32)
        h = X.tgsen(sel, S, T, Q, Z)
        dev = [torch.from_numpy(np.ascontiguousarray(M.T)).cuda().t() for M in (S, T, Q, Z)]
        d = X.tgsen_dev(sel, *dev)
        torch.cuda.synchronize()
        for M, R in zip(dev, (h[0], h[1], h[-4], h[-3])):
            assert np.array_equal(M.cpu().numpy(), R)
        for v, w in zip(d[:-2], h[2:-4]):
            assert np.array_equal(v.cpu().numpy(), w)
        assert (d[-2], d[-1]) == (h[-2], h[-1])


@pytest.mark.parametrize("sel", [[0, 0, 0, 0, 1, 0], [1, 0, 0, 1, 1, 0]], ids=lambda s: "".join(map(str, s)))
def test_real_tgsen_rejection(cuda_ok, sel):
    A, B, Q, Z = _twin_blocks_pencil(1)
    sel = np.array(sel, np.int32)
    r = oracle.lapack_tgsen0(sel, A, B, Q, Z)
    h = X.tgsen(sel, A, B, Q, Z)
    assert h[-1] == r[-1] == 1
    a, b, q, z = sign_aligned(h[0], h[1], h[5], h[6], r[5], r[6])
    for M, R in ((a, r[0]), (b, r[1]), (q, r[5]), (z, r[6])):
        assert _rel(M, R) < 1e-12
    for v, w in zip(h[2:5], r[2:5]):
        assert np.abs(v - w).max() < 1e-12 * max(np.abs(w).max(), 1.0)


def test_complex_tgsen_rejection(cuda_ok):
    import os
    d = np.load(os.path.join(os.path.dirname(__file__), "golden", "tgexc", "z_rejections.npz"))
    A, B = d["A1"], d["B1"]
    I = np.eye(3, dtype=np.complex128, order="F")
    sel = np.array([0, 0, 1], np.int32)
    r = oracle.lapack_tgsen0(sel, A, B, I, I)
    h = X.tgsen(sel, A, B, I, I)
    assert h[-1] == r[-1] == 1
    for M, R in ((h[0], r[0]), (h[1], r[1]), (h[4], r[4]), (h[5], r[5])):
        den = np.abs(R).max(0)
        den[den == 0] = 1.0
        assert float((np.abs(M - R).max(0) / den).max()) < 1e-12
    assert np.array_equal(h[2], np.diag(A)) and np.array_equal(h[3], np.diag(B))


@pytest.mark.parametrize("dt", [np.float64, np.float32, np.complex128, np.complex64], ids=["d", "s", "z", "c"])
@pytest.mark.late(6)  # runs the QZ kernels: after their own tests
def test_gges_sort_matches_lapack(cuda_ok, dt):
    n = 48
    A, B = _pencil(n, 31, dt)
    if np.dtype(dt).kind == "c":
        pred = lambda a, b: (a * np.conj(b)).real < 0  # noqa: E731
        S, T, al, be, VL, VR, sdim, info = X.gges(A, B, sort=pred)
        lam = al / be
        r = oracle.lapack_gges_sort(A.astype(np.complex128), B.astype(np.complex128), pred)
        lam_r = r[3] / r[4]
        assert np.all(np.diag(T).imag == 0) and np.all(np.diag(T).real >= 0)
    else:
        pred = lambda ar, ai, b: ar * b < 0  # noqa: E731
        S, T, ar, ai, be, VL, VR, sdim, info = X.gges(A, B, sort=pred)
        lam = (ar + 1j * ai) / be
        r = oracle.lapack_gges_sort(A.astype(np.float64), B.astype(np.float64), pred)
        lam_r = (r[3] + 1j * r[4]) / r[5]
    assert info == 0 and sdim == r[2] > 0
    single = dt in (np.float32, np.complex64)
    tol = 2e-4 if single else 1e-11
    scale = max(np.abs(A).max(), np.abs(B).max())
    assert np.abs(VL @ S @ VR.conj().T - A).max() < tol * n * scale
    assert np.abs(VL @ T @ VR.conj().T - B).max() < tol * n * scale
    assert np.abs(np.tril(T, -1)).max() == 0 and np.abs(np.tril(S, -2)).max() == 0
    assert np.all(pred(*(v[:sdim] for v in ((al, be) if np.dtype(dt).kind == "c" else (ar, ai, be)))))
    rt = 1e-3 if single else 1e-8
    assert np.allclose(np.sort_complex(lam[:sdim]), np.sort_complex(lam_r[:sdim]), rtol=rt)
    assert np.allclose(np.sort_complex(lam[sdim:]), np.sort_complex(lam_r[sdim:]), rtol=rt)


@pytest.mark.late(6)  # runs the QZ kernels: after their own tests
def test_gges_sort_device_form_matches_host_form(cuda_ok):
    import torch
    n = 40
    for dt in (np.float64, np.complex128):
        A, B = _pencil(n, 32, dt)
        pred = ((lambda a, b: (a * np.conj(b)).real < 0) if np.dtype(dt).kind == "c" else
                (lambda ar, ai, b: ar * b < 0))
        h = X.gges(A, B, sort=pred)
        dev = [torch.from_numpy(np.ascontiguousarray(M.T)).cuda().t() for M in (A, B)]
        VL, VR = (torch.zeros((n, n), dtype=dev[0].dtype, device="cuda").t() for _ in range(2))  # column-major
        d = X.gges_dev(dev[0], dev[1], VL, VR, sort=pred)
        torch.cuda.synchronize()
        for M, R in zip((dev[0], dev[1], VL, VR), (h[0], h[1], h[-4], h[-3])):
            assert np.array_equal(M.cpu().numpy(), R)
        for v, w in zip(d[:-2], h[2:-4]):
            assert np.array_equal(v.cpu().numpy(), w)
        assert (d[-2], d[-1]) == (h[-2], h[-1])
