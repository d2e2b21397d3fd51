"""xtgevc3_{d,s,z,c}trevc3 (the standard eigenproblem, P = I) against LAPACK xTREVC3.

The oracle is LAPACK's own xTREVC3 from SciPy's bundled OpenBLAS (the upstream project
benchmarks it beside dtgevc3 but has no implementation of its own).  The inputs are Schur
forms T, Q of iid N(0,1) matrices from LAPACK xGEES.  Columns are compared WITHOUT any
normalisation: LAPACK scales every eigenvector to max |re| + |im| = 1 and gives a real pair
a fixed phase, and the CUDA path must reproduce both.  Tolerance: the elementwise
difference relative to the column's largest entry, 1e-11 in double and 5e-4 in single
precision.
"""
import numpy as np
import pytest

import oracle
import xtgevc3_b200 as X

pytestmark = pytest.mark.gpu

TOL = {np.float64: 1e-11, np.complex128: 1e-11, np.float32: 5e-4, np.complex64: 5e-4}


def _schur(dt, n, seed):
    if np.issubdtype(dt, np.complexfloating):
        return oracle.schur_complex(n, seed, dt)
    return oracle.schur_real(n, seed, dt)


def _raw_err(V, W):
    den = np.abs(W).max(0)
    den[den == 0] = 1
    return float((np.abs(V - W).max(0) / den).max())


def _select(T, seed):
    """About a third of the eigenvalues, pairs by one of their two flags."""
    n = T.shape[0]
    sel = (np.random.default_rng(seed).random(n) < 0.33).astype(np.int32)
    return sel


CASES = [
    # (dtype, n, side, howmny)
    (np.float64, 70, "B", "A"),
    (np.float64, 300, "B", "B"),
    (np.float64, 257, "R", "S"),
    (np.float64, 200, "L", "B"),
    (np.float32, 160, "B", "B"),
    (np.complex128, 150, "B", "B"),
    (np.complex128, 131, "R", "A"),
    (np.complex64, 120, "B", "S"),
]


@pytest.mark.parametrize("case", CASES, ids=lambda c: f"{np.dtype(c[0]).name}-{c[1]}-{c[2]}{c[3]}")
def test_trevc3_matches_lapack(cuda_ok, case):
    dt, n, side, howmny = case
    T, Q = _schur(dt, n, 17 + n)
    sel = _select(T, n) if howmny == "S" else None
    VL0 = Q if howmny == "B" else None
    VR0 = Q if howmny == "B" else None
    rL, rR, rm, rinfo = oracle.lapack_trevc3(side, howmny, T, VL=VL0, VR=VR0, select=sel)
    VL, VR, m, info = X.trevc3(side, howmny, T, VL=None if VL0 is None else VL0.copy(order="F"),
                               VR=None if VR0 is None else VR0.copy(order="F"), select=sel)
    assert (m, info) == (rm, rinfo) and info == 0
    tol = TOL[dt]
    if side in ("R", "B"):
        assert np.isfinite(VR[:, :m]).all()
        assert _raw_err(VR[:, :m], rR[:, :m]) < tol
    if side in ("L", "B"):
        assert np.isfinite(VL[:, :m]).all()
        assert _raw_err(VL[:, :m], rL[:, :m]) < tol


@pytest.mark.parametrize("dt", [np.float64, np.complex128], ids=["d", "z"])
def test_trevc3_device_form_matches_host_form(cuda_ok, dt):
    """xtgevc3_{d,z}trevc3_dev on device-resident T, Q gives the host form's columns."""
    import torch
    n = 260
    T, Q = _schur(dt, n, 5)
    VL, VR, m, info = X.trevc3("B", "B", T, VL=Q.copy(order="F"), VR=Q.copy(order="F"))
    assert info == 0

    def dev(a):
        return torch.from_numpy(np.ascontiguousarray(a.T)).cuda().t()

    dVL, dVR = dev(Q), dev(Q)
    m2, info2 = X.trevc3_dev("B", "B", dev(T), VL=dVL, VR=dVR)
    torch.cuda.synchronize()
    assert (m2, info2) == (m, 0)
    assert _raw_err(dVL.cpu().numpy(), VL) < 1e-13
    assert _raw_err(dVR.cpu().numpy(), VR) < 1e-13


def test_trevc3_large_real_schur_matches_lapack(cuda_ok):
    """n = 1024 real Schur form, both sides, back-transformed: the grouped updates skip
    the identity's strips, the pairs get LAPACK's phase, and every column matches."""
    n = 1024
    T, Q = _schur(np.float64, n, 1024)
    rL, rR, rm, _ = oracle.lapack_trevc3("B", "B", T, VL=Q, VR=Q)
    VL, VR, m, info = X.trevc3("B", "B", T, VL=Q.copy(order="F"), VR=Q.copy(order="F"))
    assert (m, info) == (rm, 0)
    assert _raw_err(VR, rR) < 1e-10
    assert _raw_err(VL, rL) < 1e-10


@pytest.mark.parametrize("n", [1, 2, 3, 64, 65])
@pytest.mark.parametrize("dt", [np.float64, np.complex128], ids=["d", "z"])
def test_trevc3_small_and_block_boundary_orders(cuda_ok, dt, n):
    """Orders 1-3 (a real 2x2 block can be the whole matrix) and the 64-row block boundary,
    both sides, back-transformed, against LAPACK without normalisation."""
    found = None
    for seed in range(40):  # for n = 2 real, a seed whose Schur form is one 2x2 block
        T, Q = _schur(dt, n, seed)
        if dt != np.float64 or n != 2 or T[1, 0] != 0:
            found = (T, Q)
            break
    T, Q = found
    rL, rR, rm, _ = oracle.lapack_trevc3("B", "B", T, VL=Q, VR=Q)
    VL, VR, m, info = X.trevc3("B", "B", T, VL=Q.copy(order="F"), VR=Q.copy(order="F"))
    assert (m, info) == (rm, 0)
    assert _raw_err(VR, rR) < 1e-11 and _raw_err(VL, rL) < 1e-11


def test_trevc3_empty_selection(cuda_ok):
    """HOWMNY='S' with nothing selected: M = 0, INFO = 0, outputs untouched."""
    T, Q = _schur(np.float64, 50, 2)
    VR = np.full((50, 4), 7.0, order="F")
    _, VR2, m, info = X.trevc3("R", "S", T, VR=VR, select=np.zeros(50, dtype=np.int32), mm=4)
    assert (m, info) == (0, 0) and (VR2 == 7.0).all()


def test_trevc3_host_pieces_match_device_form(cuda_ok):
    """n = 1100: the host-pointer form uploads T in three pieces while the solve runs (P = I is
    built on the device, bnorm = 1 comes from the host with anorm), and its columns equal the
    device form's bit for bit."""
    import torch
    n = 1100
    T, Q = _schur(np.float64, n, 1100)
    VL, VR, m, info = X.trevc3("B", "B", T, VL=Q.copy(order="F"), VR=Q.copy(order="F"))
    assert (m, info) == (n, 0)

    def dev(a):
        return torch.from_numpy(np.ascontiguousarray(a.T)).cuda().t()

    dVL, dVR = dev(Q), dev(Q)
    m2, info2 = X.trevc3_dev("B", "B", dev(T), VL=dVL, VR=dVR)
    torch.cuda.synchronize()
    assert (m2, info2) == (m, 0)
    np.testing.assert_array_equal(dVL.cpu().numpy(), VL)
    np.testing.assert_array_equal(dVR.cpu().numpy(), VR)
