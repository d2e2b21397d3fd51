"""The CPU oracle (oracle/tgevc3_oracle.c) against the upstream library's own outputs.

The fixtures in tests/golden/ were produced by the upstream src/*.cpp (see
tests/golden/make_golden.py).  The oracle follows the same algorithm (same 32-column
panels, same whole-panel overflow guards), so its raw outputs must agree column by
column up to rounding: BLAS summation order is the only difference.
"""
import numpy as np
import pytest

import oracle
from conftest import golden_files, load_golden

# per-column max |oracle - upstream| / max |upstream|, raw (no normalisation)
TOL = {np.float64: 1e-11, np.complex128: 1e-11, np.float32: 5e-5, np.complex64: 5e-5}


@pytest.mark.parametrize("path", golden_files(), ids=lambda p: p.split("/")[-1][:-4])
def test_oracle_matches_upstream(path):
    d = load_golden(path)
    VL, VR, m, info = oracle.tgevc3(d["side"], d["howmny"], d["S"], d["P"], d["alpha"], d["beta"],
                                    alphai=d.get("alphai"), VL=d["VL_in"].copy(order="F"),
                                    VR=d["VR_in"].copy(order="F"), select=d.get("select"), impl="oracle")
    assert (m, info) == (d["m"], d["info"])
    tol = TOL[d["S"].dtype.type]
    for side, V, Vr in (("L", VL, d["VL_out"]), ("R", VR, d["VR_out"])):
        if side not in d["side"] and d["side"] != "B":
            continue
        V, Vr = V[:, :m], Vr[:, :m]
        assert np.isfinite(Vr).all()
        den = np.abs(Vr).max(0)
        den[den == 0] = 1
        err = np.abs(V - Vr).max(0) / den
        assert err.max() <= tol, (side, err.max())


def _real_pencil_residuals(d, VL, VR, m):
    ai = d["alphai"]
    alpha = d["alpha"] + 1j * ai
    out = []
    for left, V in ((True, VL), (False, VR)):
        Vc = oracle.to_complex_real_storage(V[:, :m], ai)
        out.append(oracle.residual_ratio(d["S"], d["P"], Vc, alpha, d["beta"], left=left).max())
    return out


def test_oracle_residual_bound_gges():
    """DGET52-style residual (tests/test_lapack_d.cpp:38-168) below the upstream warning level."""
    from xtgevc3_b200 import pencils
    S, P, ar, ai, be, Q, Z = pencils.gen_gges(96, 11)
    VL, VR, m, info = oracle.tgevc3("B", "A", S, P, ar, be, alphai=ai)
    assert info == 0 and m == 96
    d = dict(S=S, P=P, alpha=ar, alphai=ai, beta=be)
    rl, rr = _real_pencil_residuals(d, VL, VR, m)
    assert rl < 100 and rr < 100


def test_oracle_matches_lapack_tgevc():
    """Second oracle: LAPACK xTGEVC on the same pencil, compared after normalisation."""
    from xtgevc3_b200 import pencils
    S, P, ar, ai, be, Q, Z = pencils.gen_gges(80, 12)
    VL, VR, m, info = oracle.tgevc3("B", "A", S, P, ar, be, alphai=ai)
    vl_lap, vr_lap = oracle.lapack_tgevc(S, P)
    for V, W in ((VL, vl_lap), (VR, vr_lap)):
        a = oracle.to_complex_real_storage(V, ai)
        b = oracle.to_complex_real_storage(W, ai)
        err, _ = oracle.max_rel_diff(a, b)
        assert err < 1e-10


def test_oracle_lwork_and_info():
    from xtgevc3_b200 import pencils
    S, P, ar, ai, be = pencils.gen_quasi_triangular(20, 0)
    # bad HOWMNY
    _, _, m, info = oracle.tgevc3("B", "X", S, P, ar, be, alphai=ai)
    assert info == -2
    # MM too small
    _, _, m, info = oracle.tgevc3("B", "A", S, P, ar, be, alphai=ai, mm=5)
    assert info == -16 and m == 20
    # LWORK too small even for block size 1
    _, _, m, info = oracle.tgevc3("B", "A", S, P, ar, be, alphai=ai, lwork=10)
    assert info == -19


@pytest.mark.skipif(not oracle.ref_available(), reason="upstream library not built (oracle/Makefile ref)")
@pytest.mark.parametrize("prec", ["d", "z"])
def test_oracle_matches_upstream_library_with_many_guards(prec):
    """n = 2048 random triangular pencils (upstream test-generator structure) on which the
    overflow guards rescale hundreds of columns: the oracle against the upstream library
    built from its sources, SIDE='R'.  Guard scale factors are computed from maxima that
    differ in rounding, so the columns are compared after normalisation (1e-11)."""
    from xtgevc3_b200 import pencils
    if prec == "d":
        S, P, al, ai, be = pencils.gen_quasi_triangular(2048, 8213)
    else:
        (S, P, al, be), ai = pencils.gen_upper_triangular_complex(2048, 8213), None
    o = oracle.tgevc3("R", "A", S, P, al, be, alphai=ai, impl="oracle")[1]
    r = oracle.tgevc3("R", "A", S, P, al, be, alphai=ai, impl="ref")[1]
    assert np.isfinite(o).all() and np.isfinite(r).all()
    if ai is not None:
        o, r = oracle.to_complex_real_storage(o, ai), oracle.to_complex_real_storage(r, ai)
    err, _ = oracle.max_rel_diff(o, r)
    assert err < 1e-11, err


@pytest.mark.parametrize("dt", [np.float64, np.complex128])
def test_lapack_trevc3_oracle_residual(dt):
    """The xTREVC3 oracle (LAPACK through SciPy's OpenBLAS) on a Schur form A = Q T Q^H:
    the back-transformed eigenvectors satisfy A v = w v to a few eps (w from T's diagonal
    blocks), and every column is normalised to max |re| + |im| = 1."""
    n = 80
    T, Q = (oracle.schur_real if dt == np.float64 else oracle.schur_complex)(n, 3, dt)
    VL, VR, m, info = oracle.lapack_trevc3("B", "B", T, VL=Q, VR=Q)
    assert (m, info) == (n, 0)
    A = Q @ T @ Q.conj().T
    w = np.diag(T).astype(np.complex128)
    ai = np.zeros(n)
    if dt == np.float64:
        k = 0
        while k < n:
            if k + 1 < n and T[k + 1, k] != 0:
                wi = np.sqrt(abs(T[k, k + 1])) * np.sqrt(abs(T[k + 1, k]))
                w[k], w[k + 1] = T[k, k] + 1j * wi, T[k, k] - 1j * wi
                ai[k], ai[k + 1] = wi, -wi
                k += 2
            else:
                k += 1
        V = oracle.to_complex_real_storage(VR, ai)
        U = oracle.to_complex_real_storage(VL, ai)
    else:
        V, U = VR, VL
    eps = np.finfo(np.float64).eps
    nA = np.abs(A).sum(0).max()
    r = np.abs(A @ V - V * w[None, :]).sum(0) / (nA * np.abs(V).sum(0)) / eps
    assert r.max() < 100, r.max()
    rl = np.abs(A.conj().T @ U - U * np.conj(w)[None, :]).sum(0) / (nA * np.abs(U).sum(0)) / eps
    assert rl.max() < 100, rl.max()
    mags = np.abs(VR.real) + np.abs(VR.imag) if dt == np.complex128 else None
    if mags is not None:
        assert np.allclose(mags.max(0), 1.0)
