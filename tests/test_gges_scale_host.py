"""xGGES's scaling of badly scaled pencils (xtgevc3_b200/csrc/gges_scale.h, used by
xtgevc3_*gges*): xLASCL's factors bit for bit against LAPACK's own DLASCL, and the whole flow of
xGGES on host arrays (the scale decision, the pencil scaled into range, the QZ kernel bodies
of tests/qz_host.cpp, DGGES's guard of complex pairs, the Schur form and eigenvalues scaled
back) against LAPACK xGGES on pencils with entries near 1e+-200, where the unscaled QZ step
would overflow or underflow: the same eigenvalues (relative 1e-9), A = Q S Z^H, B = Q T Z^H to
1e-12 n of their scale, finite everything."""
import ctypes as ct

import numpy as np
import pytest
import scipy.linalg.lapack as la

import oracle
from test_qz_host import _p, host, host_qz, host_rqz  # noqa: F401  (fixture)


@pytest.mark.parametrize("cf,ct_", [(1e300, 1e-300), (1e-300, 1e300), (3.0, 7.0), (1e200, 1.5e138), (1e-200, 6.7e-139),
                                    (np.inf, 1.0), (1.0, 0.0), (2.0, 2.0), (1e308, 1e-308), (5e-324, 1.0)])
def test_lascl_steps_match_lapack(host, cf, ct_):
    x = np.random.default_rng(0).standard_normal(50) * 1e-3
    y, z = x.copy(), x.copy()
    iv = lambda v: ct.byref(ct.c_int(v))  # noqa: E731
    info = ct.c_int(0)
    oracle._openblas().scipy_dlascl_(ct.c_char_p(b"G"), iv(0), iv(0), ct.byref(ct.c_double(cf)),
                                     ct.byref(ct.c_double(ct_)), iv(50), iv(1), _p(y), iv(50), ct.byref(info),
                                     ct.c_size_t(1))
    host.host_dlascl(ct.c_double(cf), ct.c_double(ct_), 50, _p(z))
    assert np.array_equal(y, z, equal_nan=True)


def _flow(host, A, B, cplx):
    """xGGES's flow on the host: returns (S, T, Q, Z, eigenvalue arrays...)"""
    n = A.shape[0]
    A, B = np.array(A, order="F"), np.array(B, order="F")
    to = ct.c_double(0)
    g = {}
    for name, M in (("a", A), ("b", B)):
        nrm = float(np.abs(M).max())
        sc = host.host_gges_needs_scaling(ct.c_double(nrm), ct.byref(to))
        g[name] = (sc, nrm, to.value)
        if sc:
            flat = M.reshape(-1, order="F").view(np.float64)
            host.host_dlascl(ct.c_double(nrm), ct.c_double(to.value), flat.size, _p(flat))
    if cplx:
        S, T, Q, Z, info = host_qz(host, A, B)
        ev = [np.diag(S).copy(), np.diag(T).copy(), np.zeros(1)]
    else:
        S, T, Q, Z, ar, ai, be, info = host_rqz(host, A, B)
        ev = [ar.copy(), ai.copy(), be.copy()]
    assert info == 0
    host.host_gges_scale_out(int(cplx), n, _p(S), _p(T), _p(ev[0]), _p(ev[1]), _p(ev[2]), g["a"][0],
                             ct.c_double(g["a"][1]), ct.c_double(g["a"][2]), g["b"][0], ct.c_double(g["b"][1]),
                             ct.c_double(g["b"][2]))
    return S, T, Q, Z, ev, (g["a"][0], g["b"][0])


@pytest.mark.parametrize("sa,sb", [(1e200, 1.0), (1e-200, 1.0), (1.0, 1e200), (1e200, 1e-200), (1.0, 1.0)],
                         ids=["A_huge", "A_tiny", "B_huge", "both", "none"])
@pytest.mark.parametrize("cplx", [False, True], ids=["d", "z"])
def test_scaled_flow_matches_lapack_gges(host, sa, sb, cplx):
    n = 24
    rng = np.random.default_rng(9)
    A0, B0 = rng.standard_normal((n, n)), rng.standard_normal((n, n))
    if cplx:
        A0, B0 = A0 + 1j * rng.standard_normal((n, n)), B0 + 1j * rng.standard_normal((n, n))
    A, B = A0 * sa, B0 * sb
    S, T, Q, Z, ev, scaled = _flow(host, A, B, cplx)
    assert scaled == ((sa != 1.0), (sb != 1.0))
    if cplx:  # eigenvalues of the unscaled pencil (A0, B0): (alpha / sa) / (beta / sb), no overflow
        r = la.zgges(lambda a, b: 0, A, B)
        lam, lam_r = (ev[0] / sa) / (ev[1] / sb), (r[3] / sa) / (r[4] / sb)
    else:
        r = la.dgges(lambda x, y, z: 0, A, B)
        lam = ((ev[0] + 1j * ev[1]) / sa) / (ev[2] / sb)
        lam_r = ((r[3] + 1j * r[4]) / sa) / (r[5] / sb)
    for M in (S, T, Q, Z, *ev):
        assert np.all(np.isfinite(M))
    for x, y in ((lam, lam_r), (lam_r, lam)):  # each eigenvalue's nearest in the other set
        d = np.abs(x[:, None] - y[None, :]).min(1) / np.abs(x)
        assert d.max() <= 1e-9, d.max()
    for M, M0, sc in ((S, A, sa), (T, B, sb)):
        assert np.abs(Q @ M @ Z.conj().T - M0).max() <= 1e-12 * n * np.abs(M0).max()
        assert 0.1 < np.abs(M).max() / (sc * np.abs(M0 / sc).max()) < 10  # in the input's own scale
