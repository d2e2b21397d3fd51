"""xtgevc3_{d,s,z,c}tgsna (JOB = 'E': eigenvalue condition numbers) against LAPACK xTGSNA.

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
