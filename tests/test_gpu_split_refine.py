"""Refinement step of the split-precision forms: after the split pass every eigenvector's
residual is estimated from a random sketch, and the ones above the bound are solved again
with FP64 GEMMs (xtgevc3_split_refined() counts their columns).

* At the default bound (1e-12) no column of an xGGES pencil needs it: the split products
  are accurate to ~1e-14, so the refinement count must be 0 (a wrong residual formula would
  flag columns here).
* With the bound forced to 0 (XTGEVC3_REFINE_BOUND) every column is refined, so the result
  must equal the plain FP64 form's to rounding (1e-13 of the column max), through both the
  device entry point and the host-pointer one (whose downloads must pick up the rewritten
  columns), for HOWMNY 'B', 'A' and a selection.
* With a bound in between, some columns are refined and all stay within the split
  tolerance of the FP64 oracle.
"""
import numpy as np
import pytest

import oracle
import xtgevc3_b200 as X
from xtgevc3_b200 import pencils

pytestmark = pytest.mark.gpu

KINDS = {"bf16": 0, "int8": X.SPLIT_INT8, "crt": X.SPLIT_CRT}


def _dev(a, torch):
    return torch.from_numpy(np.ascontiguousarray(np.asarray(a).T)).cuda().t()


def _run(flags, side, howmny, p, sel=None, host=False):
    import torch
    S, P, ar, ai, be, Q, Z = p
    if host:
        X.set_flags(flags)
        try:
            VL, VR, m, info = X.tgevc3(side, howmny, S, P, ar, be, alphai=ai, VL=Q.copy(order="F"),
                                       VR=Z.copy(order="F"), select=sel)
        finally:
            X.set_flags(0)
        return VL[:, :m], VR[:, :m], m, info, X.split_refined()
    VL, VR = _dev(Q, torch), _dev(Z, torch)
    m, info = X.tgevc3_dev(side, howmny, _dev(S, torch), _dev(P, torch), ar, be, alphai=ai, VL=VL, VR=VR,
                           select=sel, flags=flags)
    torch.cuda.synchronize()
    ref = X.split_refined()
    return VL.t().cpu().numpy().T[:, :m], VR.t().cpu().numpy().T[:, :m], m, info, ref


def _colerr(A, B):
    den = np.abs(B).max(0)
    den[den == 0] = 1.0
    return float((np.abs(A - B).max(0) / den).max())


@pytest.mark.parametrize("kind", list(KINDS), ids=list(KINDS))
def test_no_refinement_needed_on_gges_pencil(cuda_ok, kind, monkeypatch):
    monkeypatch.delenv("XTGEVC3_REFINE_BOUND", raising=False)
    p = pencils.gen_gges(300, 81)
    VL, VR, m, info, refined = _run(X.SPLIT | KINDS[kind], "B", "B", p)
    assert (m, info) == (300, 0)
    assert refined == 0


@pytest.mark.parametrize("host", [False, True], ids=["device", "host"])
@pytest.mark.parametrize("howmny", ["B", "A", "S"])
def test_refining_every_column_gives_the_fp64_result(cuda_ok, monkeypatch, howmny, host):
    n = 257
    p = pencils.gen_gges(n, 82)
    sel = (np.random.default_rng(3).random(n) < 0.4).astype(np.int32) if howmny == "S" else None
    pl = _run(0, "B", howmny, p, sel, host)
    monkeypatch.setenv("XTGEVC3_REFINE_BOUND", "0")
    sp = _run(X.SPLIT | X.SPLIT_CRT, "B", howmny, p, sel, host)
    assert sp[2:4] == pl[2:4]
    assert sp[4] == sp[2] * 2  # both sides, every column
    for a, b in ((sp[0], pl[0]), (sp[1], pl[1])):
        assert _colerr(a, b) < 1e-13


def test_partial_refinement_stays_accurate(cuda_ok, monkeypatch):
    """Bounds from 1e-13 down to 1e-17: the refined count never decreases as the bound
    shrinks, at least one bound refines some but not all columns, and every result matches
    the FP64 oracle within the split tolerance."""
    n = 400
    p = pencils.gen_gges(n, 83)
    S, P, ar, ai, be, Q, Z = p
    RL, RR, mr, infor = oracle.tgevc3("B", "B", S, P, ar, be, alphai=ai, VL=Q.copy(order="F"), VR=Z.copy(order="F"))
    counts = []
    for bound in ("1e-13", "1e-14", "1e-15", "1e-16", "1e-17"):
        monkeypatch.setenv("XTGEVC3_REFINE_BOUND", bound)
        VL, VR, m, info, refined = _run(X.SPLIT | X.SPLIT_INT8, "B", "B", p)
        assert (m, info) == (n, 0)
        counts.append(refined)
        for a, b in ((VL, RL), (VR, RR)):
            err, _ = oracle.max_rel_diff(oracle.to_complex_real_storage(a, ai), oracle.to_complex_real_storage(b, ai))
            assert err < 1e-10, (bound, err)
    assert counts == sorted(counts), counts
    assert any(0 < c < 2 * n for c in counts), counts
