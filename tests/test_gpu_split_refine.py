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
    """Bounds from 1e-13 down to 1e-17: the same call twice gives the same refined count, the
    count never decreases as the bound shrinks, at least one bound refines some but not all
    columns, and every result matches the FP64 oracle within the split tolerance."""
    n = 400
    p = pencils.gen_gges(n, 83)
    S, P, ar, ai, be, Q, Z = p
    RL, RR, mr, infor = oracle.tgevc3("B", "B", S, P, ar, be, alphai=ai, VL=Q.copy(order="F"), VR=Z.copy(order="F"))
    counts = []
    for bound in ("1e-13", "1e-14", "1e-15", "1e-16", "1e-17"):
        monkeypatch.setenv("XTGEVC3_REFINE_BOUND", bound)
        VL, VR, m, info, refined = _run(X.SPLIT | X.SPLIT_INT8, "B", "B", p)
        assert (m, info) == (n, 0)
        again = _run(X.SPLIT | X.SPLIT_INT8, "B", "B", p)[4]
        assert again == refined, (bound, refined, again)  # the sketch is deterministic
        counts.append(refined)
        for a, b in ((VL, RL), (VR, RR)):
            err, _ = oracle.max_rel_diff(oracle.to_complex_real_storage(a, ai), oracle.to_complex_real_storage(b, ai))
            assert err < 1e-10, (bound, err)
    assert counts == sorted(counts), counts
    assert any(0 < c < 2 * n for c in counts), counts


def _rel_residuals(S, P, ar, ai, be, V):
    """Relative residual of every right eigenvector column of (S, P), both columns of a
    complex pair sharing one value: ||(b S - a P) x||_2 / ((|b| anorm + |a| bnorm) ||x||_2)
    with anorm, bnorm the largest column sums of |S|, |P| over rows <= col + 1."""
    n = S.shape[0]
    up = np.tril(np.ones((n, n), dtype=bool), 1).T  # rows <= col + 1
    anorm = np.abs(np.where(up, S, 0)).sum(0).max()
    bnorm = np.abs(np.where(up, P, 0)).sum(0).max()
    SV, PV = S @ V, P @ V
    rel = np.empty(V.shape[1])
    c = k = 0
    while k < n:
        if ai[k] == 0:
            r, x = be[k] * SV[:, c] - ar[k] * PV[:, c], V[:, c]
            w = 1
        else:  # x = v_c + i v_c+1 for (ar + i ai) / be, ai > 0 first
            a = ar[k] + 1j * ai[k]
            r = be[k] * (SV[:, c] + 1j * SV[:, c + 1]) - a * (PV[:, c] + 1j * PV[:, c + 1])
            x = V[:, c] + 1j * V[:, c + 1]
            w = 2
        den = (abs(be[k]) * anorm + abs(ar[k] + 1j * ai[k]) * bnorm) * np.linalg.norm(x)
        rel[c:c + w] = np.linalg.norm(r) / den
        c += w
        k += w
    return rel


def test_sketch_flags_track_true_residuals(cuda_ok, monkeypatch):
    """The flags come from a 16-row random sketch of each residual, so they must follow the
    true residuals: with 8 moduli the residue form leaves residuals near 1e-8 (far above
    the rounding of the sketch itself), computed here from the unrefined eigenvectors of
    (S, P).  A column is flagged when its estimate exceeds bound / 4; the estimate lies
    within a factor ~3 of the residual (chi-square spread of 16 rows), so every column with
    residual > bound must be refined and none with residual < bound / 16."""
    import torch
    n = 1100
    p = pencils.gen_gges(n, 84)
    S, P, ar, ai, be, Q, Z = p
    flags = X.SPLIT | X.SPLIT_CRT | X.slices(8)
    VR = torch.zeros((n, n), dtype=torch.float64, device="cuda").t()
    m, info = X.tgevc3_dev("R", "A", _dev(S, torch), _dev(P, torch), ar, be, alphai=ai, VR=VR,
                           flags=flags | X.SPLIT_NO_REFINE)
    assert (m, info) == (n, 0)
    V = VR.t().cpu().numpy().T[:, :m]
    rel = _rel_residuals(S, P, ar, ai, be, V)
    assert rel.max() > 1e-12, rel.max()  # well above the sketch's own rounding
    for bound in (rel.min() / 16, np.quantile(rel, 0.2), np.median(rel), np.quantile(rel, 0.8), rel.max() * 16):
        monkeypatch.setenv("XTGEVC3_REFINE_BOUND", repr(float(bound)))
        VR2 = torch.zeros((n, n), dtype=torch.float64, device="cuda").t()
        m2, info2 = X.tgevc3_dev("R", "A", _dev(S, torch), _dev(P, torch), ar, be, alphai=ai, VR=VR2, flags=flags)
        torch.cuda.synchronize()
        assert (m2, info2) == (n, 0)
        count = X.split_refined()
        lo, hi = int((rel > bound).sum()), int((rel > bound / 16).sum())
        assert lo <= count <= hi, (bound, lo, count, hi)
