"""xtgevc3_dtgevc3_dev_noalloc -- the entry point for callers that cannot allocate device
memory -- against the regular device entry point xtgevc3_dtgevc3_dev.

Both are called through the C ABI on the same inputs; the allocation-free one takes its
scratch from the 8 MiB block inside the library instead of the CUDA memory pool.  Two
calls in a row (different sizes, the second smaller, so anything left in the shared block
by the first call would show), each compared column by column within the tolerance the
parity tests use for xGGES pencils (1e-11 of the column max), and the first also against
the CPU oracle.  The largest accepted order (SIDE='B', HOWMNY='B', n = 478) runs and
matches; one more (n = 479) and larger problems are refused with return code 2 before any
device work.
"""
import oracle
import ctypes as ct

import numpy as np
import pytest

import xtgevc3_b200 as X
from xtgevc3_b200 import pencils

pytestmark = pytest.mark.gpu

TOL = 1e-11


def _colmajor(a, torch):
    return torch.from_numpy(np.ascontiguousarray(a.T)).cuda().t()


def _noalloc(torch, side, howmny, S, P, ar, ai, be, VL, VR, select=None, n=None, mm=None):
    lib = X.lib()
    m = ct.c_int(0)
    info = ct.c_int(0)
    sel = None if select is None else np.ascontiguousarray(select, dtype=np.int32)
    keep = [np.ascontiguousarray(v, dtype=np.float64) for v in (ar, ai, be)]
    p = [v.ctypes.data_as(ct.c_void_p) for v in keep]
    rc = lib.xtgevc3_dtgevc3_dev_noalloc(
        ct.c_void_p(torch.cuda.current_stream().cuda_stream), side.encode(), howmny.encode(),
        None if sel is None else sel.ctypes.data_as(ct.c_void_p), S.shape[0] if n is None else n,
        ct.c_void_p(S.data_ptr()), S.stride(1), ct.c_void_p(P.data_ptr()), P.stride(1), p[0], p[1], p[2],
        ct.c_void_p(VL.data_ptr()), VL.stride(1), ct.c_void_p(VR.data_ptr()), VR.stride(1), VR.shape[1] if mm is None else mm,
        ct.byref(m), ct.byref(info))
    torch.cuda.synchronize()
    return rc, m.value, info.value


def _max_col_err(A, B):
    den = np.abs(B).max(0)
    den[den == 0] = 1.0
    return float((np.abs(A - B).max(0) / den).max())


def _check_case(torch, n, seed, side, howmny, sel, against_oracle):
    S, P, ar, ai, be, Q, Z = pencils.gen_gges(n, seed)
    dS, dP = _colmajor(S, torch), _colmajor(P, torch)
    VL1, VR1 = _colmajor(Q, torch), _colmajor(Z, torch)
    m1, info1 = X.tgevc3_dev(side, howmny, dS, dP, ar, be, alphai=ai, VL=VL1, VR=VR1, select=sel)
    torch.cuda.synchronize()
    VL2, VR2 = _colmajor(Q, torch), _colmajor(Z, torch)
    rc, m2, info2 = _noalloc(torch, side, howmny, dS, dP, ar, ai, be, VL2, VR2, select=sel)
    assert rc == 0, X.last_error()
    assert (m2, info2) == (m1, info1) and info2 == 0
    if against_oracle:
        RL, RR, mr, infor = oracle.tgevc3(side, howmny, S, P, ar, be, alphai=ai, VL=Q.copy(order="F"),
                                          VR=Z.copy(order="F"), select=sel)
        assert (mr, infor) == (m2, 0)
    for k, (A, B) in enumerate(((VL2, VL1), (VR2, VR1))):
        a = A.t().cpu().numpy().T[:, :m2]
        b = B.t().cpu().numpy().T[:, :m1]
        assert np.isfinite(a).all()
        assert _max_col_err(a, b) <= TOL
        if against_oracle:
            R = (RL, RR)[k][:, :m2]
            err, _ = oracle.max_rel_diff(oracle.to_complex_real_storage(a, ai, howmny, sel),
                                         oracle.to_complex_real_storage(R, ai, howmny, sel))
            assert err <= TOL, err


def test_noalloc_matches_regular_entry_point_twice(cuda_ok):
    import torch
    rng = np.random.default_rng(5)
    _check_case(torch, 300, 61, "B", "B", None, against_oracle=True)
    _check_case(torch, 170, 62, "B", "S", (rng.random(170) < 0.4).astype(np.int32), against_oracle=False)


def test_noalloc_largest_accepted_order(cuda_ok):
    import torch
    # n = 478 is the largest SIDE='B', HOWMNY='B' problem whose scratch fits the block
    _check_case(torch, 478, 63, "B", "B", None, against_oracle=False)


def test_noalloc_refuses_problems_larger_than_its_scratch(cuda_ok):
    import torch
    dummy = torch.zeros(1, 1, dtype=torch.float64, device="cuda")
    # n = 479 is one more than the largest accepted SIDE='B', HOWMNY='B' order; 600 is well past it
    for n in (479, 600):
        z = np.zeros(n)
        rc, m, info = _noalloc(torch, "B", "B", dummy, dummy, z, z, np.ones(n), dummy, dummy, n=n, mm=n)
        assert rc == 2
        assert "static scratch" in X.last_error() and "n <= 478" in X.last_error()
        assert m == n and info == 0
