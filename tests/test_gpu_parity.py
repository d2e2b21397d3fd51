"""CUDA path (libxtgevc3.so through its C ABI) against the upstream outputs and the oracle.

Tolerances (stated per test): after both sides are scaled by the reference's value at the
reference's largest component (``oracle.normalize_like``), the elementwise difference
relative to the column max must be below TOL; the DGET52-style residual of
tests/test_lapack_d.cpp:38-168 (in units of eps) must be below 100, the upstream warning
level.  Eigenvectors of the random triangular pencils of the upstream self-tests are
ill-conditioned (components spread over many orders of magnitude), so those cases get a
looser elementwise bound than the xGGES pencils.
"""
import numpy as np
import pytest

import oracle
import xtgevc3_b200 as X
from conftest import golden_files, load_golden
from xtgevc3_b200 import pencils

pytestmark = pytest.mark.gpu

TOL_WELL = {np.float64: 1e-11, np.complex128: 1e-11, np.float32: 2e-4, np.complex64: 2e-4}
TOL_ILL = {np.float64: 1e-8, np.complex128: 1e-8, np.float32: 5e-3, np.complex64: 5e-3}


def as_complex(V, d):
    if d.get("alphai") is not None and np.isrealobj(V):
        return oracle.to_complex_real_storage(V, d["alphai"], d["howmny"], d.get("select"))
    return V.astype(np.complex128)


def compare(d, VL, VR, m, VLr, VRr, tol, check_resid=True):
    howmny = d["howmny"]
    for side, V, Vr in (("L", VL, VLr), ("R", VR, VRr)):
        if d["side"] not in (side, "B"):
            continue
        V, Vr = V[:, :m], Vr[:, :m]
        a, b = as_complex(V, d), as_complex(Vr, d)
        err, cols = oracle.max_rel_diff(a, b)
        assert err <= tol, (side, err, int(np.nanargmax(cols)))
        if check_resid and howmny in ("A", "S"):
            al, be = oracle.column_eigenvalues(d["alpha"], d["beta"], howmny, d.get("select"), d.get("alphai"))
            r = oracle.residual_ratio(d["S"], d["P"], a, al, be, left=(side == "L"))
            assert r.max() < 100, (side, r.max())


def run_gpu(d, **kw):
    return X.tgevc3(d["side"], d["howmny"], d["S"], d["P"], d["alpha"], d["beta"], alphai=d.get("alphai"),
                    VL=d["VL_in"].copy(order="F"), VR=d["VR_in"].copy(order="F"), select=d.get("select"), **kw)


@pytest.mark.parametrize("path", golden_files(), ids=lambda p: p.split("/")[-1][:-4])
def test_golden(cuda_ok, path):
    d = load_golden(path)
    VL, VR, m, info = run_gpu(d)
    assert (m, info) == (d["m"], d["info"])
    ill = "quasi" in d["name"] or "tri" in d["name"] or "edge" in d["name"]
    tol = (TOL_ILL if ill else TOL_WELL)[d["S"].dtype.type]
    compare(d, VL, VR, m, d["VL_out"], d["VR_out"], tol)


def _pencil(kind, n, seed, dt):
    if kind == "gges":
        out = pencils.gen_gges(n, seed, dtype=dt)
        if np.issubdtype(dt, np.complexfloating):
            S, P, a, b, Q, Z = out
            return dict(S=S, P=P, alpha=a, beta=b, alphai=None, Q=Q, Z=Z)
        S, P, ar, ai, be, Q, Z = out
        return dict(S=S, P=P, alpha=ar, alphai=ai, beta=be, Q=Q, Z=Z)
    if kind == "graded":
        S, P, a, b, Q, Z = pencils.gen_gges(n, seed, dtype=dt, graded=True)
        return dict(S=S, P=P, alpha=a, beta=b, alphai=None, Q=Q, Z=Z)
    if kind == "schur":
        S, P, ar, ai, be = pencils.gen_schur_like(n, seed, dtype=dt)
        I = np.eye(n, dtype=dt, order="F")
        return dict(S=S, P=P, alpha=ar, alphai=ai, beta=be, Q=I, Z=I.copy(order="F"))
    raise ValueError(kind)


CASES = [
    # (kind, n, seed, dtype, side, howmny)
    ("gges", 128, 21, np.float64, "B", "B"),
    ("gges", 257, 22, np.float64, "B", "A"),
    ("gges", 200, 23, np.float64, "R", "B"),
    ("gges", 190, 24, np.float64, "L", "B"),
    ("schur", 700, 25, np.float64, "B", "A"),
    ("gges", 160, 26, np.float32, "B", "B"),
    ("gges", 150, 27, np.complex128, "B", "B"),
    ("gges", 131, 28, np.complex128, "R", "A"),
    ("gges", 120, 29, np.complex64, "B", "B"),
]


@pytest.mark.parametrize("case", CASES, ids=lambda c: f"{c[0]}-{c[1]}-{np.dtype(c[3]).name}-{c[4]}{c[5]}")
def test_against_oracle(cuda_ok, case):
    kind, n, seed, dt, side, howmny = case
    p = _pencil(kind, n, seed, dt)
    d = dict(side=side, howmny=howmny, S=p["S"], P=p["P"], alpha=p["alpha"], beta=p["beta"], alphai=p["alphai"],
             VL_in=p["Q"], VR_in=p["Z"], name=kind)
    ref = oracle.tgevc3(side, howmny, d["S"], d["P"], d["alpha"], d["beta"], alphai=d["alphai"],
                        VL=p["Q"].copy(order="F"), VR=p["Z"].copy(order="F"))
    VL, VR, m, info = run_gpu(d)
    assert (m, info) == (ref[2], ref[3])
    tol = (TOL_ILL if kind == "schur" else TOL_WELL)[np.dtype(dt).type]
    compare(d, VL, VR, m, ref[0], ref[1], tol)


def test_graded_complex_scale_guards(cuda_ok):
    """zgges pencil of A, D*B with log10 d_i ~ U(-8, 8): eigenvalues over many orders of
    magnitude and several exactly infinite ones (beta = 0).

    The upstream code divides by the zero pivots of the repeated infinite eigenvalues
    (non-finite columns), and its panel-wide overflow guard then scales the whole
    32-column panel by (bignum/10)/inf = 0, so the other columns of that panel come back
    as zero vectors.  Those degenerate oracle columns are excluded from the elementwise
    comparison and checked by residual instead; the CUDA path (exact zero pivots raised
    to smin, per-column guards) must be finite everywhere."""
    p = _pencil("graded", 160, 31, np.complex128)
    I = np.eye(160, dtype=np.complex128, order="F")
    d = dict(side="R", howmny="A", S=p["S"], P=p["P"], alpha=p["alpha"], beta=p["beta"], alphai=None,
             VL_in=I, VR_in=I.copy(order="F"), name="graded")
    ref = oracle.tgevc3("R", "A", d["S"], d["P"], d["alpha"], d["beta"])[1]
    VL, VR, m, info = run_gpu(d)
    assert info == 0 and np.isfinite(VR).all()
    good = np.isfinite(ref).all(0) & (np.abs(ref).max(0) > 0)
    assert good.sum() >= 100
    err, cols = oracle.max_rel_diff(VR[:, good], ref[:, good])
    assert err < 1e-9, err
    finite_eig = np.abs(d["beta"]) > 0
    r = oracle.residual_ratio(d["S"], d["P"], VR[:, :m], d["alpha"], d["beta"])
    assert r[finite_eig].max() < 100, r[finite_eig].max()


@pytest.mark.parametrize("dt", [np.float64, np.complex128], ids=["d", "z"])
def test_growth_guards_random_triangular(cuda_ok, dt):
    """n = 2048 random triangular pencils with the structure of the upstream test
    generators (U(-1,1) parts, |P_kk| pushed away from 0; real: 2x2 blocks as well).  Close
    eigenvalues make many eigenvectors grow by more than 1e300 across the matrix, so the
    overflow guards rescale hundreds of columns, in every block of a group of blocks that
    share one trailing update, and inside 64-row blocks.  Both sides must be finite, match the oracle column by column
    (1e-11) and have a DGET52-style residual below 100."""
    n, seed = 2048, 8213
    if dt == np.float64:
        S, P, al, ai, be = pencils.gen_quasi_triangular(n, seed)
    else:
        (S, P, al, be), ai = pencils.gen_upper_triangular_complex(n, seed), None
    I = np.eye(n, dtype=dt, order="F")
    d = dict(side="B", howmny="A", S=S, P=P, alpha=al, beta=be, alphai=ai, VL_in=I, VR_in=I.copy(order="F"),
             name="random")
    ref = oracle.tgevc3("B", "A", S, P, al, be, alphai=ai)
    VL, VR, m, info = run_gpu(d)
    assert (m, info) == (ref[2], ref[3]) == (n, 0)
    assert np.isfinite(VL).all() and np.isfinite(VR).all()
    # a real eigenvalue's column starts from x_k = 1: |x_k| < 1 means a guard rescaled it
    unit_seed = np.ones(n, bool) if ai is None else (ai == 0)
    guarded = int((np.abs(np.diag(as_complex(VR, d)))[unit_seed] < 1).sum())
    assert guarded >= 50, guarded  # the case exercises the guards
    compare(d, VL, VR, m, ref[0], ref[1], TOL_WELL[dt])


@pytest.mark.parametrize("dt", [np.float64, np.complex128], ids=["d", "z"])
def test_growth_cap_graded_left(cuda_ok, dt):
    """n = 4096 random triangular pencil with the rows of P scaled by 10^U(-8,8) (a 2x2
    block's rows share one factor), left eigenvectors: consecutive rows can differ by 1e16,
    so some columns grow past the range of the format within a few rows of one block and
    only the per-row cap keeps them finite.  Every column must be finite with a DGET52-style
    residual below 100; where the upstream library is built (oracle/_ref), the columns must
    also match it (1e-11 after normalisation)."""
    n, seed = 4096, 8213
    if dt == np.float64:
        S, P, al, ai, be = pencils.gen_quasi_triangular(n, seed)
    else:
        (S, P, al, be), ai = pencils.gen_upper_triangular_complex(n, seed), None
    g = 10.0 ** np.random.default_rng(seed + 1).uniform(-8, 8, n)
    k = 0
    while ai is not None and k < n:
        if ai[k] != 0 and k + 1 < n:
            g[k + 1] = g[k]
            k += 2
        else:
            k += 1
    P = np.asfortranarray(g[:, None] * P)
    be = np.diag(P).copy()
    I = np.eye(n, dtype=dt, order="F")
    d = dict(side="L", howmny="A", S=S, P=P, alpha=al, beta=be, alphai=ai, VL_in=I, VR_in=I.copy(order="F"),
             name="graded")
    VL, VR, m, info = run_gpu(d)
    assert (m, info) == (n, 0)
    assert np.isfinite(VL).all()
    V = as_complex(VL, d)
    a_c, b_c = oracle.column_eigenvalues(al, be, alphai=ai)
    r = oracle.residual_ratio(S, P, V, a_c, b_c, left=True)
    assert r.max() < 100, r.max()
    if oracle.ref_available():
        ref = oracle.tgevc3("L", "A", S, P, al, be, alphai=ai, impl="ref")[0]
        err, _ = oracle.max_rel_diff(V, as_complex(ref, d))
        assert err < 1e-11, err


def test_selection_and_one_sided(cuda_ok):
    p = _pencil("gges", 150, 41, np.float64)
    rng = np.random.default_rng(0)
    sel = (rng.random(150) < 0.3).astype(np.int32)
    for side in ("R", "L", "B"):
        d = dict(side=side, howmny="S", S=p["S"], P=p["P"], alpha=p["alpha"], beta=p["beta"], alphai=p["alphai"],
                 VL_in=np.zeros((150, 150), order="F"), VR_in=np.zeros((150, 150), order="F"), select=sel,
                 name="sel")
        ref = oracle.tgevc3(side, "S", d["S"], d["P"], d["alpha"], d["beta"], alphai=d["alphai"], select=sel)
        VL, VR, m, info = run_gpu(d)
        assert (m, info) == (ref[2], ref[3])
        compare(d, VL, VR, m, ref[0], ref[1], TOL_WELL[np.float64])


def test_normalize_flag(cuda_ok):
    p = _pencil("gges", 140, 42, np.float64)
    d = dict(side="B", howmny="B", S=p["S"], P=p["P"], alpha=p["alpha"], beta=p["beta"], alphai=p["alphai"],
             VL_in=p["Q"], VR_in=p["Z"], name="norm")
    VL0, VR0, m, _ = run_gpu(d)
    X.set_flags(X.NORMALIZE)
    try:
        VL1, VR1, m1, _ = run_gpu(d)
    finally:
        X.set_flags(0)
    for V0, V1 in ((VL0, VL1), (VR0, VR1)):
        c1 = as_complex(V1, d)
        mx = (np.abs(c1.real) + np.abs(c1.imag)).max(0)
        np.testing.assert_allclose(mx, 1.0, rtol=1e-13)
        err, _ = oracle.max_rel_diff(c1, as_complex(V0, d))
        assert err < 1e-13


def test_simt_and_tensor_core_paths_agree(cuda_ok):
    p = _pencil("gges", 300, 43, np.float64)
    d = dict(side="B", howmny="B", S=p["S"], P=p["P"], alpha=p["alpha"], beta=p["beta"], alphai=p["alphai"],
             VL_in=p["Q"], VR_in=p["Z"], name="simt")
    VL0, VR0, m, _ = run_gpu(d)
    X.set_flags(X.SIMT)
    try:
        VL1, VR1, _, _ = run_gpu(d)
    finally:
        X.set_flags(0)
    for A, B in ((VL0, VL1), (VR0, VR1)):
        den = np.abs(B).max(0)
        assert (np.abs(A - B).max(0) / den).max() < 1e-12


@pytest.mark.parametrize("n", [1, 2, 3, 63, 64, 65, 129])
def test_small_and_boundary_sizes(cuda_ok, n):
    S, P, ar, ai, be = pencils.gen_quasi_triangular(n, 100 + n, pair_frac=0.5)
    I = np.eye(n, order="F")
    d = dict(side="B", howmny="A", S=S, P=P, alpha=ar, beta=be, alphai=ai, VL_in=I, VR_in=I.copy(order="F"),
             name="quasi")
    ref = oracle.tgevc3("B", "A", S, P, ar, be, alphai=ai)
    VL, VR, m, info = run_gpu(d)
    assert (m, info) == (ref[2], ref[3])
    compare(d, VL, VR, m, ref[0], ref[1], TOL_ILL[np.float64], check_resid=False)


def test_device_api_matches_host_api(cuda_ok):
    import torch
    p = _pencil("gges", 180, 44, np.float64)
    n = 180
    d = dict(side="B", howmny="B", S=p["S"], P=p["P"], alpha=p["alpha"], beta=p["beta"], alphai=p["alphai"],
             VL_in=p["Q"], VR_in=p["Z"], name="dev")
    VLh, VRh, m, info = run_gpu(d)

    def dev(a):  # column-major device tensor
        return torch.from_numpy(np.ascontiguousarray(a.T)).cuda().t()

    S, P, VL, VR = dev(p["S"]), dev(p["P"]), dev(p["Q"]), dev(p["Z"])
    m2, info2 = X.tgevc3_dev("B", "B", S, P, p["alpha"], p["beta"], alphai=p["alphai"], VL=VL, VR=VR)
    torch.cuda.synchronize()
    assert (m2, info2) == (m, info)
    np.testing.assert_array_equal(VL.t().cpu().numpy().T, VLh[:, :m])
    np.testing.assert_array_equal(VR.t().cpu().numpy().T, VRh[:, :m])
    assert n == m


@pytest.mark.parametrize("howmny", ["B", "A"])
@pytest.mark.parametrize("dt", [np.float64, np.float32], ids=["d", "s"])
def test_host_panels_match_device_api(cuda_ok, dt, howmny):
    """The host-pointer form of a real pencil uploads S and P in 512-column panels while the
    solve runs (right to left: the right side waits for each group's panels, the left side
    for all of them), reads the subdiagonal from the caller's S and takes anorm, bnorm from
    host threads summing in the device reduction's order.  At n = 1100 (three panels) every
    column equals the device form's, bit for bit."""
    import torch
    n = 1100
    p = _pencil("schur", n, 7, dt)
    rng = np.random.default_rng(11)
    Q = np.asfortranarray(np.linalg.qr(rng.standard_normal((n, n)))[0].astype(dt))
    Z = np.asfortranarray(np.linalg.qr(rng.standard_normal((n, n)))[0].astype(dt))
    back = howmny == "B"
    VLh, VRh, m, info = X.tgevc3("B", howmny, p["S"], p["P"], p["alpha"], p["beta"], alphai=p["alphai"],
                                 VL=Q.copy(order="F") if back else None, VR=Z.copy(order="F") if back else None)
    assert (m, info) == (n, 0)

    def dev(a):  # column-major device tensor
        return torch.from_numpy(np.ascontiguousarray(a.T)).cuda().t()

    VL = dev(Q) if back else dev(np.zeros((n, n), dtype=dt))
    VR = dev(Z) if back else dev(np.zeros((n, n), dtype=dt))
    m2, info2 = X.tgevc3_dev("B", howmny, dev(p["S"]), dev(p["P"]), p["alpha"], p["beta"], alphai=p["alphai"],
                             VL=VL, VR=VR)
    torch.cuda.synchronize()
    assert (m2, info2) == (m, info)
    np.testing.assert_array_equal(VL.t().cpu().numpy().T, VLh[:, :m])
    np.testing.assert_array_equal(VR.t().cpu().numpy().T, VRh[:, :m])


SPLIT_CASES = [
    # (kind, n, seed, side, howmny, slices, elementwise tolerance vs the FP64 oracle, slice kind)
    ("gges", 257, 71, "B", "B", 6, 1e-10, "bf16"),
    ("gges", 300, 72, "B", "A", 6, 1e-10, "bf16"),
    ("schur", 700, 73, "B", "B", 6, 1e-6, "bf16"),
    ("gges", 257, 71, "B", "B", 7, 1e-10, "int8"),
    ("gges", 300, 72, "B", "A", 7, 1e-10, "int8"),
    ("schur", 700, 73, "B", "B", 7, 1e-6, "int8"),
    ("gges", 257, 71, "B", "B", 14, 1e-10, "crt"),
    ("gges", 300, 72, "B", "A", 14, 1e-10, "crt"),
    ("schur", 700, 73, "B", "B", 14, 1e-6, "crt"),
    ("gges", 1100, 74, "B", "B", 14, 1e-10, "crt"),
]


@pytest.mark.parametrize("case", SPLIT_CASES, ids=lambda c: f"{c[0]}-{c[1]}-{c[3]}{c[4]}-{c[7]}-s{c[5]}")
def test_split_precision_form(cuda_ok, case):
    """XTGEVC3_SPLIT: updates and back-transform as slice products on the tensor cores;
    solves stay FP64.  BF16 slices: FP32 accumulation exact per 128-deep chunk, FP64
    summation, 6 slices ~48 bits per operand.  INT8 slices (XTGEVC3_SPLIT_INT8): INT32
    accumulation exact over the whole K, 7 slices ~49 bits.  Residues (XTGEVC3_SPLIT_CRT):
    one exact INT8 GEMM per modulus, 14 moduli ~47-bit operands.  The result must match the FP64
    oracle elementwise within the stated tolerance (looser on the ill-conditioned stand-in
    pencil) and its residual must meet the DGET52 bound used for the plain form."""
    kind, n, seed, side, howmny, s, tol, sk = case
    p = _pencil(kind, n, seed, np.float64)
    d = dict(side=side, howmny=howmny, S=p["S"], P=p["P"], alpha=p["alpha"], beta=p["beta"], alphai=p["alphai"],
             VL_in=p["Q"], VR_in=p["Z"], name=kind)
    ref = oracle.tgevc3(side, howmny, d["S"], d["P"], d["alpha"], d["beta"], alphai=d["alphai"],
                        VL=p["Q"].copy(order="F"), VR=p["Z"].copy(order="F"))
    X.set_flags(X.SPLIT | X.slices(s) | {"bf16": 0, "int8": X.SPLIT_INT8, "crt": X.SPLIT_CRT}[sk])
    try:
        VL, VR, m, info = run_gpu(d)
    finally:
        X.set_flags(0)
    assert (m, info) == (ref[2], ref[3])
    compare(d, VL, VR, m, ref[0], ref[1], tol, check_resid=(howmny == "A"))


def _overflow_pencil(n, seed, jump, left):
    """Real triangular pencil whose eigenvectors grow by ~jump once per 64-row block: the
    strictly upper part of one row per block (right eigenvectors) or of one column per
    block (left eigenvectors) is scaled by jump.  Over a column the growth passes the
    overflow threshold many times over, so the overflow guards rescale many columns, while
    within one row block it stays representable."""
    rng = np.random.default_rng(seed)
    S = np.triu(rng.standard_normal((n, n)), 1)
    if left:
        S[:, np.arange(31, n, 64)] *= jump
    else:
        S[np.arange(n - 32, 0, -64), :] *= jump
    S = np.triu(S, 1)
    S[np.diag_indices(n)] = np.arange(1, n + 1) * (1 + 0.1 * rng.random(n))
    P = np.triu(rng.standard_normal((n, n)), 1) * 1e-3
    P[np.diag_indices(n)] = 1.0 + rng.random(n)
    S, P = np.asfortranarray(S), np.asfortranarray(P)
    return S, P, np.diag(S).copy(), np.zeros(n), np.diag(P).copy()


@pytest.mark.parametrize("side", ["R", "L"])
def test_lookahead_matches_serial_path_with_guards(cuda_ok, side):
    """The look-ahead schedule (XTGEVC3_LOOKAHEAD: trailing updates of block pairs on a
    second stream, guard scaling of the rows they write deferred to a later kernel) must
    agree with the default serial schedule, which sums the trailing updates of four blocks
    in one GEMM, to rounding also when the overflow guards rescale many columns: the same
    guards fire, so the raw columns agree within 1e-9 of their largest entry.  It must also
    match the oracle column by column after normalisation (the oracle rescales whole
    32-column panels where this implementation rescales single columns)."""
    n = 1536
    S, P, ar, ai, be = _overflow_pencil(n, 91, 1e16, side == "L")
    I = np.eye(n, order="F")
    d = dict(side=side, howmny="A", S=S, P=P, alpha=ar, beta=be, alphai=ai, VL_in=I, VR_in=I.copy(order="F"),
             name="overflow")
    X.set_flags(X.LOOKAHEAD)
    try:
        VL0, VR0, m, info = run_gpu(d)
    finally:
        X.set_flags(0)
    V0 = VL0 if side == "L" else VR0
    assert info == 0 and np.isfinite(V0).all()
    # the guards fired: columns come back with their seed entry x_k scaled below 1
    assert (np.abs(np.diag(V0[:, :n])) < 1).sum() >= 8
    VL1, VR1, _, _ = run_gpu(d)  # the default, serial schedule
    V1 = VL1 if side == "L" else VR1
    den = np.abs(V1).max(0)
    den[den == 0] = 1
    raw = (np.abs(V0 - V1).max(0) / den).max()
    assert raw < 1e-9, raw
    ref = oracle.tgevc3(side, "A", S, P, ar, be, alphai=ai)
    compare(d, VL0, VR0, m, ref[0], ref[1], TOL_ILL[np.float64], check_resid=False)


@pytest.mark.parametrize("sk,side", [("int8", "R"), ("int8", "L"), ("bf16", "R"), ("crt", "R"), ("crt", "L")])
def test_split_form_guards_across_groups(cuda_ok, sk, side):
    """Split-precision form on the n = 1536 pencil whose eigenvectors grow by 1e16 per row
    block: its trailing updates (groups of eight row blocks, K = 2 x 512, at least 512 rows)
    run as slice products, and guards that fire in a group's upper blocks rescale the
    operand rows of up to seven blocks below them.  Must be finite, show the guards firing
    and match the oracle after normalisation (1e-8, as the plain form on this pencil)."""
    n = 1536
    S, P, ar, ai, be = _overflow_pencil(n, 91, 1e16, side == "L")
    I = np.eye(n, order="F")
    d = dict(side=side, howmny="A", S=S, P=P, alpha=ar, beta=be, alphai=ai, VL_in=I, VR_in=I.copy(order="F"),
             name="overflow")
    X.set_flags(X.SPLIT | {"int8": X.SPLIT_INT8 | X.slices(7), "bf16": X.slices(6), "crt": X.SPLIT_CRT}[sk])
    try:
        VL, VR, m, info = run_gpu(d)
    finally:
        X.set_flags(0)
    V = VL if side == "L" else VR
    assert info == 0 and np.isfinite(V).all()
    assert (np.abs(np.diag(V[:, :n])) < 1).sum() >= 8
    # guards rescale a column's finished rows and its residual sketch together: the check
    # must not flag the rescaled columns wholesale
    assert X.split_refined() < n // 8, X.split_refined()
    ref = oracle.tgevc3(side, "A", S, P, ar, be, alphai=ai)
    compare(d, VL, VR, m, ref[0], ref[1], TOL_ILL[np.float64], check_resid=False)


def test_config_dgges_n1024_both_sides_back_transformed(cuda_ok):
    """The plain dtgevc3 configuration at its own size: a real pencil of order 1024 made by
    xGGES (ordering off) from seeded iid N(0,1) A, B, SIDE='B', HOWMNY='B' with Q and Z.
    Against the upstream library built from its sources (oracle/_ref; the C restatement
    where that library is absent): INFO and M equal, every column within 1e-11 of the column
    max after normalisation; and the DGET52-style residual of the back-transformed
    eigenvectors against the original pencil (A, B) = (Q S Z^T, Q P Z^T) below 100."""
    n = 1024
    S, P, ar, ai, be, Q, Z = pencils.gen_gges(n, 1024)
    impl = "ref" if oracle.ref_available() else "oracle"
    RL, RR, mr, infor = oracle.tgevc3("B", "B", S, P, ar, be, alphai=ai, VL=Q.copy(order="F"),
                                      VR=Z.copy(order="F"), impl=impl)
    VL, VR, m, info = X.tgevc3("B", "B", S, P, ar, be, alphai=ai, VL=Q.copy(order="F"), VR=Z.copy(order="F"))
    assert (m, info) == (mr, infor) == (n, 0)
    A, B = Q @ S @ Z.T, Q @ P @ Z.T
    al, bc = oracle.column_eigenvalues(ar, be, alphai=ai)
    for side, V, R in (("L", VL, RL), ("R", VR, RR)):
        a = oracle.to_complex_real_storage(V, ai)
        b = oracle.to_complex_real_storage(R, ai)
        err, cols = oracle.max_rel_diff(a, b)
        assert err <= 1e-11, (side, err, int(np.nanargmax(cols)))
        r = oracle.residual_ratio(A, B, a, al, bc, left=(side == "L"))
        assert r.max() < 100, (side, r.max())


@pytest.mark.parametrize("n", [700, 1500, 3000, 6000, 8300])
def test_normalize_one_pass_kernel_sizes(cuda_ok, n):
    """XTGEVC3_NORMALIZE over every register tile of the one-pass kernel (rows per thread 4,
    8, 16, 32) and the two-pass form past 8192 rows, on the device with a selection: every
    normalised eigenvector (a real pair jointly) has max |re| + |im| = 1 and is the
    unnormalised one times a positive scalar (to rounding)."""
    import torch
    S, P, ar, ai, be = pencils.gen_schur_like(n, 50 + n)
    sel = (np.random.default_rng(n).random(n) < 0.3).astype(np.int32)
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a.T)).cuda().t()  # noqa: E731
    dS, dP = dev(S), dev(P)
    outs = []
    for flags in (0, X.NORMALIZE):
        VL = torch.zeros(n, n, dtype=torch.float64, device="cuda").t()
        VR = torch.zeros(n, n, dtype=torch.float64, device="cuda").t()
        m, info = X.tgevc3_dev("B", "S", dS, dP, ar, be, alphai=ai, VL=VL, VR=VR, select=sel, flags=flags)
        assert info == 0
        outs.append((VL[:, :m], VR[:, :m]))
    # columns of each eigenvector: a pair's two columns share one scale
    items, k, c = [], 0, 0
    while k < n:
        pair = ai[k] != 0 and k + 1 < n
        if sel[k] or (pair and sel[k + 1]):
            items.append((c, pair))
            c += 2 if pair else 1
        k += 2 if pair else 1
    for side in (0, 1):
        V0, V1 = outs[0][side], outs[1][side]
        for c, pair in items:
            a0 = V0[:, c:c + (2 if pair else 1)]
            a1 = V1[:, c:c + (2 if pair else 1)]
            mx = float(a1.abs().sum(1).max()) if pair else float(a1.abs().max())
            assert abs(mx - 1.0) < 1e-14, (side, c, mx)
            s = float((a0.abs().sum(1).max()) if pair else a0.abs().max())
            assert float((a0 / s - a1).abs().max()) < 1e-15 * 4, (side, c)


@pytest.mark.parametrize("case", ["gges_B", "gges_sel_L", "guards_A"])
def test_tensor_core_solves_match_warp_solves(cuda_ok, monkeypatch, case):
    """XTGEVC3_DIAG_TC=1 runs the real double diagonal solves with their in-block updates on
    the FP64 tensor cores (eight columns of a warp share each sub-block's row updates as
    m8n8k4 MMAs) instead of the default one-eigenvector-per-warp kernel.  Both must give the
    same eigenvectors to rounding
    (column max difference 1e-12 after normalisation): an xGGES pencil with Q, Z, both
    sides; a selection, left side; and a random triangular pencil whose columns the growth
    guards rescale (n = 2048, HOWMNY 'A')."""
    if case == "guards_A":
        n = 2048
        S, P, al, ai, be = pencils.gen_quasi_triangular(n, 8213)
        Q = Z = np.eye(n, order="F")
        side, howmny, sel = "B", "A", None
    else:
        n = 700
        S, P, al, ai, be, Q, Z = pencils.gen_gges(n, 77)
        side, howmny = ("B", "B") if case == "gges_B" else ("L", "S")
        sel = (np.random.default_rng(5).random(n) < 0.35).astype(np.int32) if howmny == "S" else None
    out = {}
    for simt in ("0", "1"):
        monkeypatch.setenv("XTGEVC3_DIAG_TC", "0" if simt == "1" else "1")
        out[simt] = X.tgevc3(side, howmny, S, P, al, be, alphai=ai, VL=Q.copy(order="F"), VR=Z.copy(order="F"),
                             select=sel)
    (VL, VR, m, info), (VLs, VRs, ms, infos) = out["0"], out["1"]
    assert (m, info) == (ms, infos)
    d = dict(alphai=ai, howmny=howmny, select=sel)
    for sd, A, B in (("L", VL, VLs), ("R", VR, VRs)):
        if side not in (sd, "B"):
            continue
        assert np.isfinite(A[:, :m]).all()
        err, _ = oracle.max_rel_diff(as_complex(A[:, :m], d), as_complex(B[:, :m], d))
        assert err < 1e-12, (sd, err)


@pytest.mark.parametrize("form", ["plain", "crt"])
def test_host_row_panels_match_device_api(cuda_ok, form):
    """From n = 4096 the host-pointer form uploads Q and Z in row panels (two here) and runs
    each side's back-transform panel by panel as its rows arrive (V rows = Z rows X),
    downloading every panel's rows at once; every column must equal the device form's (one
    back-transform over all rows), bit for bit, in the FP64 form and in the residue form."""
    import torch
    n = 4096
    p = _pencil("schur", n, 9, np.float64)
    g = torch.Generator(device="cuda").manual_seed(13)
    Qd = torch.linalg.qr(torch.randn(n, n, device="cuda", dtype=torch.float64, generator=g))[0]
    Zd = torch.linalg.qr(torch.randn(n, n, device="cuda", dtype=torch.float64, generator=g))[0]
    Q, Z = np.asfortranarray(Qd.cpu().numpy()), np.asfortranarray(Zd.cpu().numpy())
    flags = X.SPLIT | X.SPLIT_CRT if form == "crt" else 0
    X.set_flags(flags)
    try:
        VLh, VRh, m, info = X.tgevc3("B", "B", p["S"], p["P"], p["alpha"], p["beta"], alphai=p["alphai"],
                                     VL=Q.copy(order="F"), VR=Z.copy(order="F"))
    finally:
        X.set_flags(0)
    assert (m, info) == (n, 0)

    def dev(a):  # column-major device tensor
        return torch.from_numpy(np.ascontiguousarray(a.T)).cuda().t()

    VL, VR = dev(Q), dev(Z)
    m2, info2 = X.tgevc3_dev("B", "B", dev(p["S"]), dev(p["P"]), p["alpha"], p["beta"], alphai=p["alphai"],
                             VL=VL, VR=VR, flags=flags)
    torch.cuda.synchronize()
    assert (m2, info2) == (m, info)
    assert np.isfinite(VLh[:, :m]).all() and np.isfinite(VRh[:, :m]).all()
    np.testing.assert_array_equal(VL.t().cpu().numpy().T, VLh[:, :m])
    np.testing.assert_array_equal(VR.t().cpu().numpy().T, VRh[:, :m])
