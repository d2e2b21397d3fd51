"""The C-ABI library: it loads, exports every symbol the headers declare, and implements
the upstream argument checks (INFO, M, LWORK query) -- all without touching a GPU."""
import ctypes as ct
import os
import re
import subprocess

import numpy as np
import pytest

import xtgevc3_b200 as X
from conftest import ROOT

HEADERS = [os.path.join(ROOT, "include", h) for h in ("xtgevc3.h", "tgevc3.h")]


def declared_c_functions():
    src = open(HEADERS[0]).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(xtgevc3_\w+)\s*\(", src)))


def exported():
    out = subprocess.run(["nm", "-D", "--defined-only", X.lib()._name], capture_output=True, text=True).stdout
    return {line.split()[-1] for line in out.splitlines() if line.strip()}


def test_exports_c_abi():
    syms = exported()
    decl = declared_c_functions()
    assert len(decl) >= 11
    missing = [f for f in decl if f not in syms]
    assert not missing, missing


def test_exports_cpp_dropin_symbols():
    """include/tgevc3.h keeps C++ linkage, like the upstream header: the mangled names of
    the four upstream functions must be defined by libxtgevc3.so."""
    syms = exported()
    demangled = subprocess.run(["c++filt"], input="\n".join(sorted(syms)), capture_output=True,
                               text=True).stdout.splitlines()
    for p, t in (("d", "double"), ("s", "float"), ("z", "std::complex<double>"), ("c", "std::complex<float>")):
        want = f"{p}tgevc3(char, char, int const*, int, {t} const*, int, {t} const*, int"
        assert any(d.startswith(want) for d in demangled), p


@pytest.mark.parametrize("pfx", ["d", "s", "z", "c"])
def test_lwork_query_and_info_codes(pfx):
    from xtgevc3_b200 import pencils
    n = 17
    if pfx in "ds":
        dt = np.float64 if pfx == "d" else np.float32
        S, P, ar, ai, be = pencils.gen_quasi_triangular(n, 3, dtype=dt)
        kw = dict(alphai=ai)
        al = ar
    else:
        dt = np.complex128 if pfx == "z" else np.complex64
        S, P, al, be = pencils.gen_upper_triangular_complex(n, 3, dtype=dt)
        kw = {}
    # LWORK = -1 query: upstream formula 2n(b+1) + 4(b+1)^2 + 2(b+1), b = 32
    lib = X.lib()
    m = ct.c_int(-1)
    info = ct.c_int(-99)
    q = np.zeros(2, dtype=dt)
    rdt = np.float64 if pfx in "dz" else np.float32
    head = [b"B", b"A", None, n, S.ctypes.data_as(ct.c_void_p), n, P.ctypes.data_as(ct.c_void_p), n]
    VL = np.zeros((n, n), dtype=dt, order="F")
    VR = np.zeros((n, n), dtype=dt, order="F")
    if pfx in "ds":
        eig = [np.ascontiguousarray(a, dtype=rdt) for a in (al, kw["alphai"], be)]
    else:
        eig = [np.ascontiguousarray(a, dtype=dt) for a in (al, be)]
    eigp = [e.ctypes.data_as(ct.c_void_p) for e in eig]
    f = getattr(lib, f"xtgevc3_{pfx}tgevc3")
    f(*head, *eigp, VL.ctypes.data_as(ct.c_void_p), n, VR.ctypes.data_as(ct.c_void_p), n, n, ct.byref(m),
      q.ctypes.data_as(ct.c_void_p), -1, ct.byref(info))
    assert info.value == 0 and m.value == n
    assert int(np.real(q[0])) == X.lwork_query(pfx, n) == 2 * n * 33 + 4 * 33 * 33 + 66
    # bad HOWMNY -> -2 (SIDE is not validated upstream)
    _, _, _, inf = X.tgevc3("B", "Q", S, P, al, be, **kw)
    assert inf == -2
    # MM < M -> -16, and M is still reported
    _, _, mm, inf = X.tgevc3("B", "A", S, P, al, be, mm=3, **kw)
    assert inf == -16 and mm == n
    # LWORK too small for every block size -> -19
    _, _, mm, inf = X.tgevc3("B", "A", S, P, al, be, lwork=5, **kw)
    assert inf == -19
    # n = 0 -> info 0, m = 0
    e = np.zeros((0, 0), dtype=dt, order="F")
    _, _, mm, inf = X.tgevc3("B", "A", e, e, np.zeros(0, dt), np.zeros(0, dt),
                             **({"alphai": np.zeros(0, dt)} if pfx in "ds" else {}), mm=0)
    assert inf == 0 and mm == 0
    # HOWMNY='S' with no selection: nothing computed, info 0
    _, _, mm, inf = X.tgevc3("B", "S", S, P, al, be, select=np.zeros(n, np.int32), **kw)
    assert inf == 0 and mm == 0


def test_selection_count_pairs():
    """A pair counts (2 columns) when either flag is set; a pair flag on the last row is real."""
    from xtgevc3_b200 import pencils
    S, P, ar, ai, be = pencils.gen_quasi_triangular(30, 9, pair_frac=0.6)
    pairs = [k for k in range(29) if ai[k] > 0]
    k = pairs[0]
    sel = np.zeros(30, np.int32)
    sel[k + 1] = 1  # only the second flag of the pair
    _, _, m, info = X.tgevc3("R", "S", S, P, ar, be, alphai=ai, select=sel, mm=0)
    assert info == -16 and m == 2


def test_flags_roundtrip():
    old = X.get_flags()
    X.set_flags(X.NORMALIZE | X.SIMT)
    assert X.get_flags() == 3
    X.set_flags(old)


def _fake_desc(n=8, **over):
    """A descriptor with distinct non-NULL (never dereferenced) addresses."""
    d = X.PencilDesc()
    d.n = n
    for i, key in enumerate(("S", "P", "alphar", "alphai", "beta", "Q", "Z", "VL", "VR")):
        setattr(d, key, ct.c_void_p(0x100000 * (i + 1)))
    for ld in ("lds", "ldp", "ldq", "ldz", "ldvl", "ldvr"):
        setattr(d, ld, n)
    for k, v in over.items():
        setattr(d, k, v)
    return d


@pytest.mark.parametrize("case,msg", [
    (dict(side=b"X"), "side"),
    (dict(howmny=b"S"), "howmny"),
    (dict(n=-1), "n < 0"),
    (dict(S=None), "NULL input"),
    (dict(lds=4), "lds/ldp"),
    (dict(VR=ct.c_void_p(0x100000 * 7 + 8)), "in place"),
    (dict(config=X.batch_config(8, 16)), "unknown tile configuration"),
])
def test_batched_create_argument_checks(case, msg):
    """Bad batched arguments are refused with -1 and a message before any CUDA call."""
    case = dict(case)
    side = case.pop("side", b"B")
    howmny = case.pop("howmny", b"B")
    config = case.pop("config", 0)
    arr = (X.PencilDesc * 2)(_fake_desc(8), _fake_desc(**{"n": 8, **case}))
    plan = ct.c_void_p()
    L = X.lib()
    for pfx in "ds":
        rc = getattr(L, f"xtgevc3_{pfx}tgevc3_batched_create")(side, howmny, 2, ct.cast(arr, ct.c_void_p), config,
                                                                ct.byref(plan))
        assert rc == -1 and not plan.value
        assert msg in X.last_error(), X.last_error()


def test_batched_default_config_roundtrip():
    old = X.batched_get_default("d")
    X.batched_set_default("d", X.batch_config(32, 32))
    assert X.batched_get_default("d") == X.batch_config(32, 32)
    X.batched_set_default("d", 0)
    assert X.batched_get_default("d") == old


@pytest.mark.parametrize("prec,n,ld,null,msg", [
    (b"q", 4, 4, False, "prec"),
    (b"d", -1, 4, False, "n < 0"),
    (b"d", 4, 4, True, "NULL"),
    (b"z", 8, 4, False, "leading dimension"),
])
def test_adjoint_argument_checks(prec, n, ld, null, msg):
    """xtgevc3_adjoint refuses bad arguments with -1 and a message, before any CUDA call."""
    L = X.lib()
    L.xtgevc3_adjoint.argtypes = [ct.c_char] + [ct.c_void_p] + [ct.c_int] + [ct.c_void_p, ct.c_int] * 2 + \
        [ct.c_void_p] * 3 + [ct.c_void_p, ct.c_int] * 4
    L.xtgevc3_adjoint.restype = ct.c_int
    p = None if null else ct.c_void_p(0x1000)
    rc = L.xtgevc3_adjoint(prec, None, n, p, ld, p, ld, p, p, p, p, ld, p, ld, p, ld, p, ld)
    assert rc == -1
    assert msg in X.last_error(), X.last_error()


def test_noalloc_refuses_oversize_before_device_work():
    """xtgevc3_dtgevc3_dev_noalloc: the 8 MiB block holds SIDE='B', HOWMNY='B' up to n = 478;
    n = 479 needs 8,393,728 bytes and is refused with return code 2 before any CUDA call
    (so the device pointers here, never dereferenced, may be dummies)."""
    L = X.lib()
    n = 479
    z, o = np.zeros(n), np.ones(n)
    m, info = ct.c_int(0), ct.c_int(0)
    dev = ct.c_void_p(0x1000)
    host = [a.ctypes.data_as(ct.c_void_p) for a in (z, z, o)]
    rc = L.xtgevc3_dtgevc3_dev_noalloc(None, b"B", b"B", None, n, dev, n, dev, n, *host, dev, n, dev, n, n,
                                       ct.byref(m), ct.byref(info))
    assert rc == 2
    assert "n=479" in X.last_error() and "8393728 bytes" in X.last_error(), X.last_error()


@pytest.mark.parametrize("pfx", ["d", "z"])
def test_trevc3_info_codes_and_query(pfx):
    """xtgevc3_{d,z}trevc3: LAPACK xTREVC3's INFO codes in its order, answered before any
    CUDA call (-1 SIDE, -2 HOWMNY, -4 N, -6 LDT, -8 LDVL, -10 LDVR, -11 MM < M, -14 LWORK,
    -16 LRWORK), and the workspace query (minimum max(1, 3n) real, max(1, 2n) complex)."""
    n = 6
    dt = np.float64 if pfx == "d" else np.complex128
    T = np.asfortranarray(np.triu(np.arange(1, n * n + 1, dtype=np.float64).reshape(n, n)).astype(dt))
    V = np.zeros((n, n), dtype=dt, order="F")

    def call(side=b"B", howmny=b"A", nn=n, ldt=n, ldvl=n, ldvr=n, mm=n, lwork=None, lrwork=n, sel=None):
        m, info = ct.c_int(-7), ct.c_int(0)
        work = np.zeros(4 * n, dtype=dt)
        lw = (3 if pfx == "d" else 2) * n if lwork is None else lwork
        if pfx == "d":
            X.lib().xtgevc3_dtrevc3(side, howmny, sel, nn, T.ctypes.data, ldt, V.ctypes.data, ldvl, V.ctypes.data,
                                   ldvr, mm, ct.byref(m), work.ctypes.data, lw, ct.byref(info))
        else:
            rwork = np.zeros(n)
            X.lib().xtgevc3_ztrevc3(side, howmny, sel, nn, T.ctypes.data, ldt, V.ctypes.data, ldvl, V.ctypes.data,
                                   ldvr, mm, ct.byref(m), work.ctypes.data, lw, rwork.ctypes.data, lrwork,
                                   ct.byref(info))
        return info.value, m.value, work
    assert call(side=b"X")[0] == -1
    assert call(howmny=b"Q")[0] == -2
    assert call(nn=-1)[0] == -4
    assert call(ldt=n - 1)[0] == -6
    assert call(ldvl=n - 1)[0] == -8
    assert call(side=b"R", ldvl=1)[0] != -8  # VL not referenced for SIDE='R'
    assert call(ldvr=n - 1)[0] == -10
    info, m, _ = call(mm=n - 1)
    assert (info, m) == (-11, n)
    assert call(lwork=1)[0] == -14
    if pfx == "z":
        assert call(lrwork=0)[0] == -16
    info, m, work = call(lwork=-1)
    assert info == 0 and int(np.real(work[0])) == (3 if pfx == "d" else 2) * n
    sel = np.zeros(n, dtype=np.int32)
    sel[[1, 4]] = 1
    info, m, _ = call(howmny=b"S", sel=sel.ctypes.data, lwork=-1)
    assert (info, m) == (0, 2)


def test_tgsna_info_codes_and_query():
    """xtgevc3_dtgsna: LAPACK xTGSNA's INFO codes in its order, answered before any CUDA
    call, and its LWORK: N for JOB = 'E', 2 N (N + 2) + 16 with DIF (JOB = 'V' / 'B'); LDVL
    and LDVR are not checked for JOB = 'V' (VL, VR not referenced); complex pencils' LWORK
    with DIF is 2 N^2 (Z/CTGSNA)."""
    n = 5
    A = np.asfortranarray(np.triu(np.arange(1.0, n * n + 1).reshape(n, n)))
    V = np.zeros((n, n), order="F")
    L = X.lib()

    def call(job=b"E", howmny=b"A", nn=n, lda=n, ldb=n, ldvl=n, ldvr=n, mm=n, lwork=n, sel=None):
        m, info = ct.c_int(-7), ct.c_int(0)
        s = np.zeros(n)
        work = np.zeros(n)
        L.xtgevc3_dtgsna(job, howmny, sel, nn, A.ctypes.data, lda, A.ctypes.data, ldb, V.ctypes.data, ldvl,
                         V.ctypes.data, ldvr, s.ctypes.data, None, mm, ct.byref(m), work.ctypes.data, lwork, None,
                         ct.byref(info))
        return info.value, m.value, work
    assert call(job=b"X")[0] == -1
    lw_dif = 2 * n * (n + 2) + 16
    info, m, work = call(job=b"V", ldvl=1, ldvr=1, lwork=-1)
    assert (info, m, int(work[0])) == (0, n, lw_dif)
    assert call(job=b"V", ldvl=1, ldvr=1, lwork=lw_dif - 1)[0] == -18
    assert call(job=b"B", ldvl=n - 1, lwork=-1)[0] == -10
    zA = A.astype(np.complex128)
    zwork = np.zeros(2, dtype=np.complex128)
    m, info = ct.c_int(0), ct.c_int(0)
    L.xtgevc3_ztgsna(b"V", b"A", None, n, zA.ctypes.data, n, zA.ctypes.data, n, zA.ctypes.data, 1, zA.ctypes.data, 1,
                     None, None, n, ct.byref(m), zwork.ctypes.data, -1, None, ct.byref(info))
    assert (info.value, m.value, int(zwork[0].real)) == (0, n, 2 * n * n)  # ZTGSNA's LWORK with DIF
    assert call(howmny=b"B")[0] == -2
    assert call(nn=-1)[0] == -4
    assert call(lda=n - 1)[0] == -6
    assert call(ldb=n - 1)[0] == -8
    assert call(ldvl=n - 1)[0] == -10
    assert call(ldvr=n - 1)[0] == -12
    assert call(mm=n - 1)[:2] == (-15, n)
    assert call(lwork=0)[0] == -18
    info, m, work = call(lwork=-1)
    assert (info, m, int(work[0])) == (0, n, n)


def test_tgexc_info_codes_and_quick_returns():
    """xtgevc3_ztgexc: LAPACK ZTGEXC's INFO codes in its order (-3 N, -5 LDA, -7 LDB, -9 LDQ,
    -11 LDZ, -12 IFST, -13 ILST), answered before any CUDA call, and its quick returns
    (N <= 1, IFST = ILST) with the pencil untouched."""
    n = 5
    A = np.asfortranarray(np.triu(np.arange(1.0, n * n + 1).reshape(n, n)).astype(np.complex128))
    A0 = A.copy()
    L = X.lib()

    def call(wq=1, wz=1, nn=n, lda=n, ldb=n, ldq=n, ldz=n, ifst=1, ilst=3):
        il, info = ct.c_int(ilst), ct.c_int(7)
        L.xtgevc3_ztgexc(wq, wz, nn, A.ctypes.data, lda, A.ctypes.data, ldb, A.ctypes.data, ldq, A.ctypes.data, ldz,
                         ifst, ct.byref(il), ct.byref(info))
        return info.value, il.value
    assert call(nn=-1)[0] == -3
    assert call(lda=n - 1)[0] == -5
    assert call(ldb=n - 1)[0] == -7
    assert call(ldq=n - 1)[0] == -9
    assert call(ldq=0, wq=0)[0] == -9
    assert call(ldq=1, wq=0, ldz=n - 1)[0] == -11
    assert call(ldz=0, wz=0)[0] == -11
    assert call(ifst=0)[0] == -12 and call(ifst=n + 1)[0] == -12
    assert call(ilst=0)[0] == -13 and call(ilst=n + 1)[0] == -13
    assert call(nn=0, ifst=1, ilst=1)[0] == -12  # IFST > N
    assert call(nn=1, ifst=1, ilst=1, lda=1, ldb=1, ldq=1, ldz=1) == (0, 1)
    assert call(ifst=3, ilst=3) == (0, 3)
    assert (A == A0).all()


@pytest.mark.parametrize("pfx,dt", [("d", np.float64), ("s", np.float32)])
def test_real_tgexc_info_codes_and_quick_returns(pfx, dt):
    """xtgevc3_dtgexc / stgexc (IFST by pointer, in and out as in D/STGEXC): LAPACK's INFO
    codes in its order, answered before any CUDA call with IFST and ILST untouched, and the
    N <= 1 quick return."""
    n = 5
    A = np.asfortranarray(np.triu(np.arange(1.0, n * n + 1).reshape(n, n)).astype(dt))
    A0 = A.copy()
    f = getattr(X.lib(), f"xtgevc3_{pfx}tgexc")

    def call(wq=1, wz=1, nn=n, lda=n, ldb=n, ldq=n, ldz=n, ifst=1, ilst=3):
        fs, il, info = ct.c_int(ifst), ct.c_int(ilst), ct.c_int(7)
        f(wq, wz, nn, A.ctypes.data, lda, A.ctypes.data, ldb, A.ctypes.data, ldq, A.ctypes.data, ldz, ct.byref(fs),
          ct.byref(il), ct.byref(info))
        return info.value, fs.value, il.value
    assert call(nn=-1)[0] == -3
    assert call(lda=n - 1)[0] == -5
    assert call(ldb=n - 1)[0] == -7
    assert call(ldq=0, wq=0)[0] == -9
    assert call(ldz=n - 1)[0] == -11
    assert call(ifst=0) == (-12, 0, 3) and call(ifst=n + 1)[0] == -12
    assert call(ilst=0) == (-13, 1, 0) and call(ilst=n + 1)[0] == -13
    assert call(nn=1, ifst=1, ilst=1, lda=1, ldb=1, ldq=1, ldz=1) == (0, 1, 1)
    assert (A == A0).all()


def test_tgexc_python_wrapper_argument_errors():
    """xtgevc3_b200.tgexc passes 1-based positions through: out-of-range IFST / ILST come back
    as LAPACK's -12 / -13 (no CUDA call), with the arrays unchanged."""
    n = 4
    A = np.triu(np.ones((n, n), dtype=np.complex128))
    for ifst, ilst, code in ((0, 2, -12), (n + 1, 2, -12), (2, 0, -13), (2, n + 1, -13)):
        a, b, q, z, il, info = X.tgexc(A, A, A, A, ifst, ilst)
        assert info == code and il == ilst
        assert (a == A).all() and (q == A).all()
