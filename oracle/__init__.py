"""CPU oracle for the xTGEVC3 path -- TEST INFRASTRUCTURE ONLY.

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU legs of ``bench.py`` import
this package, and only as the checker / CPU baseline.  The product
(``xtgevc3_b200``) never imports it.

Contents
  * ctypes bindings of two CPU implementations with the upstream argument list:
      - ``oracle`` : this repository's C restatement (oracle/tgevc3_oracle.c),
      - ``ref``    : the upstream sources compiled as they are (oracle/_ref, built by
                     ``make -C oracle ref`` where the upstream tree is present);
  * LAPACK from SciPy's bundled OpenBLAS (Fortran interface where SciPy's wrapper drops an
    output) as the oracle of the LAPACK-compatible entry points: xTGEVC, xTREVC3, xTGSNA
    (JOB 'E', 'V', 'B'), xTGEXC and the single swap xTGEX2, xTGSEN, xTGSYL and xGGES with
    ordering;
  * residual checks and the comparison normalisation (the seeded pencil generators live
    in ``xtgevc3_b200.pencils`` and are re-exported here for the tests).
"""
from __future__ import annotations

import ctypes as ct
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "_build", "liboracle_tgevc3.so")
REF_SO = os.path.join(HERE, "_ref", "libref_tgevc3.so")

_libs: dict = {}


def build(ref: bool | str = False) -> None:
    """Compile the C restatement; with ``ref=True`` also the upstream sources (an error
    when they are missing), with ``ref="if-present"`` only where the upstream tree is found
    (its location: the Makefile's REFDIR, overridable by XTGEVC3_REFERENCE_DIR)."""
    subprocess.run(["make", "-s", "-C", HERE, "all"], check=True)
    if ref == "if-present":
        subprocess.run(["make", "-s", "-C", HERE, "ref-if-present"], check=True)
    elif ref:
        subprocess.run(["make", "-s", "-C", HERE, "ref"], check=True)


def _load(path: str, prefix: str):
    lib = ct.CDLL(path)
    P = ct.c_void_p
    I = ct.c_int
    Ch = ct.c_char
    for p in "ds":
        f = getattr(lib, f"{prefix}{p}tgevc3")
        f.argtypes = [Ch, Ch, P, I, P, I, P, I, P, P, P, P, I, P, I, I, P, P, I, P]
        f.restype = None
    for p in "zc":
        f = getattr(lib, f"{prefix}{p}tgevc3")
        f.argtypes = [Ch, Ch, P, I, P, I, P, I, P, P, P, I, P, I, I, P, P, I, P]
        f.restype = None
    return lib


def oracle_lib():
    if "oracle" not in _libs:
        if not os.path.exists(ORACLE_SO):
            build()
        _libs["oracle"] = _load(ORACLE_SO, "oracle_")
    return _libs["oracle"]


def ref_available() -> bool:
    return os.path.exists(REF_SO)


def ref_lib():
    if "ref" not in _libs:
        if not ref_available():
            raise FileNotFoundError(REF_SO)
        lib = _load(REF_SO, "ref_")
        lib.ref_set_num_threads.argtypes = [ct.c_int]
        _libs["ref"] = lib
    return _libs["ref"]


def set_ref_threads(n: int) -> None:
    ref_lib().ref_set_num_threads(int(n))


_PREFIX = {np.float64: "d", np.float32: "s", np.complex128: "z", np.complex64: "c"}


def _ptr(a):
    return None if a is None else a.ctypes.data_as(ct.c_void_p)


def tgevc3(side, howmny, S, P, alpha, beta, alphai=None, VL=None, VR=None, select=None,
           impl="oracle", lwork=None, mm=None):
    """Call ``<impl>_{d,s,z,c}tgevc3`` with the upstream argument list.

    Real pencils pass ``alpha`` = alphar and ``alphai``; complex pencils pass complex
    ``alpha``.  S, P, VL, VR are Fortran-ordered; VL/VR are updated in place (they hold
    Q/Z on entry for HOWMNY='B') and also returned.  Returns (VL, VR, m, info).
    """
    lib = oracle_lib() if impl == "oracle" else ref_lib()
    dt = S.dtype.type
    pfx = _PREFIX[dt]
    n = S.shape[0]
    fn = getattr(lib, f"{'oracle_' if impl == 'oracle' else 'ref_'}{pfx}tgevc3")
    S = np.asfortranarray(S)
    P = np.asfortranarray(P)
    sel = None if select is None else np.ascontiguousarray(select, dtype=np.int32)
    mm = n if mm is None else mm
    if VL is None:
        VL = np.zeros((n, max(mm, 1)), dtype=dt, order="F")
    if VR is None:
        VR = np.zeros((n, max(mm, 1)), dtype=dt, order="F")
    m = ct.c_int(0)
    info = ct.c_int(0)
    q = np.zeros(2, dtype=dt)
    ld = max(n, 1)
    rdt = np.float64 if pfx in "dz" else np.float32
    args_head = [side.encode(), howmny.encode(), _ptr(sel), n, _ptr(S), ld, _ptr(P), ld]
    if pfx in "ds":
        al = np.ascontiguousarray(alpha, dtype=rdt)
        ai = np.ascontiguousarray(alphai, dtype=rdt)
        be = np.ascontiguousarray(beta, dtype=rdt)
        eig = [_ptr(al), _ptr(ai), _ptr(be)]
    else:
        al = np.ascontiguousarray(alpha, dtype=dt)
        be = np.ascontiguousarray(beta, dtype=dt)
        eig = [_ptr(al), _ptr(be)]
    tail = [_ptr(VL), ld, _ptr(VR), ld, mm, ct.byref(m)]
    if lwork is None:
        fn(*args_head, *eig, *tail, _ptr(q), -1, ct.byref(info))
        if info.value != 0:
            return VL, VR, m.value, info.value
        lwork = int(np.real(q[0]))
    work = np.zeros(max(lwork, 1), dtype=dt)
    fn(*args_head, *eig, *tail, _ptr(work), lwork, ct.byref(info))
    return VL, VR, m.value, info.value


from xtgevc3_b200.pencils import (gen_quasi_triangular, gen_upper_triangular_complex,  # noqa: E402,F401
                                  gen_gges, gen_schur_like)


def _openblas():
    if "openblas" not in _libs:
        import glob
        import scipy
        d = os.path.join(os.path.dirname(scipy.__file__), "..", "scipy.libs")
        _libs["openblas"] = ct.CDLL(sorted(glob.glob(os.path.join(d, "libscipy_openblas*.so")))[0])
    return _libs["openblas"]


def lapack_tgevc(S, P):
    """Second oracle: LAPACK xTGEVC (SIDE='B', HOWMNY='A') from SciPy's bundled OpenBLAS,
    called through its Fortran interface.  Returns (VL, VR); LAPACK normalises each
    eigenvector so that max |re| + |im| = 1."""
    dt = S.dtype.type
    pfx = _PREFIX[dt]
    n = S.shape[0]
    f = getattr(_openblas(), f"scipy_{pfx}tgevc_")
    S = np.asfortranarray(S)
    P = np.asfortranarray(P)
    VL = np.zeros((n, n), dtype=dt, order="F")
    VR = np.zeros((n, n), dtype=dt, order="F")
    cplx = pfx in "zc"
    rdt = np.float64 if pfx in "dz" else np.float32
    work = np.zeros(6 * n if not cplx else 2 * n, dtype=dt)
    rwork = np.zeros(2 * n, dtype=rdt)
    iv = lambda v: ct.byref(ct.c_int(v))  # noqa: E731
    m = ct.c_int(0)
    info = ct.c_int(0)
    args = [ct.c_char_p(b"B"), ct.c_char_p(b"A"), None, iv(n), _ptr(S), iv(n), _ptr(P), iv(n), _ptr(VL), iv(n),
            _ptr(VR), iv(n), iv(n), ct.byref(m), _ptr(work)]
    if cplx:
        args.append(_ptr(rwork))
    args += [ct.byref(info), ct.c_size_t(1), ct.c_size_t(1)]
    f(*args)
    if info.value != 0:
        raise RuntimeError(f"{pfx}tgevc info={info.value}")
    return VL, VR


def lapack_trevc3(side, howmny, T, VL=None, VR=None, select=None, mm=None):
    """Oracle of the xTREVC3 entry points: LAPACK xTREVC3 from SciPy's bundled OpenBLAS,
    called through its Fortran interface with the workspace its query asks for.  VL/VR hold
    Q on entry for HOWMNY='B'.  SELECT is copied (LAPACK rewrites a pair's flags).  Returns
    (VL, VR, m, info)."""
    dt = T.dtype.type
    pfx = _PREFIX[dt]
    n = T.shape[0]
    f = getattr(_openblas(), f"scipy_{pfx}trevc3_")
    T = np.asfortranarray(T)
    mm = n if mm is None else mm
    VL = np.zeros((n, max(mm, 1)), dtype=dt, order="F") if VL is None else np.asfortranarray(VL).copy(order="F")
    VR = np.zeros((n, max(mm, 1)), dtype=dt, order="F") if VR is None else np.asfortranarray(VR).copy(order="F")
    sel = np.zeros(max(n, 1), dtype=np.int32) if select is None else np.ascontiguousarray(select, dtype=np.int32).copy()
    cplx = pfx in "zc"
    rdt = np.float64 if pfx in "dz" else np.float32
    iv = lambda v: ct.byref(ct.c_int(v))  # noqa: E731
    m = ct.c_int(0)
    info = ct.c_int(0)

    def call(work, lwork, rwork, lrwork):
        args = [ct.c_char_p(side.encode()), ct.c_char_p(howmny.encode()), _ptr(sel), iv(n), _ptr(T), iv(max(n, 1)),
                _ptr(VL), iv(max(n, 1)), _ptr(VR), iv(max(n, 1)), iv(mm), ct.byref(m), _ptr(work), iv(lwork)]
        if cplx:
            args += [_ptr(rwork), iv(lrwork)]
        args += [ct.byref(info), ct.c_size_t(1), ct.c_size_t(1)]
        f(*args)

    q, rq = np.zeros(2, dtype=dt), np.zeros(2, dtype=rdt)
    call(q, -1, rq, -1)
    if info.value != 0:
        return VL, VR, m.value, info.value
    lwork = max(int(np.real(q[0])), 1)
    lrwork = max(int(rq[0]), n, 1)
    call(np.zeros(lwork, dtype=dt), lwork, np.zeros(lrwork, dtype=rdt), lrwork)
    return VL, VR, m.value, info.value


def lapack_tgsna(howmny, A, B, VL, VR, select=None, job="E"):
    """Oracle of the xTGSNA entry points: LAPACK xTGSNA from SciPy's bundled OpenBLAS.
    JOB = 'E' returns (S, m, info); JOB = 'V' / 'B' returns (S, DIF, m, info) (VL, VR may
    then be None for 'V': not referenced)."""
    dt = A.dtype.type
    pfx = _PREFIX[dt]
    n = A.shape[0]
    f = getattr(_openblas(), f"scipy_{pfx}tgsna_")
    A, B = np.asfortranarray(A), np.asfortranarray(B)
    if VL is None:
        VL = np.zeros((max(n, 1), max(n, 1)), dtype=dt, order="F")
    if VR is None:
        VR = np.zeros((max(n, 1), max(n, 1)), dtype=dt, order="F")
    VL, VR = np.asfortranarray(VL), np.asfortranarray(VR)
    rdt = np.float64 if pfx in "dz" else np.float32
    mm = VR.shape[1]
    sel = np.zeros(max(n, 1), dtype=np.int32) if select is None else np.ascontiguousarray(select, dtype=np.int32).copy()
    S = np.zeros(max(mm, 1), dtype=rdt)
    D = np.zeros(max(mm, 1), dtype=rdt)
    iv = lambda v: ct.byref(ct.c_int(v))  # noqa: E731
    m, info = ct.c_int(0), ct.c_int(0)
    if job == "E":
        lwork = max(n, 1)
    else:
        lwork = max(1, 2 * n * (n + 2) + 16) if pfx in "ds" else max(1, 2 * n * n)
    work = np.zeros(lwork, dtype=dt)
    iwork = np.zeros(n + 6, dtype=np.int32)
    ld = max(n, 1)
    f(ct.c_char_p(job.encode()), ct.c_char_p(howmny.encode()), _ptr(sel), iv(n), _ptr(A), iv(ld), _ptr(B), iv(ld),
      _ptr(VL), iv(ld), _ptr(VR), iv(ld), _ptr(S), _ptr(D), iv(mm), ct.byref(m), _ptr(work), iv(lwork), _ptr(iwork),
      ct.byref(info), ct.c_size_t(1), ct.c_size_t(1))
    if job == "E":
        return S[:m.value], m.value, info.value
    return S[:m.value], D[:m.value], m.value, info.value


def lapack_tgexc(A, B, Q, Z, ifst, ilst):
    """Oracle of the xTGEXC entry points: LAPACK Z/C/D/STGEXC through SciPy (ifst, ilst
    1-based; Q, Z may be None: not updated).  Returns (A, B, Q, Z, info)."""
    import scipy.linalg.lapack as lapack
    dt = A.dtype.type
    f = getattr(lapack, {np.complex128: "ztgexc", np.complex64: "ctgexc", np.float64: "dtgexc",
                         np.float32: "stgexc"}[dt])
    n = A.shape[0]
    wq, wz = Q is not None, Z is not None
    Qa = Q if wq else np.eye(n, dtype=A.dtype)
    Za = Z if wz else np.eye(n, dtype=A.dtype)
    out = f(A, B, Qa, Za, ifst, ilst, wantq=int(wq), wantz=int(wz))
    a, b, q, z, info = out[0], out[1], out[2], out[3], out[-1]  # real forms also return WORK
    return a, b, (q if wq else None), (z if wz else None), info


def lapack_tgexc_ilst(A, B, Q, Z, ifst, ilst):
    """LAPACK ZTGEXC / CTGEXC called through its Fortran interface in SciPy's OpenBLAS, so
    that ILST on exit is returned as well (SciPy's wrapper drops it): on a rejected swap it
    is the row the eigenvalue had reached.  Q, Z are updated (WANTQ = WANTZ = true).
    Returns (A, B, Q, Z, ilst, info)."""
    dt = A.dtype.type
    pfx = {np.complex128: "z", np.complex64: "c"}[dt]
    f = getattr(_openblas(), f"scipy_{pfx}tgexc_")
    n = A.shape[0]
    A, B, Q, Z = (np.asfortranarray(M).copy(order="F") for M in (A, B, Q, Z))
    iv = lambda v: ct.byref(ct.c_int(v))  # noqa: E731
    f_ = ct.c_int(ifst)
    l_ = ct.c_int(ilst)
    info = ct.c_int(0)
    ld = max(n, 1)
    f(iv(1), iv(1), iv(n), _ptr(A), iv(ld), _ptr(B), iv(ld), _ptr(Q), iv(ld), _ptr(Z), iv(ld), ct.byref(f_),
      ct.byref(l_), ct.byref(info))
    return A, B, Q, Z, l_.value, info.value


def _real_fortran_args(A, B, Q, Z):
    n = A.shape[0]
    wq, wz = Q is not None, Z is not None
    A, B = (np.asfortranarray(M).copy(order="F") for M in (A, B))
    Q = np.asfortranarray(Q).copy(order="F") if wq else np.eye(n, dtype=A.dtype, order="F")
    Z = np.asfortranarray(Z).copy(order="F") if wz else np.eye(n, dtype=A.dtype, order="F")
    return n, wq, wz, A, B, Q, Z


def lapack_tgexc_real(A, B, Q, Z, ifst, ilst):
    """LAPACK DTGEXC / STGEXC called through its Fortran interface in SciPy's OpenBLAS, so
    that IFST and ILST on exit are returned too (moved to the first row of their 2x2 blocks;
    on a rejected swap ILST is the row the block had reached).  Q, Z None: WANTQ / WANTZ
    false.  Returns (A, B, Q, Z, ifst, ilst, info)."""
    pfx = {np.float64: "d", np.float32: "s"}[A.dtype.type]
    f = getattr(_openblas(), f"scipy_{pfx}tgexc_")
    n, wq, wz, A, B, Q, Z = _real_fortran_args(A, B, Q, Z)
    iv = lambda v: ct.byref(ct.c_int(v))  # noqa: E731
    f_, l_, info = ct.c_int(ifst), ct.c_int(ilst), ct.c_int(0)
    lwork = 4 * n + 16
    work = np.zeros(lwork, dtype=A.dtype)
    ld = max(n, 1)
    f(iv(int(wq)), iv(int(wz)), iv(n), _ptr(A), iv(ld), _ptr(B), iv(ld), _ptr(Q), iv(ld), _ptr(Z), iv(ld),
      ct.byref(f_), ct.byref(l_), _ptr(work), iv(lwork), ct.byref(info))
    return A, B, (Q if wq else None), (Z if wz else None), f_.value, l_.value, info.value


def lapack_tgex2_real(A, B, Q, Z, j1, n1, n2):
    """LAPACK DTGEX2 / STGEX2 (one swap of the adjacent diagonal blocks of sizes n1, n2 at
    row j1, 1-based) through its Fortran interface in SciPy's OpenBLAS.  Returns (A, B, Q, Z,
    info); info = 1: the swap was rejected and the pencil left as it was."""
    pfx = {np.float64: "d", np.float32: "s"}[A.dtype.type]
    f = getattr(_openblas(), f"scipy_{pfx}tgex2_")
    n, wq, wz, A, B, Q, Z = _real_fortran_args(A, B, Q, Z)
    iv = lambda v: ct.byref(ct.c_int(v))  # noqa: E731
    info = ct.c_int(0)
    lwork = max(1, n * (n1 + n2), 2 * (n1 + n2) ** 2) + 64
    work = np.zeros(lwork, dtype=A.dtype)
    ld = max(n, 1)
    f(iv(int(wq)), iv(int(wz)), iv(n), _ptr(A), iv(ld), _ptr(B), iv(ld), _ptr(Q), iv(ld), _ptr(Z), iv(ld),
      iv(j1), iv(n1), iv(n2), _ptr(work), iv(lwork), ct.byref(info))
    return A, B, (Q if wq else None), (Z if wz else None), info.value


def lapack_tgsyl(trans, ijob, A, B, C, D, E, F):
    """LAPACK D/S/Z/CTGSYL through its Fortran interface in SciPy's OpenBLAS: the generalized
    Sylvester equation A R - L B = scale C, D R - L E = scale F (TRANS = 'N').  Returns (R, L,
    scale, dif, info) (R, L new arrays)."""
    dt = A.dtype.type
    pfx = {np.float64: "d", np.float32: "s", np.complex128: "z", np.complex64: "c"}[dt]
    rt = {np.float64: ct.c_double, np.float32: ct.c_float, np.complex128: ct.c_double, np.complex64: ct.c_float}[dt]
    f = getattr(_openblas(), f"scipy_{pfx}tgsyl_")
    m, n = C.shape
    A, B, D, E = (np.asfortranarray(M).copy(order="F") for M in (A, B, D, E))
    C, F = (np.asfortranarray(M).copy(order="F") for M in (C, F))
    iv = lambda v: ct.byref(ct.c_int(v))  # noqa: E731
    scale, dif, info = rt(0), rt(0), ct.c_int(0)
    lwork = max(1, 2 * m * n)
    work = np.zeros(lwork, dtype=dt)
    iwork = np.zeros(m + n + 6, dtype=np.int32)
    f(ct.c_char_p(trans.encode()), iv(ijob), iv(m), iv(n), _ptr(A), iv(max(m, 1)), _ptr(B), iv(max(n, 1)), _ptr(C),
      iv(max(m, 1)), _ptr(D), iv(max(m, 1)), _ptr(E), iv(max(n, 1)), _ptr(F), iv(max(m, 1)), ct.byref(scale),
      ct.byref(dif), _ptr(work), iv(lwork), _ptr(iwork), ct.byref(info), ct.c_size_t(1))
    return C, F, scale.value, dif.value, info.value


def lapack_tgsen0(select, A, B, Q, Z):
    """LAPACK x TGSEN with IJOB = 0 (SciPy's wrapper of D/S/Z/CTGSEN): the eigenvalues that
    select flags move to the leading rows of the generalized Schur pencil (A, B), Q and Z
    updated.  Returns (A, B, eigenvalue arrays..., Q, Z, m, info): real (alphar, alphai, beta),
    complex (alpha, beta)."""
    import scipy.linalg.lapack as la
    pfx = {np.float64: "d", np.float32: "s", np.complex128: "z", np.complex64: "c"}[A.dtype.type]
    sel = np.asarray(select, dtype=np.int32)
    r = getattr(la, f"{pfx}tgsen")(sel, A, B, Q, Z, ijob=0)
    if pfx in "ds":
        a, b, ar, ai, be, q, z, m, _, _, _, info = r
        return a, b, ar, ai, be, q, z, int(m), int(info)
    a, b, al, be, q, z, m, _, _, _, info = r
    return a, b, al, be, q, z, int(m), int(info)


def lapack_gges_sort(A, B, sort):
    """LAPACK xGGES with SORT = 'S' (SciPy's wrapper), sort a predicate as SELCTG (real:
    sort(alphar, alphai, beta), complex: sort(alpha, beta)).  Returns (S, T, sdim, eigenvalue
    arrays..., VSL, VSR, info)."""
    import scipy.linalg.lapack as la
    pfx = {np.float64: "d", np.float32: "s", np.complex128: "z", np.complex64: "c"}[A.dtype.type]
    f = getattr(la, f"{pfx}gges")
    if pfx in "ds":  # f2py passes as many values as the callback names
        r = f(lambda ar, ai, b: int(bool(sort(ar, ai, b))), A, B, sort_t=1)
    else:
        r = f(lambda a, b: int(bool(sort(a, b))), A, B, sort_t=1)
    return tuple(x for i, x in enumerate(r) if i != len(r) - 2)  # work dropped


def complex_schur_pencil(n, seed, dtype=np.complex128):
    """Complex generalized Schur form (LAPACK xGGES through SciPy's qz) of a pencil with iid
    complex N(0,1) entries: returns (A, B, Q, Z) with the original pencil = (Q A Z^H, Q B Z^H)."""
    import scipy.linalg
    rng = np.random.default_rng(seed)
    a = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
    b = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
    AA, BB, Q, Z = scipy.linalg.qz(a.astype(dtype), b.astype(dtype), output="complex")
    return tuple(np.asfortranarray(M.astype(dtype)) for M in (AA, BB, Q, Z))


def schur_real(n, seed, dtype=np.float64):
    """Real Schur form of an iid N(0,1) matrix (LAPACK xGEES through SciPy: T quasi-upper
    triangular with standardised 2x2 blocks, Q orthogonal)."""
    import scipy.linalg
    A = np.random.default_rng(seed).standard_normal((n, n))
    T, Q = scipy.linalg.schur(A.astype(dtype), output="real")
    return np.asfortranarray(T), np.asfortranarray(Q)


def schur_complex(n, seed, dtype=np.complex128):
    """Complex Schur form of an iid complex N(0,1) matrix (LAPACK xGEES through SciPy)."""
    import scipy.linalg
    rng = np.random.default_rng(seed)
    A = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
    T, Q = scipy.linalg.schur(A.astype(dtype), output="complex")
    return np.asfortranarray(T), np.asfortranarray(Q)


# --------------------------------------------------------------------------------------
# residuals and normalisation
# --------------------------------------------------------------------------------------

def eig_columns(alphai, n_cols=None):
    """Yield (col, is_pair) for real eigenvector storage: a pair occupies (Re, Im) columns."""
    k = 0
    n = len(alphai) if n_cols is None else n_cols
    while k < n:
        pair = alphai[k] != 0 and k + 1 < len(alphai)
        yield k, pair
        k += 2 if pair else 1


def selected_items(n, howmny, select=None, alphai=None):
    """(k, is_pair) of every computed eigenvector in output order (upstream selection rule,
    src/dtgevc3.cpp:1193-1207: a pair counts when either flag is set)."""
    items = []
    k = 0
    while k < n:
        pair = alphai is not None and alphai[k] != 0 and k + 1 < n
        sel = howmny in ("A", "B")
        if howmny == "S" and select is not None:
            sel = bool(select[k]) or (pair and bool(select[k + 1]))
        if sel:
            items.append((k, pair))
        k += 2 if pair else 1
    return items


def to_complex_real_storage(V, alphai, howmny="A", select=None):
    """Real (Re, Im)-pair storage -> complex matrix with one column per eigenvalue
    (a pair's second column becomes the conjugate eigenvector)."""
    n, m = V.shape
    W = V.astype(np.complex128)
    c = 0
    for k, pair in selected_items(len(alphai), howmny, select, alphai):
        if c >= m:
            break
        if pair:
            W[:, c] = V[:, c] + 1j * V[:, c + 1]
            W[:, c + 1] = V[:, c] - 1j * V[:, c + 1]
            c += 2
        else:
            c += 1
    return W


def column_eigenvalues(alpha, beta, howmny="A", select=None, alphai=None):
    """(alpha, beta) of each output column, complex alpha for real pencils."""
    n = len(beta)
    a = np.asarray(alpha) + (1j * np.asarray(alphai) if alphai is not None else 0)
    idx = []
    for k, pair in selected_items(n, howmny, select, alphai):
        idx += [k, k + 1] if pair else [k]
    idx = np.array(idx, dtype=int)
    return a[idx], np.asarray(beta)[idx]


def residual_ratio(S, P, V, alpha, beta, left=False):
    """Per column: ||beta*S*v - alpha*P*v||_1 / ((|beta|*||S||_1 + |alpha|*||P||_1) * ||v||_1) / eps,
    the DGET52-style measure of tests/test_lapack_d.cpp:38-168 (complex V, complex alpha)."""
    eps = np.finfo(np.float64 if V.real.dtype == np.float64 else np.float32).eps
    S = S.astype(np.complex128)
    P = P.astype(np.complex128)
    V = V.astype(np.complex128)
    # the ratio is invariant under (S, alpha) -> (S, alpha)/s and (P, beta) -> (P, beta)/p;
    # working with unit-norm S, P keeps pencils scaled near overflow finite here
    nS0 = max(np.abs(S).sum(0).max(), 1e-300)
    nP0 = max(np.abs(P).sum(0).max(), 1e-300)
    S, alpha = S / nS0, np.asarray(alpha) / nS0
    P, beta = P / nP0, np.asarray(beta) / nP0
    V = V / np.maximum(np.abs(V).max(0), 1e-300)[None, :]
    nS = nP = 1.0
    if left:
        R = (S.conj().T @ V) * np.conj(beta)[None, :] - (P.conj().T @ V) * np.conj(alpha)[None, :]
    else:
        R = (S @ V) * beta[None, :] - (P @ V) * alpha[None, :]
    nv = np.abs(V).sum(0)
    nv[nv == 0] = 1.0
    den = (np.abs(beta) * nS + np.abs(alpha) * nP) * nv
    den = np.maximum(den, np.finfo(np.float64).tiny)
    return np.abs(R).sum(0) / den / eps


def normalize_like(V, Vref):
    """Scale each complex column of V and Vref by their value at the row where |Vref| is
    largest, so both carry the same (scale, phase) convention.  Returns (V', Vref')."""
    idx = np.argmax(np.abs(Vref), axis=0)
    cols = np.arange(V.shape[1])
    a = V[idx, cols]
    b = Vref[idx, cols]
    a = np.where(a == 0, 1, a)
    b = np.where(b == 0, 1, b)
    return V / a[None, :], Vref / b[None, :]


def max_rel_diff(V, Vref):
    """Max over columns of max|v - vref| / max|vref| after ``normalize_like``; also
    returns the per-column array.  Non-finite reference columns are reported as nan."""
    Vn, Rn = normalize_like(V, Vref)
    num = np.abs(Vn - Rn).max(0)
    den = np.abs(Rn).max(0)
    den[den == 0] = 1.0
    err = num / den
    bad = ~np.isfinite(Vref).all(0)
    err[bad] = np.nan
    return (np.nanmax(err) if np.isfinite(err).any() else 0.0), err
