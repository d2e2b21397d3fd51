"""xtgevc3_b200 -- generalized eigenvectors of a (quasi-)triangular pencil on NVIDIA B200.

Python view of the C ABI in include/xtgevc3.h (libxtgevc3.so, built by
``python -m xtgevc3_b200.build``).  Two call forms:

``tgevc3(side, howmny, S, P, alpha, beta, alphai=..., VL=..., VR=..., select=...)``
    The upstream argument list (include/tgevc3.h:9-12 of vlovero/xTGEVC3) on host
    (numpy, Fortran-ordered) arrays; calls the drop-in entry point
    ``xtgevc3_{d,s,z,c}tgevc3``.  Returns (VL, VR, m, info).

``tgevc3_dev(side, howmny, S, P, alpha, beta, alphai=..., VL=..., VR=..., select=..., flags=0)``
    Matrices are CUDA tensors in column-major layout (``stride(0) == 1``, e.g.
    ``torch.empty(n, n, device='cuda').t()``); eigenvalue arrays / select stay on the host.
    Calls ``xtgevc3_{d,s,z,c}tgevc3_dev`` on torch's current stream.  Returns (m, info).

There is no CPU fallback: importing the package loads the CUDA library and raises if it
cannot be loaded or built.
"""
from __future__ import annotations

import ctypes as ct
import os

import numpy as np

from . import build as _build

NORMALIZE = 1
SIMT = 2
SPLIT = 4
SPLIT_INT8 = 8
LOOKAHEAD = 16
SPLIT_CRT = 32
SPLIT_NO_REFINE = 64


def split_refined() -> int:
    """Eigenvector columns the calling thread's last split-form call solved again in FP64."""
    return int(lib().xtgevc3_split_refined())


def slices(s: int) -> int:
    """Flag bits selecting s slices for the SPLIT form (BF16: 1..6, INT8: 1..7) or the
    modulus count of the residue form (SPLIT_CRT: 2..16)."""
    return int(s) << 8


def split_gemm(kind, A, B, C=None, accumulate=False, slices=0, stream=None):
    """C (+)= A B through a split-precision tensor-core path (xtgevc3_split_gemm_dev): kind 0
    BF16 slices, 1 INT8 digit slices, 2 INT8 residues.  A, B, C: column-major float64 CUDA
    tensors (C allocated when None).  Returns C."""
    import torch
    M, K = A.shape
    N = B.shape[1]
    if C is None:
        C = torch.zeros(N, M, dtype=torch.float64, device=A.device).t()
    ap, lda = _colmajor(A)
    bp, ldb = _colmajor(B)
    cp, ldc = _colmajor(C)
    st = ct.c_void_p(stream if stream is not None else torch.cuda.current_stream().cuda_stream)
    rc = lib().xtgevc3_split_gemm_dev(st, int(kind), int(slices), M, N, K, ap, lda, bp, ldb, cp, ldc,
                                      int(bool(accumulate)))
    if rc != 0:
        raise RuntimeError(f"xtgevc3_split_gemm_dev failed ({rc}): {last_error()}")
    return C

_HERE = os.path.dirname(os.path.abspath(__file__))
_lib = None

_P = ct.c_void_p
_I = ct.c_int
_C = ct.c_char
# SELCTG of xGGES (include/xtgevc3.h: xtgevc3_dselect3 ... xtgevc3_cselect2)
_SELECT = {
    "d": ct.CFUNCTYPE(ct.c_int, ct.POINTER(ct.c_double), ct.POINTER(ct.c_double), ct.POINTER(ct.c_double)),
    "s": ct.CFUNCTYPE(ct.c_int, ct.POINTER(ct.c_float), ct.POINTER(ct.c_float), ct.POINTER(ct.c_float)),
    "z": ct.CFUNCTYPE(ct.c_int, ct.POINTER(ct.c_double), ct.POINTER(ct.c_double)),
    "c": ct.CFUNCTYPE(ct.c_int, ct.POINTER(ct.c_float), ct.POINTER(ct.c_float)),
}
_U = ct.c_uint


def lib():
    """The loaded libxtgevc3.so (built on first use if it is missing)."""
    global _lib
    if _lib is None:
        path = _build.LIB
        if not os.path.exists(path):
            _build.build()
        L = ct.CDLL(path)
        for p in "ds":
            f = getattr(L, f"xtgevc3_{p}tgevc3")
            f.argtypes = [_C, _C, _P, _I, _P, _I, _P, _I, _P, _P, _P, _P, _I, _P, _I, _I, _P, _P, _I, _P]
            f.restype = None
            f = getattr(L, f"xtgevc3_{p}tgevc3_dev")
            f.argtypes = [_U, _P, _C, _C, _P, _I, _P, _I, _P, _I, _P, _P, _P, _P, _I, _P, _I, _I, _P, _P]
            f.restype = _I
        for p in "zc":
            f = getattr(L, f"xtgevc3_{p}tgevc3")
            f.argtypes = [_C, _C, _P, _I, _P, _I, _P, _I, _P, _P, _P, _I, _P, _I, _I, _P, _P, _I, _P]
            f.restype = None
            f = getattr(L, f"xtgevc3_{p}tgevc3_dev")
            f.argtypes = [_U, _P, _C, _C, _P, _I, _P, _I, _P, _I, _P, _P, _P, _I, _P, _I, _I, _P, _P]
            f.restype = _I
        for p in "ds":  # xTREVC3
            f = getattr(L, f"xtgevc3_{p}trevc3")
            f.argtypes = [_C, _C, _P, _I, _P, _I, _P, _I, _P, _I, _I, _P, _P, _I, _P]
            f.restype = None
        for p in "zc":
            f = getattr(L, f"xtgevc3_{p}trevc3")
            f.argtypes = [_C, _C, _P, _I, _P, _I, _P, _I, _P, _I, _I, _P, _P, _I, _P, _I, _P]
            f.restype = None
        for p in "dszc":  # xTGSNA (JOB = 'E')
            f = getattr(L, f"xtgevc3_{p}tgsna")
            f.argtypes = [_C, _C, _P, _I, _P, _I, _P, _I, _P, _I, _P, _I, _P, _P, _I, _P, _P, _I, _P, _P]
            f.restype = None
            f = getattr(L, f"xtgevc3_{p}tgsna_dev")
            f.argtypes = [_P, _C, _C, _P, _I, _P, _I, _P, _I, _P, _I, _P, _I, _P, _I, _P, _P]
            f.restype = _I
        for p in "zc":  # generalized Schur form of a complex pencil (xGGES, no ordering)
            f = getattr(L, f"xtgevc3_{p}gges")
            f.argtypes = [_C, _C, _I, _P, _I, _P, _I, _P, _P, _P, _I, _P, _I, _P]
            f.restype = None
            f = getattr(L, f"xtgevc3_{p}gges_dev")
            f.argtypes = [_P, _C, _C, _I, _P, _I, _P, _I, _P, _P, _P, _I, _P, _I, _P]
            f.restype = _I
        for p in "ds":  # real pencils: alphar, alphai, beta
            f = getattr(L, f"xtgevc3_{p}gges")
            f.argtypes = [_C, _C, _I, _P, _I, _P, _I, _P, _P, _P, _P, _I, _P, _I, _P]
            f.restype = None
            f = getattr(L, f"xtgevc3_{p}gges_dev")
            f.argtypes = [_P, _C, _C, _I, _P, _I, _P, _I, _P, _P, _P, _P, _I, _P, _I, _P]
            f.restype = _I
        for p in "zcds":  # xGGES with ordering: SORT, SELCTG, SDIM in LAPACK's positions
            sel = _SELECT[p]
            nv = 2 if p in "zc" else 3
            f = getattr(L, f"xtgevc3_{p}gges_sort")
            f.argtypes = [_C, _C, _C, sel, _I, _P, _I, _P, _I, _P] + [_P] * nv + [_P, _I, _P, _I, _P]
            f.restype = None
            f = getattr(L, f"xtgevc3_{p}gges_sort_dev")
            f.argtypes = [_P, _C, _C, _C, sel, _I, _P, _I, _P, _I, _P] + [_P] * nv + [_P, _I, _P, _I, _P]
            f.restype = _I
        for p in "dszc":  # xTGSEN: ..., M, PL, PR, DIF, INFO
            nv = 2 if p in "zc" else 3
            f = getattr(L, f"xtgevc3_{p}tgsen")
            f.argtypes = [_I, _I, _I, _P, _I, _P, _I, _P, _I] + [_P] * nv + [_P, _I, _P, _I, _P, _P, _P, _P, _P]
            f.restype = None
            f = getattr(L, f"xtgevc3_{p}tgsen_dev")
            f.argtypes = [_P, _I, _I, _I, _P, _I, _P, _I, _P, _I] + [_P] * nv + [_P, _I, _P, _I, _P, _P, _P, _P, _P]
            f.restype = _I
        for p in "dszc":  # xTGSYL (TRANS = 'N')
            f = getattr(L, f"xtgevc3_{p}tgsyl")
            f.argtypes = [_C, _I, _I, _I] + [_P, _I] * 6 + [_P, _P, _P]
            f.restype = None
            f = getattr(L, f"xtgevc3_{p}tgsyl_dev")
            f.argtypes = [_P, _C, _I, _I, _I] + [_P, _I] * 6 + [_P, _P, _P]
            f.restype = _I
        for p in "dszc":  # xGGBAL / xGGBAK (JOB 'N' or 'P')
            f = getattr(L, f"xtgevc3_{p}ggbal")
            f.argtypes = [_C, _I, _P, _I, _P, _I, _P, _P, _P, _P, _P]
            f.restype = None
            f = getattr(L, f"xtgevc3_{p}ggbak")
            f.argtypes = [_C, _C, _I, _I, _I, _P, _P, _I, _P, _I, _P]
            f.restype = None
        for p in "dszc":  # xTGSNA DIF on the device
            f = getattr(L, f"xtgevc3_{p}tgsna_dif_dev")
            f.argtypes = [_P, _C, _P, _I, _P, _I, _P, _I, _P, _I, _P, _P]
            f.restype = _I
        for p in "zc":  # xTGEXC, complex pencils
            f = getattr(L, f"xtgevc3_{p}tgexc")
            f.argtypes = [_I, _I, _I, _P, _I, _P, _I, _P, _I, _P, _I, _I, _P, _P]
            f.restype = None
            f = getattr(L, f"xtgevc3_{p}tgexc_dev")
            f.argtypes = [_P, _I, _I, _I, _P, _I, _P, _I, _P, _I, _P, _I, _I, _P, _P]
            f.restype = _I
        for p in "ds":  # xTGEXC, real pencils: IFST in and out
            f = getattr(L, f"xtgevc3_{p}tgexc")
            f.argtypes = [_I, _I, _I, _P, _I, _P, _I, _P, _I, _P, _I, _P, _P, _P]
            f.restype = None
            f = getattr(L, f"xtgevc3_{p}tgexc_dev")
            f.argtypes = [_P, _I, _I, _I, _P, _I, _P, _I, _P, _I, _P, _I, _P, _P, _P]
            f.restype = _I
        for p in "dszc":
            f = getattr(L, f"xtgevc3_{p}trevc3_dev")
            f.argtypes = [_U, _P, _C, _C, _P, _I, _P, _I, _P, _I, _P, _I, _I, _P, _P]
            f.restype = _I
        L.xtgevc3_set_flags.argtypes = [_U]
        L.xtgevc3_set_flags.restype = None
        L.xtgevc3_get_flags.restype = _U
        L.xtgevc3_last_error.restype = ct.c_char_p
        L.xtgevc3_trace_enable.argtypes = [_I]
        L.xtgevc3_trace_enable.restype = None
        L.xtgevc3_trace_reset.restype = None
        L.xtgevc3_trace_get.argtypes = [_I, _P, _P, _P, _P]
        L.xtgevc3_trace_get.restype = _I
        L.xtgevc3_trace_name.argtypes = [_I]
        L.xtgevc3_trace_name.restype = ct.c_char_p
        L.xtgevc3_launch_count.restype = ct.c_longlong
        L.xtgevc3_dtgevc3_dev_noalloc.argtypes = [_P, _C, _C, _P, _I, _P, _I, _P, _I, _P, _P, _P, _P, _I, _P, _I,
                                                  _I, _P, _P]
        L.xtgevc3_dtgevc3_dev_noalloc.restype = _I
        for p in "ds":
            f = getattr(L, f"xtgevc3_{p}tgevc3_batched_create")
            f.argtypes = [_C, _C, _I, _P, _U, _P]
            f.restype = _I
            f = getattr(L, f"xtgevc3_{p}tgevc3_batched_tune")
            f.argtypes = [_C, _C, _I, _P, _I, _P, _P]
            f.restype = _I
        L.xtgevc3_batched_run.argtypes = [_P, _P]
        L.xtgevc3_batched_run.restype = _I
        L.xtgevc3_batched_wait.argtypes = [_P, _P]
        L.xtgevc3_batched_wait.restype = _I
        L.xtgevc3_batched_destroy.argtypes = [_P]
        L.xtgevc3_batched_destroy.restype = None
        L.xtgevc3_batched_info.argtypes = [_P, _P, _P, _P]
        L.xtgevc3_batched_info.restype = _I
        L.xtgevc3_batched_set_default.argtypes = [_C, _U]
        L.xtgevc3_batched_set_default.restype = None
        L.xtgevc3_batched_get_default.argtypes = [_C]
        L.xtgevc3_batched_get_default.restype = _U
        _lib = L
    return _lib


def trace_enable(on: bool = True) -> None:
    """Time every library kernel with CUDA events (per kernel class; see trace())."""
    lib().xtgevc3_trace_enable(1 if on else 0)


def trace_reset() -> None:
    lib().xtgevc3_trace_reset()


def trace() -> dict:
    """{class name: {launches, ms, flops, bytes}} accumulated since trace_reset()."""
    out = {}
    L = lib()
    for cls in range(16):
        n = ct.c_longlong(0)
        ms = ct.c_double(0)
        fl = ct.c_double(0)
        by = ct.c_double(0)
        if L.xtgevc3_trace_get(cls, ct.byref(n), ct.byref(ms), ct.byref(fl), ct.byref(by)) != 0:
            break
        out[L.xtgevc3_trace_name(cls).decode()] = dict(launches=n.value, ms=ms.value, flops=fl.value,
                                                        bytes=by.value)
    return out


def launch_count() -> int:
    """Kernels launched by the library so far in this process."""
    return int(lib().xtgevc3_launch_count())


def set_flags(flags: int) -> None:
    """Flags used by the host-pointer (drop-in) entry points (NORMALIZE, SIMT)."""
    lib().xtgevc3_set_flags(int(flags))


def get_flags() -> int:
    return int(lib().xtgevc3_get_flags())


def last_error() -> str:
    return lib().xtgevc3_last_error().decode()


_PFX = {np.float64: "d", np.float32: "s", np.complex128: "z", np.complex64: "c"}


def _ptr(a):
    return None if a is None else a.ctypes.data_as(_P)


def lwork_query(prefix: str, n: int) -> int:
    """The upstream LWORK=-1 answer for order n (2n(b+1) + 4(b+1)^2 + 2(b+1), b = 32)."""
    b = 32
    return 2 * n * (b + 1) + 4 * (b + 1) ** 2 + 2 * (b + 1)


def tgevc3(side, howmny, S, P, alpha, beta, alphai=None, VL=None, VR=None, select=None, mm=None, lwork=None):
    """Host-array form of s/d/c/ztgevc3 (see module docstring).  VL/VR are updated in place."""
    L = lib()
    dt = S.dtype.type
    pfx = _PFX[dt]
    n = S.shape[0]
    S = np.asfortranarray(S)
    P = np.asfortranarray(P)
    sel = None if select is None else np.ascontiguousarray(select, dtype=np.int32)
    mm = n if mm is None else mm
    if VL is None:
        VL = np.zeros((n, max(mm, 1)), dtype=dt, order="F")
    if VR is None:
        VR = np.zeros((n, max(mm, 1)), dtype=dt, order="F")
    assert VL.flags.f_contiguous and VR.flags.f_contiguous
    m = ct.c_int(0)
    info = ct.c_int(0)
    ld = max(n, 1)
    rdt = np.float64 if pfx in "dz" else np.float32
    head = [side.encode(), howmny.encode(), _ptr(sel), n, _ptr(S), ld, _ptr(P), ld]
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
    fn = getattr(L, f"xtgevc3_{pfx}tgevc3")
    if lwork is None:
        q = np.zeros(2, dtype=dt)
        fn(*head, *eig, *tail, _ptr(q), -1, ct.byref(info))
        if info.value != 0:
            return VL, VR, m.value, info.value
        lwork = int(np.real(q[0]))
    work = np.zeros(max(min(lwork, 4), 1), dtype=dt)  # the GPU path never touches WORK beyond the query
    fn(*head, *eig, *tail, _ptr(work), lwork, ct.byref(info))
    if info.value > 0:
        raise RuntimeError(f"xtgevc3_{pfx}tgevc3 failed: {last_error()}")
    return VL, VR, m.value, info.value


def _colmajor(t):
    """(pointer, leading dimension) of a column-major 2-D CUDA tensor."""
    if t is None:
        return None, 1
    if t.dim() != 2 or t.stride(0) != 1:
        raise ValueError("matrices must be column-major (stride(0) == 1), e.g. torch.empty(n, n).t()")
    return ct.c_void_p(t.data_ptr()), max(t.stride(1), t.shape[0], 1)


def tgevc3_dev(side, howmny, S, P, alpha, beta, alphai=None, VL=None, VR=None, select=None, flags=0,
               stream=None):
    """Device form (see module docstring).  Raises on CUDA failure; returns (m, info)."""
    import torch
    L = lib()
    tdt = S.dtype
    pfx = {torch.float64: "d", torch.float32: "s", torch.complex128: "z", torch.complex64: "c"}[tdt]
    n = S.shape[0]
    sp, lds = _colmajor(S)
    pp, ldp = _colmajor(P)
    vlp, ldvl = _colmajor(VL)
    vrp, ldvr = _colmajor(VR)
    mm = max(VL.shape[1] if VL is not None else 0, VR.shape[1] if VR is not None else 0)
    sel = None if select is None else np.ascontiguousarray(select, dtype=np.int32)
    rdt = np.float64 if pfx in "dz" else np.float32
    cdt = np.complex128 if pfx == "z" else np.complex64
    if stream is None:
        stream = torch.cuda.current_stream().cuda_stream
    m = ct.c_int(0)
    info = ct.c_int(0)
    head = [int(flags), ct.c_void_p(stream), side.encode(), howmny.encode(), _ptr(sel), n, sp, lds, pp, ldp]
    if pfx in "ds":
        al = np.ascontiguousarray(alpha, dtype=rdt)
        ai = np.ascontiguousarray(alphai, dtype=rdt)
        be = np.ascontiguousarray(beta, dtype=rdt)
        eig = [_ptr(al), _ptr(ai), _ptr(be)]
    else:
        al = np.ascontiguousarray(alpha, dtype=cdt)
        be = np.ascontiguousarray(beta, dtype=cdt)
        eig = [_ptr(al), _ptr(be)]
    rc = getattr(L, f"xtgevc3_{pfx}tgevc3_dev")(*head, *eig, vlp, ldvl, vrp, ldvr, mm, ct.byref(m), ct.byref(info))
    if rc != 0:
        raise RuntimeError(f"xtgevc3_{pfx}tgevc3_dev failed: {last_error()}")
    return m.value, info.value


# ---- standard problem (xTREVC3) ------------------------------------------------------------
def trevc3(side, howmny, T, VL=None, VR=None, select=None, mm=None, lwork=None):
    """Host-array form of s/d/c/ztrevc3: eigenvectors of the quasi-triangular Schur factor T
    with LAPACK xTREVC3's conventions (include/xtgevc3.h).  VL/VR (Q on entry for
    HOWMNY='B') are updated in place.  Returns (VL, VR, m, info)."""
    L = lib()
    dt = T.dtype.type
    pfx = _PFX[dt]
    n = T.shape[0]
    T = np.asfortranarray(T)
    sel = None if select is None else np.ascontiguousarray(select, dtype=np.int32)
    mm = n if mm is None else mm
    if VL is None:
        VL = np.zeros((n, max(mm, 1)), dtype=dt, order="F")
    if VR is None:
        VR = np.zeros((n, max(mm, 1)), dtype=dt, order="F")
    assert VL.flags.f_contiguous and VR.flags.f_contiguous
    m, info = ct.c_int(0), ct.c_int(0)
    ld = max(n, 1)
    fn = getattr(L, f"xtgevc3_{pfx}trevc3")
    head = [side.encode(), howmny.encode(), _ptr(sel), n, _ptr(T), ld, _ptr(VL), ld, _ptr(VR), ld, mm, ct.byref(m)]
    rdt = np.float64 if pfx in "dz" else np.float32
    q, rq = np.zeros(2, dtype=dt), np.zeros(2, dtype=rdt)
    if lwork is None:
        extra = [_ptr(rq), -1] if pfx in "zc" else []
        fn(*head, _ptr(q), -1, *extra, ct.byref(info))
        if info.value != 0:
            return VL, VR, m.value, info.value
        lwork = int(np.real(q[0]))
    lrwork = max(n, 1)
    work = np.zeros(max(min(lwork, 4), 1), dtype=dt)  # the GPU path never touches WORK beyond the query
    rwork = np.zeros(1, dtype=rdt)
    extra = [_ptr(rwork), lrwork] if pfx in "zc" else []
    fn(*head, _ptr(work), lwork, *extra, ct.byref(info))
    if info.value > 0:
        raise RuntimeError(f"xtgevc3_{pfx}trevc3 failed: {last_error()}")
    return VL, VR, m.value, info.value


def trevc3_dev(side, howmny, T, VL=None, VR=None, select=None, flags=0, stream=None):
    """Device form of xTREVC3 on column-major CUDA tensors.  Raises on CUDA failure;
    returns (m, info)."""
    import torch
    L = lib()
    pfx = {torch.float64: "d", torch.float32: "s", torch.complex128: "z", torch.complex64: "c"}[T.dtype]
    n = T.shape[0]
    tp, ldt = _colmajor(T)
    vlp, ldvl = _colmajor(VL)
    vrp, ldvr = _colmajor(VR)
    mm = max(VL.shape[1] if VL is not None else 0, VR.shape[1] if VR is not None else 0)
    sel = None if select is None else np.ascontiguousarray(select, dtype=np.int32)
    if stream is None:
        stream = torch.cuda.current_stream().cuda_stream
    m, info = ct.c_int(0), ct.c_int(0)
    rc = getattr(L, f"xtgevc3_{pfx}trevc3_dev")(int(flags), ct.c_void_p(stream), side.encode(), howmny.encode(),
                                                 _ptr(sel), n, tp, ldt, vlp, ldvl, vrp, ldvr, mm, ct.byref(m),
                                                 ct.byref(info))
    if rc != 0:
        raise RuntimeError(f"xtgevc3_{pfx}trevc3_dev failed: {last_error()}")
    return m.value, info.value


def tgsna(howmny, A, B, VL, VR, select=None, job="E"):
    """Host-array form of s/d/c/ztgsna.  JOB = 'E': reciprocal condition numbers S of the
    selected eigenvalues of the Schur pencil (A, B) from its eigenvectors VL, VR (Schur
    coordinates, as tgevc3 returns them with HOWMNY 'A' or 'S'); returns (S, m, info).
    JOB = 'V' / 'B': also the eigenvector condition estimates DIF; returns (S, DIF, m, info)
    with S None for 'V' (VL, VR may then be None)."""
    L = lib()
    dt = A.dtype.type
    pfx = _PFX[dt]
    n = A.shape[0]
    A, B = np.asfortranarray(A), np.asfortranarray(B)
    wants = job != "V"
    if VL is None or VR is None:
        VL = VR = np.zeros((max(n, 1), max(n, 1)), dtype=dt, order="F")
    VL, VR = np.asfortranarray(VL), np.asfortranarray(VR)
    rdt = np.float64 if pfx in "dz" else np.float32
    mm = VR.shape[1]
    sel = None if select is None else np.ascontiguousarray(select, dtype=np.int32)
    S = np.zeros(max(mm, 1), dtype=rdt)
    D = np.zeros(max(mm, 1), dtype=rdt)
    m, info = ct.c_int(0), ct.c_int(0)
    lwork = max(n, 1) if job == "E" else max(1, 2 * n * (n + 2) + 16 if pfx in "ds" else 2 * n * n)
    work = np.zeros(lwork, dtype=dt)
    ld = max(n, 1)
    getattr(L, f"xtgevc3_{pfx}tgsna")(job.encode(), howmny.encode(), _ptr(sel), n, _ptr(A), ld, _ptr(B), ld, _ptr(VL),
                                      max(VL.shape[0], 1), _ptr(VR), max(VR.shape[0], 1), _ptr(S), _ptr(D), mm,
                                      ct.byref(m), _ptr(work), lwork, None, ct.byref(info))
    if info.value > 0:
        raise RuntimeError(f"xtgevc3_{pfx}tgsna failed: {last_error()}")
    if job == "E":
        return S[:m.value], m.value, info.value
    return (S[:m.value] if wants else None), D[:m.value], m.value, info.value


def tgsna_dif_dev(A, B, howmny="A", select=None, stream=None):
    """Device form of the DIF estimates (xTGSNA with JOB = 'V') on column-major CUDA
    tensors.  Returns (DIF as a real CUDA tensor of m entries, m, info)."""
    import torch
    L = lib()
    pfx = {torch.float64: "d", torch.float32: "s", torch.complex128: "z", torch.complex64: "c"}[A.dtype]
    rdt = {"d": torch.float64, "s": torch.float32, "z": torch.float64, "c": torch.float32}[pfx]
    n = A.shape[0]
    st = ct.c_void_p(stream if stream is not None else torch.cuda.current_stream().cuda_stream)
    sel = None if select is None else np.ascontiguousarray(select, dtype=np.int32)
    dif = torch.zeros(max(n, 1), dtype=rdt, device=A.device)
    m, info = ct.c_int(0), ct.c_int(0)
    rc = getattr(L, f"xtgevc3_{pfx}tgsna_dif_dev")(st, howmny.encode(), _ptr(sel), n, ct.c_void_p(A.data_ptr()),
                                                  max(A.stride(1), 1), ct.c_void_p(B.data_ptr()), max(B.stride(1), 1),
                                                  ct.c_void_p(dif.data_ptr()), max(n, 1), ct.byref(m), ct.byref(info))
    if rc:
        raise RuntimeError(f"xtgevc3_{pfx}tgsna_dif_dev failed: {last_error()}")
    return dif[:m.value], m.value, info.value


def _selctg(pfx, sort):
    """The C SELCTG for a Python predicate: real sort(alphar, alphai, beta), complex
    sort(alpha, beta) (Python floats / complex numbers) -> truth value; a NULL pointer for None."""
    typ = _SELECT[pfx]
    if sort is None:
        return typ()
    if pfx in "zc":
        return typ(lambda a, b: 1 if sort(complex(a[0], a[1]), complex(b[0], b[1])) else 0)
    return typ(lambda ar, ai, b: 1 if sort(ar[0], ai[0], b[0]) else 0)


def gges(A, B, jobvsl="V", jobvsr="V", sort=None):
    """Host-array form of z/c/d/sgges: the generalized Schur form of the pencil (A, B),
    A = VSL S VSR^H, B = VSL T VSR^H.  Complex: returns (S, T, alpha, beta, VSL, VSR, info);
    real: (S, T, alphar, alphai, beta, VSL, VSR, info).  New arrays; VSL / VSR None for 'N'.
    With sort (a predicate: real sort(alphar, alphai, beta), complex sort(alpha, beta)) the
    eigenvalues it selects lead (xGGES with SORT = 'S', xtgevc3_*gges_sort) and SDIM comes
    before info: (..., VSL, VSR, sdim, info)."""
    L = lib()
    dt = A.dtype.type
    pfx = {np.complex128: "z", np.complex64: "c", np.float64: "d", np.float32: "s"}[dt]
    n = A.shape[0]
    S, T = np.array(A, order="F", dtype=dt), np.array(B, order="F", dtype=dt)
    VL = np.zeros((n, n), dtype=dt, order="F") if jobvsl == "V" else None
    VR = np.zeros((n, n), dtype=dt, order="F") if jobvsr == "V" else None
    info = ct.c_int(0)
    ld = max(n, 1)
    if pfx in "zc":
        eig = [np.zeros(max(n, 1), dtype=dt) for _ in range(2)]
    else:
        eig = [np.zeros(max(n, 1), dtype=dt) for _ in range(3)]
    if sort is None:
        getattr(L, f"xtgevc3_{pfx}gges")(jobvsl.encode(), jobvsr.encode(), n, _ptr(S), ld, _ptr(T), ld,
                                         *[_ptr(e) for e in eig], _ptr(VL), ld, _ptr(VR), ld, ct.byref(info))
    else:
        sdim, sel = ct.c_int(-1), _selctg(pfx, sort)
        getattr(L, f"xtgevc3_{pfx}gges_sort")(jobvsl.encode(), jobvsr.encode(), b"S", sel, n, _ptr(S), ld, _ptr(T), ld,
                                              ct.byref(sdim), *[_ptr(e) for e in eig], _ptr(VL), ld, _ptr(VR), ld,
                                              ct.byref(info))
    if info.value == n + 1:  # a CUDA call failed (n + 2, n + 3: xGGES's ordering results)
        raise RuntimeError(f"xtgevc3_{pfx}gges failed: {last_error()}")
    out = (S, T, *[e[:n] for e in eig], VL, VR)
    return (*out, info.value) if sort is None else (*out, sdim.value, info.value)


def gges_dev(A, B, VSL=None, VSR=None, stream=None, sort=None):
    """Device form of z/c/d/sgges on column-major CUDA tensors: A, B become S, T in place, VSL /
    VSR (when given) the orthogonal / unitary factors.  Returns (alpha, beta, info) (complex)
    or (alphar, alphai, beta, info) (real), the eigenvalue arrays CUDA tensors.  With sort (as
    for gges; called on the host) the selected eigenvalues lead and SDIM comes before info."""
    import torch
    L = lib()
    pfx = {torch.complex128: "z", torch.complex64: "c", torch.float64: "d", torch.float32: "s"}[A.dtype]
    n = A.shape[0]
    st = ct.c_void_p(stream if stream is not None else torch.cuda.current_stream().cuda_stream)
    eig = [torch.zeros(max(n, 1), dtype=A.dtype, device=A.device) for _ in range(2 if pfx in "zc" else 3)]
    info = ct.c_int(0)

    def ld(t):
        return max(t.stride(1), 1) if t is not None else 1

    def ptr(t):
        return ct.c_void_p(t.data_ptr()) if t is not None else None

    jl, jr = b"V" if VSL is not None else b"N", b"V" if VSR is not None else b"N"
    if sort is None:
        rc = getattr(L, f"xtgevc3_{pfx}gges_dev")(st, jl, jr, n, ptr(A), ld(A), ptr(B), ld(B), *[ptr(e) for e in eig],
                                                 ptr(VSL), ld(VSL), ptr(VSR), ld(VSR), ct.byref(info))
    else:
        sdim, sel = ct.c_int(-1), _selctg(pfx, sort)
        rc = getattr(L, f"xtgevc3_{pfx}gges_sort_dev")(st, jl, jr, b"S", sel, n, ptr(A), ld(A), ptr(B), ld(B),
                                                      ct.byref(sdim), *[ptr(e) for e in eig], ptr(VSL), ld(VSL),
                                                      ptr(VSR), ld(VSR), ct.byref(info))
    if rc:
        raise RuntimeError(f"xtgevc3_{pfx}gges_dev failed: {last_error()}")
    out = [e[:n] for e in eig]
    return (*out, info.value) if sort is None else (*out, sdim.value, info.value)


def tgsen(select, A, B, Q=None, Z=None, ijob=0):
    """Host-array form of d/s/z/ctgsen: the eigenvalues flagged in select move to the leading
    rows (Q, Z None: not updated).  Returns (A, B, eigenvalue arrays..., Q, Z, m, info) as new
    arrays, the eigenvalue arrays (alphar, alphai, beta) or (alpha, beta); with ijob 1, 2 or 4
    (real pencils) PL, PR and DIF (2 values) come before info: (..., m, pl, pr, dif, info)."""
    L = lib()
    dt = A.dtype.type
    pfx = {np.complex128: "z", np.complex64: "c", np.float64: "d", np.float32: "s"}[dt]
    n = A.shape[0]
    a, b = np.array(A, order="F", dtype=dt), np.array(B, order="F", dtype=dt)
    q = np.array(Q, order="F", dtype=dt) if Q is not None else None
    z = np.array(Z, order="F", dtype=dt) if Z is not None else None
    sel = np.ascontiguousarray(select, dtype=np.int32)
    ev = [np.zeros(max(n, 1), dtype=dt) for _ in range(2 if pfx in "zc" else 3)]
    m, info = ct.c_int(0), ct.c_int(0)
    rdt = np.float32 if pfx in "sc" else np.float64
    est = np.zeros(4, dtype=rdt)  # PL, PR, DIF(1), DIF(2)
    ld = max(n, 1)
    getattr(L, f"xtgevc3_{pfx}tgsen")(ijob, int(q is not None), int(z is not None), _ptr(sel), n, _ptr(a), ld, _ptr(b),
                                      ld, *[_ptr(e) for e in ev], _ptr(q), ld, _ptr(z), ld, ct.byref(m),
                                      _ptr(est[0:1]), _ptr(est[1:2]), _ptr(est[2:4]), ct.byref(info))
    if info.value == n + 1 and n > 0:
        raise RuntimeError(f"xtgevc3_{pfx}tgsen failed: {last_error()}")
    out = (a, b, *[e[:n] for e in ev], q, z, m.value)
    if ijob == 0:
        return (*out, info.value)
    return (*out, float(est[0]), float(est[1]), est[2:4].copy(), info.value)


def tgsen_dev(select, A, B, Q=None, Z=None, stream=None, ijob=0):
    """Device form of d/s/z/ctgsen on column-major CUDA tensors (in place; select a host array).
    Returns (eigenvalue tensors..., m, info); with ijob 1, 2 or 4 (..., m, pl, pr, dif, info)."""
    import torch
    L = lib()
    pfx = {torch.complex128: "z", torch.complex64: "c", torch.float64: "d", torch.float32: "s"}[A.dtype]
    n = A.shape[0]
    st = ct.c_void_p(stream if stream is not None else torch.cuda.current_stream().cuda_stream)
    sel = np.ascontiguousarray(select, dtype=np.int32)
    ev = [torch.zeros(max(n, 1), dtype=A.dtype, device=A.device) for _ in range(2 if pfx in "zc" else 3)]
    m, info = ct.c_int(0), ct.c_int(0)

    def ld(t):
        return max(t.stride(1), 1) if t is not None else 1

    def ptr(t):
        return ct.c_void_p(t.data_ptr()) if t is not None else None

    est = np.zeros(4, dtype=np.float32 if pfx in "sc" else np.float64)
    rc = getattr(L, f"xtgevc3_{pfx}tgsen_dev")(st, ijob, int(Q is not None), int(Z is not None), _ptr(sel), n, ptr(A),
                                              ld(A), ptr(B), ld(B), *[ptr(e) for e in ev], ptr(Q), ld(Q), ptr(Z),
                                              ld(Z), ct.byref(m), _ptr(est[0:1]), _ptr(est[1:2]), _ptr(est[2:4]),
                                              ct.byref(info))
    if rc:
        raise RuntimeError(f"xtgevc3_{pfx}tgsen_dev failed: {last_error()}")
    out = (*[e[:n] for e in ev], m.value)
    if ijob == 0:
        return (*out, info.value)
    return (*out, float(est[0]), float(est[1]), est[2:4].copy(), info.value)


def tgsyl(ijob, A, B, C, D, E, F, trans="N"):
    """Host-array form of d/s/z/ctgsyl: TRANS = 'N', A R - L B = scale C, D R - L E = scale F;
    TRANS = 'T' (real types), A^T R + D^T L = scale C, R B^T + L E^T = -scale F.  Returns (R, L,
    scale, dif, info) (new arrays; dif meaningful for ijob 1 and 3 with TRANS = 'N')."""
    L = lib()
    dt = A.dtype.type
    pfx = {np.float64: "d", np.float32: "s", np.complex128: "z", np.complex64: "c"}[dt]
    m, n = C.shape
    A, B, D, E = (np.array(M, order="F", dtype=dt) for M in (A, B, D, E))
    Rm, Lm = np.array(C, order="F", dtype=dt), np.array(F, order="F", dtype=dt)
    sd = np.zeros(2, dtype=np.float32 if pfx in "sc" else np.float64)
    info = ct.c_int(0)
    lm, ln = max(m, 1), max(n, 1)
    getattr(L, f"xtgevc3_{pfx}tgsyl")(trans.encode(), ijob, m, n, _ptr(A), lm, _ptr(B), ln, _ptr(Rm), lm, _ptr(D), lm, _ptr(E), ln,
                                      _ptr(Lm), lm, _ptr(sd[0:1]), _ptr(sd[1:2]), ct.byref(info))
    if info.value == m + n + 1:
        raise RuntimeError(f"xtgevc3_{pfx}tgsyl failed: {last_error()}")
    return Rm, Lm, float(sd[0]), float(sd[1]), info.value


def ggbal(A, B, job="P"):
    """Host-array form of d/s/z/cggbal (JOB 'N' or 'P'): returns (A, B, ilo, ihi, lscale, rscale,
    info) with the balanced A, B as new arrays."""
    L = lib()
    dt = A.dtype.type
    pfx = {np.complex128: "z", np.complex64: "c", np.float64: "d", np.float32: "s"}[dt]
    n = A.shape[0]
    a, b = np.array(A, order="F", dtype=dt), np.array(B, order="F", dtype=dt)
    rdt = np.float32 if pfx in "sc" else np.float64
    ls, rs = np.zeros(max(n, 1), dtype=rdt), np.zeros(max(n, 1), dtype=rdt)
    ilo, ihi, info = ct.c_int(0), ct.c_int(0), ct.c_int(0)
    getattr(L, f"xtgevc3_{pfx}ggbal")(job.encode(), n, _ptr(a), max(n, 1), _ptr(b), max(n, 1), ct.byref(ilo),
                                      ct.byref(ihi), _ptr(ls), _ptr(rs), ct.byref(info))
    if info.value == n + 1 and n > 0:
        raise RuntimeError(f"xtgevc3_{pfx}ggbal failed: {last_error()}")
    return a, b, ilo.value, ihi.value, ls[:n], rs[:n], info.value


def ggbak(V, ilo, ihi, lscale, rscale, side="L", job="P"):
    """Host-array form of d/s/z/cggbak (JOB 'N' or 'P'): returns (V back-permuted, info)."""
    L = lib()
    dt = V.dtype.type
    pfx = {np.complex128: "z", np.complex64: "c", np.float64: "d", np.float32: "s"}[dt]
    n, m = V.shape
    v = np.array(V, order="F", dtype=dt)
    rdt = np.float32 if pfx in "sc" else np.float64
    ls, rs = (np.ascontiguousarray(x, dtype=rdt) for x in (lscale, rscale))
    info = ct.c_int(0)
    getattr(L, f"xtgevc3_{pfx}ggbak")(job.encode(), side.encode(), n, ilo, ihi, _ptr(ls), _ptr(rs), m, _ptr(v),
                                      max(n, 1), ct.byref(info))
    if info.value == n + 1 and n > 0:
        raise RuntimeError(f"xtgevc3_{pfx}ggbak failed: {last_error()}")
    return v, info.value


def tgexc(A, B, Q=None, Z=None, ifst=1, ilst=1, with_ifst=False):
    """Host-array form of z/c/d/stgexc: move the eigenvalue (real pencils: the 1x1 or 2x2
    diagonal block) at row ifst of the generalized Schur pencil (A, B) to row ilst (1-based,
    as LAPACK), updating Q and Z when given.  Returns (A, B, Q, Z, ilst, info) with new
    arrays, or (A, B, Q, Z, ifst, ilst, info) with with_ifst (real pencils: IFST moves to the
    first row of its 2x2 block, as in D/STGEXC)."""
    L = lib()
    dt = A.dtype.type
    pfx = {np.complex128: "z", np.complex64: "c", np.float64: "d", np.float32: "s"}[dt]
    n = A.shape[0]
    A, B = np.array(A, order="F", dtype=dt), np.array(B, order="F", dtype=dt)
    Qc = None if Q is None else np.array(Q, order="F", dtype=dt)
    Zc = None if Z is None else np.array(Z, order="F", dtype=dt)
    fs, il, info = ct.c_int(ifst), ct.c_int(ilst), ct.c_int(0)
    ld = max(n, 1)
    getattr(L, f"xtgevc3_{pfx}tgexc")(int(Qc is not None), int(Zc is not None), n, _ptr(A), ld, _ptr(B), ld, _ptr(Qc),
                                      ld, _ptr(Zc), ld, ct.byref(fs) if pfx in "ds" else ifst, ct.byref(il),
                                      ct.byref(info))
    if info.value == 1 and last_error():  # a rejected swap (INFO = 1) leaves no error text
        raise RuntimeError(f"xtgevc3_{pfx}tgexc failed: {last_error()}")
    if with_ifst:
        return A, B, Qc, Zc, fs.value, il.value, info.value
    return A, B, Qc, Zc, il.value, info.value


def tgexc_dev(A, B, Q=None, Z=None, ifst=1, ilst=1, stream=None, with_ifst=False):
    """Device form of z/c/d/stgexc on column-major CUDA tensors (reordered in place).  Returns
    (ilst, info), or (ifst, ilst, info) with with_ifst."""
    import torch
    L = lib()
    pfx = {torch.complex128: "z", torch.complex64: "c", torch.float64: "d", torch.float32: "s"}[A.dtype]
    n = A.shape[0]
    st = ct.c_void_p(stream if stream is not None else torch.cuda.current_stream().cuda_stream)
    fs, il, info = ct.c_int(ifst), ct.c_int(ilst), ct.c_int(0)

    def ld(t):
        return max(t.stride(1), 1) if t is not None else max(n, 1)

    def ptr(t):
        return ct.c_void_p(t.data_ptr()) if t is not None else None

    rc = getattr(L, f"xtgevc3_{pfx}tgexc_dev")(st, int(Q is not None), int(Z is not None), n, ptr(A), ld(A), ptr(B),
                                              ld(B), ptr(Q), ld(Q), ptr(Z), ld(Z),
                                              ct.byref(fs) if pfx in "ds" else ifst, ct.byref(il), ct.byref(info))
    if rc:
        raise RuntimeError(f"xtgevc3_{pfx}tgexc_dev failed: {last_error()}")
    if with_ifst:
        return fs.value, il.value, info.value
    return il.value, info.value


# ---- batched form ------------------------------------------------------------------------
class PencilDesc(ct.Structure):
    """xtgevc3_dpencil / xtgevc3_spencil (include/xtgevc3.h): device pointers of one pencil."""
    _fields_ = [("n", _I), ("lds", _I), ("ldp", _I), ("ldq", _I), ("ldz", _I), ("ldvl", _I), ("ldvr", _I),
                ("S", _P), ("P", _P), ("alphar", _P), ("alphai", _P), ("beta", _P), ("Q", _P), ("Z", _P),
                ("VL", _P), ("VR", _P)]


def batch_config(nt: int, h: int) -> int:
    """XTGEVC3_BATCH_CONFIG(nt, h): NT eigenvector columns per tile, row blocks of H rows."""
    return (int(nt) << 8) | int(h)


def _descs(pencils):
    """ctypes array of descriptors for a list of dicts of CUDA tensors (matrices column-major:
    S, P, and as needed Q, Z, VL, VR; vectors alphar, alphai, beta)."""
    import torch
    arr = (PencilDesc * len(pencils))()
    prec = None
    for i, p in enumerate(pencils):
        S = p["S"]
        prec = prec or {torch.float64: "d", torch.float32: "s"}[S.dtype]
        d = arr[i]
        d.n = S.shape[0]
        for key, ld in (("S", "lds"), ("P", "ldp"), ("Q", "ldq"), ("Z", "ldz"), ("VL", "ldvl"), ("VR", "ldvr")):
            t = p.get(key)
            ptr, l = _colmajor(t)
            setattr(d, key, ptr)
            setattr(d, ld, l if t is not None else max(d.n, 1))
        for key in ("alphar", "alphai", "beta"):
            t = p[key]
            if not t.is_contiguous():
                raise ValueError(f"{key} must be contiguous")
            setattr(d, key, ct.c_void_p(t.data_ptr()))
    return arr, prec or "d"


class Batch:
    """Plan of the batched form (xtgevc3_{d,s}tgevc3_batched_create) over CUDA tensors.

    ``pencils``: list of dicts with S, P, alphar, alphai, beta and, as the side and howmny
    need them, Q, Z (read only) and VL, VR (outputs, not overlapping Q / Z).  The plan keeps
    the tensors alive; ``run()`` launches the captured graph on torch's current stream
    (or ``stream``), ``wait()`` synchronises and raises if the kernel reported a failure.
    """

    def __init__(self, side, howmny, pencils, config=0):
        L = lib()
        self._keep = pencils
        self._arr, self.prec = _descs(pencils)
        self._plan = ct.c_void_p()
        rc = getattr(L, f"xtgevc3_{self.prec}tgevc3_batched_create")(
            side.encode(), howmny.encode(), len(pencils), ct.cast(self._arr, _P), int(config), ct.byref(self._plan))
        if rc != 0:
            raise RuntimeError(f"batched create failed ({rc}): {last_error()}")

    @staticmethod
    def _stream(stream):
        import torch
        return ct.c_void_p(torch.cuda.current_stream().cuda_stream if stream is None else stream)

    def run(self, stream=None):
        if lib().xtgevc3_batched_run(self._plan, self._stream(stream)) != 0:
            raise RuntimeError(f"batched run failed: {last_error()}")

    def wait(self, stream=None):
        rc = lib().xtgevc3_batched_wait(self._plan, self._stream(stream))
        if rc != 0:
            raise RuntimeError(f"batched wait ({rc}): {last_error()}")

    def info(self):
        c, g, u = ct.c_uint(0), ct.c_int(0), ct.c_int(0)
        lib().xtgevc3_batched_info(self._plan, ct.byref(c), ct.byref(g), ct.byref(u))
        return dict(nt=c.value >> 8, h=c.value & 255, grid=g.value, units=u.value)

    def close(self):
        if self._plan:
            lib().xtgevc3_batched_destroy(self._plan)
            self._plan = ct.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def batched_tune(side, howmny, pencils, reps=3):
    """Time every tile configuration on this batch; the fastest becomes the process default
    for the precision.  Returns (config, ms)."""
    arr, prec = _descs(pencils)
    best, ms = ct.c_uint(0), ct.c_float(0)
    rc = getattr(lib(), f"xtgevc3_{prec}tgevc3_batched_tune")(side.encode(), howmny.encode(), len(pencils),
                                                               ct.cast(arr, _P), int(reps), ct.byref(best),
                                                               ct.byref(ms))
    if rc != 0:
        raise RuntimeError(f"batched tune failed ({rc}): {last_error()}")
    return best.value, ms.value


def batched_set_default(prec: str, config: int) -> None:
    lib().xtgevc3_batched_set_default(prec.encode(), int(config))


def batched_get_default(prec: str) -> int:
    return int(lib().xtgevc3_batched_get_default(prec.encode()))


# ---- adjoint -------------------------------------------------------------------------------
def adjoint(S, P, alpha, beta, X, G, alphai=None, stream=None):
    """dL/dS, dL/dP for the right eigenvectors X (SIDE='R', HOWMNY='A') given G = dL/dX
    (xtgevc3_adjoint).  S, P, X, G: column-major CUDA tensors; alpha/alphai/beta: host
    arrays.  Returns (dS, dP) as new column-major CUDA tensors."""
    import torch
    L = lib()
    L.xtgevc3_adjoint.argtypes = [_C, _P, _I, _P, _I, _P, _I, _P, _P, _P, _P, _I, _P, _I, _P, _I, _P, _I]
    L.xtgevc3_adjoint.restype = _I
    tdt = S.dtype
    pfx = {torch.float64: "d", torch.float32: "s", torch.complex128: "z", torch.complex64: "c"}[tdt]
    n = S.shape[0]
    dS = torch.zeros(n, n, dtype=tdt, device=S.device).t()
    dP = torch.zeros(n, n, dtype=tdt, device=S.device).t()
    rdt = np.float64 if pfx in "dz" else np.float32
    cdt = np.complex128 if pfx == "z" else np.complex64
    if pfx in "ds":
        al = np.ascontiguousarray(alpha, dtype=rdt)
        ai = np.ascontiguousarray(alphai, dtype=rdt)
        be = np.ascontiguousarray(beta, dtype=rdt)
    else:
        al = np.ascontiguousarray(alpha, dtype=cdt)
        ai = None
        be = np.ascontiguousarray(beta, dtype=cdt)
    if stream is None:
        stream = torch.cuda.current_stream().cuda_stream
    args = [pfx.encode(), ct.c_void_p(stream), n]
    for t in (S, P):
        p, ld = _colmajor(t)
        args += [p, ld]
    args += [_ptr(al), _ptr(ai), _ptr(be)]
    for t in (X, G, dS, dP):
        p, ld = _colmajor(t)
        args += [p, ld]
    rc = L.xtgevc3_adjoint(*args)
    if rc != 0:
        raise RuntimeError(f"xtgevc3_adjoint failed ({rc}): {last_error()}")
    return dS, dP
