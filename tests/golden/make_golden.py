"""Generate the golden fixtures of tests/golden/*.npz from the upstream library itself.

Run in a checkout where the upstream sources are available and built:
    make -C oracle ref && python tests/golden/make_golden.py

Every fixture is one call of the upstream ``{d,s,z,c}tgevc3`` (oracle/_ref, the upstream
src/*.cpp compiled as they are) on seeded or static inputs; its outputs are stored as
produced, so the C restatement under oracle/ and the CUDA path can be pinned to them
without the upstream tree.  Inputs:
  * the static 4x4 pencils of the upstream self-tests (tests/test_dtgevc3.cpp:322-326,
    355-359, 388-395 and tests/test_ztgevc3.cpp:152-184) and their 1e+-150 scalings;
  * random quasi-triangular / triangular pencils with the structure of the upstream
    generators, the overflow/underflow scalings of tests/test_lapack_d.cpp:328-344;
  * xGGES pencils of Gaussian A, B (with Q, Z for HOWMNY='B');
  * selections (HOWMNY='S') and one-sided calls.
"""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
import oracle  # noqa: E402
from xtgevc3_b200 import pencils  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))

# upstream static 4x4 pencils, column-major (tests/test_dtgevc3.cpp:322-326, 355-359)
S4 = np.array([1, 0, 0, 0, 2, 2, -5, 0, 3, 5, 2, 0, 4, -1, 2, 3], dtype=np.float64).reshape(4, 4, order="F")
P4 = np.array([2, 0, 0, 0, 1, 1, 0, 0, -1, 0, 1, 0, 3, 2, -1, 2], dtype=np.float64).reshape(4, 4, order="F")
P4_inf = P4.copy(order="F")
P4_inf[3, 3] = 0.0
AR4 = np.array([1.0, 2.0, 2.0, 3.0])
AI4 = np.array([0.0, 5.0, -5.0, 0.0])
B4 = np.array([2.0, 1.0, 1.0, 2.0])
B4_inf = np.array([2.0, 1.0, 1.0, 0.0])


def complex_static():
    """tests/test_ztgevc3.cpp:152-184 (upper triangular complex 4x4)."""
    S = np.zeros((4, 4), dtype=np.complex128, order="F")
    P = np.zeros((4, 4), dtype=np.complex128, order="F")
    ent = {(0, 0): (1 + 1j, 2), (0, 1): (2, 1 + 1j), (1, 1): (2 - 1j, 1 - 1j), (0, 2): (-5 + 1j, 0),
           (1, 2): (2j, -1), (2, 2): (3, 1 + 1j), (0, 3): (5, 0), (1, 3): (2 + 1j, 2j), (2, 3): (4 - 1j, 3),
           (3, 3): (3 + 2j, 2 - 1j)}
    for (i, j), (s, p) in ent.items():
        S[i, j] = s
        P[i, j] = p
    return S, P, np.diag(S).copy(), np.diag(P).copy()


def save(name, side, howmny, S, P, alpha, beta, alphai=None, VL=None, VR=None, select=None):
    n = S.shape[0]
    dt = S.dtype
    VL_in = np.asfortranarray(np.eye(n, dtype=dt) if VL is None else VL)
    VR_in = np.asfortranarray(np.eye(n, dtype=dt) if VR is None else VR)
    VLo, VRo, m, info = oracle.tgevc3(side, howmny, S, P, alpha, beta, alphai=alphai, VL=VL_in.copy(order="F"),
                                      VR=VR_in.copy(order="F"), select=select, impl="ref")
    d = dict(side=side, howmny=howmny, S=S, P=P, alpha=alpha, beta=beta, VL_in=VL_in, VR_in=VR_in,
             VL_out=VLo, VR_out=VRo, m=m, info=info)
    if alphai is not None:
        d["alphai"] = alphai
    if select is not None:
        d["select"] = np.asarray(select, dtype=np.int32)
    np.savez_compressed(os.path.join(OUT, f"{name}.npz"), **d)
    print(f"{name:28s} n={n:4d} {dt} side={side} howmny={howmny} m={m} info={info}")


def main():
    if not oracle.ref_available():
        raise SystemExit("oracle/_ref/libref_tgevc3.so missing: run `make -C oracle ref` first")
    oracle.set_ref_threads(1)
    # static real 4x4 (regular, infinite eigenvalue, scaled)
    save("d_static4", "B", "B", S4, P4, AR4, B4, alphai=AI4)
    save("d_static4_inf", "B", "B", S4, P4_inf, AR4, B4_inf, alphai=AI4)
    for tag, s in (("1e150", 1e150), ("1e-150", 1e-150)):
        save(f"d_static4_scaled_{tag}", "B", "B", S4 * s, P4 * s, AR4 * s, B4 * s, alphai=AI4 * s)
    save("s_static4", "B", "B", S4.astype(np.float32), P4.astype(np.float32), AR4.astype(np.float32),
         B4.astype(np.float32), alphai=AI4.astype(np.float32))
    for tag, s in (("1e30", 1e30), ("1e-30", 1e-30)):
        f = np.float32
        save(f"s_static4_scaled_{tag}", "B", "B", (S4 * s).astype(f), (P4 * s).astype(f), (AR4 * s).astype(f),
             (B4 * s).astype(f), alphai=(AI4 * s).astype(f))
    Sc, Pc, ac, bc = complex_static()
    save("z_static4", "B", "B", Sc, Pc, ac, bc)
    save("c_static4", "B", "B", Sc.astype(np.complex64), Pc.astype(np.complex64), ac.astype(np.complex64),
         bc.astype(np.complex64))

    # random quasi-triangular (upstream generator structure)
    for n, seed in ((10, 1), (40, 2), (97, 3)):
        S, P, ar, ai, be = pencils.gen_quasi_triangular(n, seed)
        save(f"d_quasi_n{n}", "B", "B", S, P, ar, be, alphai=ai)
    S, P, ar, ai, be = pencils.gen_quasi_triangular(70, 4)
    save("d_quasi_n70_selR", "R", "S", S, P, ar, be, alphai=ai, select=(np.arange(70) % 3 == 0))
    save("d_quasi_n70_selL", "L", "S", S, P, ar, be, alphai=ai, select=(np.arange(70) % 5 == 1))
    save("d_quasi_n70_A", "B", "A", S, P, ar, be, alphai=ai)
    # overflow / underflow scalings (tests/test_lapack_d.cpp:328-344), n = 30
    eps, safemin = np.finfo(np.float64).eps, np.finfo(np.float64).tiny
    smlnum = safemin / eps
    bignum = 1.0 / smlnum
    S, P, ar, ai, be = pencils.gen_quasi_triangular(30, 5)
    tri1 = np.triu(np.ones((30, 30)), -1)
    tri0 = np.triu(np.ones((30, 30)))
    for tag, ss, sp in (("S_big", bignum, 1), ("S_small", smlnum, 1), ("P_big", 1, bignum), ("P_small", 1, smlnum),
                        ("SP_big", bignum, bignum), ("SP_small", smlnum, smlnum)):
        S2 = np.asfortranarray(S * np.where(tri1 > 0, ss, 1.0))
        P2 = np.asfortranarray(P * np.where(tri0 > 0, sp, 1.0))
        save(f"d_edge_{tag}", "B", "B", S2, P2, ar * ss, be * sp, alphai=ai * ss)
    # xGGES pencils with Q, Z
    S, P, ar, ai, be, Q, Z = pencils.gen_gges(64, 7)
    save("d_gges_n64_BB", "B", "B", S, P, ar, be, alphai=ai, VL=Q, VR=Z)
    sel = np.zeros(64, dtype=np.int32)
    sel[[0, 5, 6, 17, 30, 31, 50, 63]] = 1
    save("d_gges_n64_sel", "B", "S", S, P, ar, be, alphai=ai, select=sel)
    S, P, ar, ai, be, Q, Z = pencils.gen_gges(48, 8, dtype=np.float32)
    save("s_gges_n48_BB", "B", "B", S, P, ar, be, alphai=ai, VL=Q, VR=Z)
    # complex
    for n, seed in ((10, 1), (45, 2)):
        S, P, a, b = pencils.gen_upper_triangular_complex(n, seed)
        save(f"z_tri_n{n}", "B", "B", S, P, a, b)
    S, P, a, b, Q, Z = pencils.gen_gges(40, 9, dtype=np.complex128)
    save("z_gges_n40_BB", "B", "B", S, P, a, b, VL=Q, VR=Z)
    save("z_gges_n40_sel", "R", "S", S, P, a, b, select=(np.arange(40) % 4 == 0))
    S, P, a, b, Q, Z = pencils.gen_gges(36, 10, dtype=np.complex64)
    save("c_gges_n36_BB", "B", "B", S, P, a, b, VL=Q, VR=Z)


if __name__ == "__main__":
    main()
