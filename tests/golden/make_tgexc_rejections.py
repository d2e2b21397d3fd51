"""Generates tests/golden/tgexc/z_rejections.npz: small complex upper-triangular pencils on
which LAPACK ZTGEXC rejects a swap (INFO = 1) after zero or more accepted swaps.

A rejected swap needs a badly scaled pencil: entries are drawn with magnitudes 10^U(lo, hi),
lo ~ -U(0, 150), hi ~ U(0, 150), random phases, and in some pencils an infinite eigenvalue
(B(3,3) = 0) or an eigenvalue equal to the first one.  Kept: the first pencils (seeded
search) whose forward move 1 -> 3 or backward move 3 -> 1 LAPACK rejects with every output
finite, one each of: a forward move with a swap applied before the rejection, a backward
move with a swap applied before it, and a move rejected at its first swap.  The fixture
holds inputs only; the tests run LAPACK on them again.

    python tests/golden/make_tgexc_rejections.py
"""
import os
import sys
import warnings

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", ".."))
import oracle  # noqa: E402


def main():
    warnings.simplefilter("ignore")
    rng = np.random.default_rng(0)

    def draw(shape, lo, hi):
        return 10 ** rng.uniform(lo, hi, shape) * np.exp(2j * np.pi * rng.random(shape))

    want = {("fwd", True): None, ("bwd", True): None, ("any", False): None}
    for _ in range(200000):
        lo, hi = -rng.uniform(0, 150), rng.uniform(0, 150)
        A, B = np.triu(draw((3, 3), lo, hi)), np.triu(draw((3, 3), lo, hi))
        r = rng.random()
        if r < 0.3:
            B[2, 2] = 0
        elif r < 0.6:
            A[2, 2] = A[0, 0] * B[2, 2] / B[0, 0]
        if not (np.isfinite(A).all() and np.isfinite(B).all()):
            continue
        for f, l, d in ((1, 3, "fwd"), (3, 1, "bwd")):
            I = np.eye(3, dtype=np.complex128, order="F")
            a, b, q, z, il, info = oracle.lapack_tgexc_ilst(A, B, I, I, f, l)
            if info == 0 or not all(np.isfinite(M).all() for M in (a, b, q, z)):
                continue
            partial = not np.array_equal(a, A)
            key = (d, True) if partial else ("any", False)
            if want.get(key, 0) is None:
                want[key] = (A.copy(), B.copy(), f, l)
        if all(v is not None for v in want.values()):
            break
    arrays = {}
    for i, (k, (A, B, f, l)) in enumerate(sorted(want.items())):
        arrays[f"A{i}"], arrays[f"B{i}"] = A, B
        arrays[f"move{i}"] = np.array([f, l])
    np.savez(os.path.join(HERE, "tgexc", "z_rejections.npz"), **arrays)
    print({k: (v[2], v[3]) for k, v in want.items()})


if __name__ == "__main__":
    main()
