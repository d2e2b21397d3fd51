"""The C++ drop-in interface called from C++: tests/dropin_caller.cpp includes
include/tgevc3.h and calls dtgevc3 / ztgevc3 with the upstream tests' pattern (LWORK = -1
query, then the call), linked with g++ against libxtgevc3.so -- the mangled C++ symbols,
not the extern "C" twins.  On CPU the program must compile and link; on a GPU its INFO, M,
LWORK answer and eigenvectors must match the upstream library / the oracle."""
import os
import subprocess

import numpy as np
import pytest

import oracle
import xtgevc3_b200 as X
from conftest import ROOT
from xtgevc3_b200 import pencils


def _build(tmp_path):
    exe = str(tmp_path / "dropin_caller")
    lib = X.lib()._name
    cmd = ["g++", "-O1", "-std=c++17", "-I", os.path.join(ROOT, "include"), os.path.join(ROOT, "tests",
           "dropin_caller.cpp"), "-o", exe, lib, f"-Wl,-rpath,{os.path.dirname(lib)}"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def test_dropin_caller_links_against_mangled_symbols(tmp_path):
    exe = _build(tmp_path)
    nm = subprocess.run(["nm", "-u", "-C", exe], capture_output=True, text=True).stdout
    assert "dtgevc3(char, char, int const*, int, double const*" in nm
    assert "ztgevc3(char, char, int const*, int, std::complex<double> const*" in nm
    assert "xtgevc3_" not in nm  # the extern "C" twins are not what it calls


@pytest.mark.gpu
@pytest.mark.parametrize("prec,side,howmny,n", [("d", "B", "B", 150), ("d", "R", "A", 97), ("z", "B", "B", 60)])
def test_dropin_caller_matches_oracle(cuda_ok, tmp_path, prec, side, howmny, n):
    exe = _build(tmp_path)
    if prec == "d":
        S, P, ar, ai, be, Q, Z = pencils.gen_gges(n, 700 + n)
        parts = [S, P, ar, ai, be, Q, Z]
        dt = np.float64
        ref = oracle.tgevc3(side, howmny, S, P, ar, be, alphai=ai, VL=Q.copy(order="F"), VR=Z.copy(order="F"),
                            impl="ref" if oracle.ref_available() else "oracle")
    else:
        A, B, Q, Z = oracle.complex_schur_pencil(n, 700 + n)
        al, be = np.diag(A).copy(), np.diag(B).copy()
        S, P = A, B
        parts = [S, P, al, be, Q, Z]
        dt = np.complex128
        ref = oracle.tgevc3(side, howmny, S, P, al, be, VL=Q.copy(order="F"), VR=Z.copy(order="F"),
                            impl="ref" if oracle.ref_available() else "oracle")
    fin, fout = str(tmp_path / "in.bin"), str(tmp_path / "out.bin")
    with open(fin, "wb") as f:
        for a in parts:
            f.write(np.asarray(a, dtype=dt).tobytes(order="F"))
    r = subprocess.run([exe, prec, side, howmny, str(n), fin, fout], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    raw = open(fout, "rb").read()
    lwork, m, info = np.frombuffer(raw[:12], dtype=np.int32)
    b = 33  # the upstream workspace formula with its panel width 32 (b + 1 = 33)
    assert lwork == 2 * n * b + 4 * b * b + 2 * b
    assert (m, info) == (ref[2], ref[3]) == (n, 0)
    V = np.frombuffer(raw[12:], dtype=dt)
    VL = V[:n * n].reshape(n, n, order="F")
    VR = V[n * n:].reshape(n, n, order="F")
    for s, mine, theirs in (("L", VL, ref[0]), ("R", VR, ref[1])):
        if side not in (s, "B"):
            continue
        if prec == "d":
            a, c = oracle.to_complex_real_storage(mine, ai), oracle.to_complex_real_storage(theirs[:, :n], ai)
        else:
            a, c = mine, theirs[:, :n]
        err, _ = oracle.max_rel_diff(a, c)
        assert err < 1e-11, (s, err)
