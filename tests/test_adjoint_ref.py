"""Pinning of the adjoint's dense reference (tests/adjoint_ref.py) on the CPU.

No adjoint exists upstream, so the reference gradient is pinned in two steps: its
forward must reproduce the oracle's right eigenvectors (the upstream algorithm), and its
autograd gradient must match central finite differences (step 1e-6) of the oracle's
forward, with the eigenvalues held fixed, on sampled entries that include the column
attaining each pencil norm, the 2x2 seed entries of complex pairs and the subdiagonal of
S (the upstream solves are Hessenberg solves: L depends on every subdiagonal entry of a
real S, zero or not; P is triangular by contract and gets no gradient below it)."""
import numpy as np
import pytest

import oracle
from xtgevc3_b200 import pencils

import adjoint_ref


def fd_entries(S, n, rng, extra):
    ent = {(int(i), int(j)) for i, j in zip(rng.integers(0, n, 60), rng.integers(0, n, 60)) if i <= j}
    for j in (int(np.argmax(np.abs(np.triu(S, -1)).sum(0))),):
        ent |= {(i, j) for i in range(min(j + 2, n))}
    ent |= {(j + 1, j) for j in range(0, n - 1, 3)}  # S's subdiagonal, zeros included
    return sorted(ent | set(extra))


@pytest.mark.parametrize("dt,n,seed", [(np.float64, 28, 3), (np.complex128, 20, 4)], ids=["d", "z"])
def test_reference_gradient_matches_finite_differences(dt, n, seed):
    real = dt == np.float64
    if real:
        S, P, ar, ai, be, Q, Z = pencils.gen_gges(n, seed, dtype=dt)
        al = ar
    else:
        S, P, al, be, Q, Z = pencils.gen_gges(n, seed, dtype=dt)
        ai = None
    rng = np.random.default_rng(seed)
    G = rng.standard_normal((n, n)) if real else rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
    gS, gP, Xr = adjoint_ref.gradient(S, P, al, be, G, alphai=ai)
    X0 = oracle.tgevc3("R", "A", S, P, al, be, alphai=ai)[1]
    assert np.abs(Xr - X0).max() <= 1e-13 * np.abs(X0).max()

    def loss(S_, P_):
        X = oracle.tgevc3("R", "A", S_, P_, al, be, alphai=ai)[1]
        return float(np.sum(G.real * X.real + (G.imag * X.imag if not real else 0)))

    seeds = []
    if real:
        k = 0
        while k < n - 1:
            if ai[k] != 0:
                seeds += [(k, k), (k, k + 1)]
                k += 2
            else:
                k += 1
        assert seeds, "pencil without complex pairs"
    h = 1e-6
    scale = max(np.abs(gS).max(), np.abs(gP).max())
    worst = 0.0
    for (i, j) in fd_entries(S, n, rng, seeds):
        for which in ("S", "P"):
            if which == "P" and i > j:
                assert gP[i, j] == 0  # P is triangular by contract
                continue
            for part in ((1.0,) if real else (1.0, 1j)):
                E = np.zeros((n, n), dtype=dt)
                E[i, j] = h * part
                if which == "S":
                    fd = (loss(S + E, P) - loss(S - E, P)) / (2 * h)
                    g = gS[i, j]
                else:
                    fd = (loss(S, P + E) - loss(S, P - E)) / (2 * h)
                    g = gP[i, j]
                comp = g.real if part == 1.0 else np.imag(g)
                worst = max(worst, abs(fd - comp) / scale)
    assert worst < 1e-7, worst
