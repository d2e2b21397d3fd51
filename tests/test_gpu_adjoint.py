"""xtgevc3_adjoint on the GPU against central finite differences of the oracle (n = 64,
step 1e-6) and against the dense autograd reference of tests/adjoint_ref.py (n = 256 for
FP64; complex64 pencils of n = 128).

Tolerances, relative to the largest gradient entry: 1e-6 against finite differences
(their truncation and rounding error), 1e-9 against the reference in FP64 / complex128,
2e-3 in FP32 / complex64 (the FP32 eigenvectors themselves carry ~1e-5..1e-4 relative
error on these pencils)."""
import numpy as np
import pytest

import oracle
import xtgevc3_b200 as X
from xtgevc3_b200 import pencils

import adjoint_ref

pytestmark = pytest.mark.gpu


def dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(np.asarray(a).T)).cuda().t()


def host(t):
    return t.t().cpu().numpy().T


def pencil(dt, n, seed):
    if np.issubdtype(dt, np.complexfloating):
        S, P, al, be, Q, Z = pencils.gen_gges(n, seed, dtype=dt)
        return S, P, al, None, be
    S, P, ar, ai, be, Q, Z = pencils.gen_gges(n, seed, dtype=dt)
    return S, P, ar, ai, be


def gpu_grad(S, P, al, ai, be, G):
    """Forward on the GPU (SIDE='R', HOWMNY='A'), then the adjoint; returns (dS, dP, X)."""
    n = S.shape[0]
    dS_, dP_ = dev(S), dev(P)
    VR = dev(np.zeros((n, n), dtype=S.dtype))
    m, info = X.tgevc3_dev("R", "A", dS_, dP_, al, be, alphai=ai, VR=VR)
    assert (m, info) == (n, 0)
    gS, gP = X.adjoint(dS_, dP_, al, be, VR, dev(G), alphai=ai)
    return host(gS), host(gP), host(VR)


def rand_g(dt, n, seed):
    rng = np.random.default_rng(seed)
    g = rng.standard_normal((n, n))
    if np.issubdtype(dt, np.complexfloating):
        g = g + 1j * rng.standard_normal((n, n))
    return g.astype(dt)


def test_adjoint_d_vs_finite_differences_n64(cuda_ok):
    n = 64
    S, P, ar, ai, be = pencil(np.float64, n, 61)
    G = rand_g(np.float64, n, 62)
    gS, gP, _ = gpu_grad(S, P, ar, ai, be, G)

    def loss(S_, P_):
        return float(np.sum(G * oracle.tgevc3("R", "A", S_, P_, ar, be, alphai=ai)[1]))

    rng = np.random.default_rng(63)
    ent = {(int(i), int(j)) for i, j in zip(rng.integers(0, n, 120), rng.integers(0, n, 120)) if i <= j}
    jS = int(np.argmax(np.abs(np.triu(S, -1)).sum(0)))
    jP = int(np.argmax(np.abs(np.triu(P, -1)).sum(0)))
    ent |= {(i, jS) for i in range(0, min(jS + 2, n), 3)} | {(i, jP) for i in range(0, min(jP + 2, n), 3)}
    ent |= {(j + 1, j) for j in range(0, n - 1, 2)}  # S's subdiagonal, zeros included
    k = 0
    while k < n - 1:
        if ai[k] != 0:
            ent |= {(k, k), (k, k + 1), (k + 1, k)}
            k += 2
        else:
            k += 1
    h = 1e-6
    scale = max(np.abs(gS).max(), np.abs(gP).max())
    worst = 0.0
    for i, j in sorted(ent):
        E = np.zeros((n, n))
        E[i, j] = h
        fs = (loss(S + E, P) - loss(S - E, P)) / (2 * h)
        worst = max(worst, abs(fs - gS[i, j]) / scale)
        if i <= j:  # P is triangular by contract
            fp = (loss(S, P + E) - loss(S, P - E)) / (2 * h)
            worst = max(worst, abs(fp - gP[i, j]) / scale)
    assert worst < 1e-6, worst
    # entries the forward never reads carry no gradient
    assert not gS[np.tril(np.ones((n, n), bool), -2)].any()
    assert not gP[np.tril(np.ones((n, n), bool), -1)].any()


@pytest.mark.parametrize("dt,n,seed,tol", [(np.float64, 256, 71, 1e-9), (np.complex128, 160, 72, 1e-9),
                                           (np.float32, 96, 73, 2e-3)], ids=["d256", "z160", "s96"])
def test_adjoint_vs_dense_reference(cuda_ok, dt, n, seed, tol):
    S, P, al, ai, be = pencil(dt, n, seed)
    G = rand_g(dt, n, seed + 1)
    gS, gP, Xg = gpu_grad(S, P, al, ai, be, G)
    wide = np.complex128 if np.issubdtype(dt, np.complexfloating) else np.float64
    rS, rP, _ = adjoint_ref.gradient(S.astype(wide), P.astype(wide), np.asarray(al).astype(wide),
                                     np.asarray(be).astype(wide), G.astype(wide),
                                     alphai=None if ai is None else ai.astype(np.float64))
    scale = max(np.abs(rS).max(), np.abs(rP).max())
    err = max(np.abs(gS - rS).max(), np.abs(gP - rP).max()) / scale
    assert err < tol, err


def test_adjoint_c_batch_of_pencils(cuda_ok):
    """ctgevc3 adjoint on several complex64 pencils of n = 128 against the complex128
    reference."""
    for seed in (81, 82, 83):
        n = 128
        S, P, al, ai, be = pencil(np.complex64, n, seed)
        G = rand_g(np.complex64, n, seed + 10)
        gS, gP, _ = gpu_grad(S, P, al, ai, be, G)
        rS, rP, _ = adjoint_ref.gradient(S.astype(np.complex128), P.astype(np.complex128),
                                         al.astype(np.complex128), be.astype(np.complex128),
                                         G.astype(np.complex128))
        scale = max(np.abs(rS).max(), np.abs(rP).max())
        err = max(np.abs(gS - rS).max(), np.abs(gP - rP).max()) / scale
        assert err < 2e-3, (seed, err)
