"""Seeded synthetic pencils (S, P) in generalized Schur form.

These are inputs, not checkers: the tests and bench.py both use them.

* ``gen_gges``       -- the generalized Schur form of iid N(0,1) A, B computed by LAPACK
                        xGGES (no eigenvalue ordering), as the workloads of this path are
                        specified; with ``graded`` B is first scaled by diag(10**U(-8, 8)).
* ``gen_schur_like`` -- a stand-in for ``gen_gges`` at sizes where xGGES is too slow to run
                        (about 1.5 h at n = 8192 on 8 host cores).  It draws a pencil that is
                        already in real generalized Schur form with the statistics measured on
                        xGGES output of Gaussian pencils: strictly-upper entries iid N(0,1),
                        diagonal magnitudes ~0.67*sqrt(n), eigenvalues lambda = g1/g2 with
                        g1, g2 Gaussian (about sqrt(2n/pi) real, the rest conjugate pairs),
                        2x2 blocks standardised as xGGES returns them (P diagonal on the block).
* ``gen_quasi_triangular`` / ``gen_upper_triangular_complex`` -- random (quasi-)triangular
                        pencils with the structure of the upstream self-tests
                        (tests/test_dtgevc3.cpp:266-316, tests/test_ztgevc3.cpp:126-144).
* ``gen_bench_triangular`` -- the upstream benchmark's pencils
                        (benchmarks/bench_dtgevc3.cpp:26-48, bench_ztgevc3.cpp:28-50):
                        upper-triangular S and P with U(-1,1) entries (complex: U(-1,1) real and
                        imaginary parts), P's diagonal real, p + sign(p) with p ~ U(-1,1).
"""
from __future__ import annotations

import numpy as np

_PFX = {np.float64: "d", np.float32: "s", np.complex128: "z", np.complex64: "c"}

def gen_quasi_triangular(n, seed=0, pair_frac=0.4, dtype=np.float64):
    """Random real quasi-triangular pencil with the structure of the upstream test
    generator (tests/test_dtgevc3.cpp:266-316): U(-1,1) upper triangles, |P_kk| pushed
    away from 0 by one, and about ``pair_frac`` of the diagonal made of 2x2 blocks with
    P = I on the block and S = [[a, b], [-b, a]] (eigenvalues a +- i|b|)."""
    rng = np.random.default_rng(seed)
    S = np.triu(rng.uniform(-1, 1, (n, n)))
    P = np.triu(rng.uniform(-1, 1, (n, n)))
    d = np.diag(P).copy()
    P[np.diag_indices(n)] = d + np.where(d >= 0, 1.0, -1.0)
    ar = np.zeros(n)
    ai = np.zeros(n)
    be = np.zeros(n)
    k = 0
    while k < n:
        if k < n - 1 and rng.integers(0, 100) < int(round(pair_frac * 100)):
            P[k, k] = P[k + 1, k + 1] = 1.0
            P[k, k + 1] = P[k + 1, k] = 0.0
            a = S[k, k]
            S[k + 1, k + 1] = a
            b = S[k, k + 1]
            if b == 0.0:
                b = 1.0
            S[k + 1, k] = -b
            ar[k] = ar[k + 1] = a
            ai[k], ai[k + 1] = abs(b), -abs(b)
            be[k] = be[k + 1] = 1.0
            k += 2
        else:
            ar[k], ai[k], be[k] = S[k, k], 0.0, P[k, k]
            k += 1
    S, P = np.asfortranarray(S.astype(dtype)), np.asfortranarray(P.astype(dtype))
    return S, P, ar.astype(dtype), ai.astype(dtype), be.astype(dtype)


def gen_upper_triangular_complex(n, seed=0, dtype=np.complex128):
    """Random complex upper-triangular pencil (the structure of the upstream complex test
    generator): U(-1,1) real and imaginary parts, |P_kk| pushed away from 0."""
    rng = np.random.default_rng(seed)
    S = np.triu(rng.uniform(-1, 1, (n, n)) + 1j * rng.uniform(-1, 1, (n, n)))
    P = np.triu(rng.uniform(-1, 1, (n, n)) + 1j * rng.uniform(-1, 1, (n, n)))
    d = np.diag(P).copy()
    P[np.diag_indices(n)] = d + d / np.abs(d)
    S, P = np.asfortranarray(S.astype(dtype)), np.asfortranarray(P.astype(dtype))
    return S, P, np.diag(S).copy(), np.diag(P).copy()


def gen_bench_triangular(n, seed=0, dtype=np.float64):
    """Upper-triangular pencil with the distributions of the upstream benchmark's generators
    (seeded numpy draws stand in for their std::mt19937 stream): S and P entries U(-1,1)
    (complex: both parts), P's diagonal real p + sign(p), p ~ U(-1,1), so |P_kk| in [1, 2).
    Returns (S, P, alpha, beta) with alpha = diag(S), beta = diag(P); a real pencil has no 2x2
    blocks (alphai = 0)."""
    rng = np.random.default_rng(seed)
    cplx = np.issubdtype(dtype, np.complexfloating)

    def draw():
        m = rng.uniform(-1, 1, (n, n))
        return np.triu(m + 1j * rng.uniform(-1, 1, (n, n)) if cplx else m)

    S, P = draw(), draw()
    p = rng.uniform(-1, 1, n)
    P[np.diag_indices(n)] = p + np.where(p >= 0, 1.0, -1.0)
    S, P = np.asfortranarray(S.astype(dtype)), np.asfortranarray(P.astype(dtype))
    return S, P, np.diag(S).copy(), np.diag(P).copy()


def gen_gges(n, seed=0, dtype=np.float64, graded=False):
    """Generalized Schur pencil of iid N(0,1) A, B via LAPACK xGGES (no ordering).

    Returns (S, P, alpha..., Q, Z): real -> (S, P, alphar, alphai, beta, Q, Z);
    complex -> (S, P, alpha, beta, Q, Z).  ``graded`` multiplies B from the left by
    diag(10**U(-8, 8)) first, so that the eigenvalues span many orders of magnitude.
    """
    import scipy.linalg.lapack as L
    rng = np.random.default_rng(seed)
    cplx = np.issubdtype(dtype, np.complexfloating)
    if cplx:
        A = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
        B = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
    else:
        A = rng.standard_normal((n, n))
        B = rng.standard_normal((n, n))
    if graded:
        B = (10.0 ** rng.uniform(-8, 8, n))[:, None] * B
    A = np.asfortranarray(A.astype(dtype))
    B = np.asfortranarray(B.astype(dtype))
    pfx = _PFX[np.dtype(dtype).type]
    f = getattr(L, f"{pfx}gges")
    out = f(lambda *a: 0, A, B, sort_t=0)
    if cplx:
        S, T, sdim, alpha, beta, Q, Z, work, info = out
        assert info == 0, info
        return (np.asfortranarray(S), np.asfortranarray(T), alpha, beta,
                np.asfortranarray(Q), np.asfortranarray(Z))
    S, T, sdim, ar, ai, be, Q, Z, work, info = out
    assert info == 0, info
    return (np.asfortranarray(S), np.asfortranarray(T), ar, ai, be,
            np.asfortranarray(Q), np.asfortranarray(Z))




def gen_schur_like(n, seed=0, dtype=np.float64, with_qz=False):
    """Real quasi-triangular pencil in generalized Schur form (see module docstring).

    Returns (S, P, alphar, alphai, beta) as Fortran-ordered arrays; with ``with_qz`` also
    random orthogonal Q, Z (QR of Gaussian matrices; slow on the host above n ~ 2048).
    """
    rng = np.random.default_rng(seed)
    S = np.triu(rng.standard_normal((n, n)), 1)
    P = np.triu(rng.standard_normal((n, n)), 1)
    n_real = int(round(np.sqrt(2.0 * n / np.pi)))
    if (n - n_real) % 2:
        n_real += 1
    n_real = min(n_real, n)
    n_pairs = (n - n_real) // 2
    # block layout: shuffle real 1x1 blocks among the 2x2 blocks
    kinds = np.array([1] * n_real + [2] * n_pairs)
    rng.shuffle(kinds)
    ar = np.zeros(n)
    ai = np.zeros(n)
    be = np.zeros(n)
    scale = 0.67 * np.sqrt(n)
    k = 0
    for kind in kinds:
        if kind == 1:
            p = scale * rng.uniform(0.2, 1.5) * rng.choice([-1.0, 1.0])
            lam = rng.standard_normal() / rng.standard_normal()
            P[k, k] = p
            S[k, k] = lam * p
            ar[k], ai[k], be[k] = S[k, k], 0.0, p
            k += 1
        else:
            g = (rng.standard_normal(2) @ [1, 1j]) / (rng.standard_normal(2) @ [1, 1j])
            x, y = g.real, abs(g.imag) + 1e-3
            p1, p2 = scale * rng.uniform(0.2, 1.5, 2)
            c = y * np.exp(0.5 * rng.standard_normal()) * rng.choice([-1.0, 1.0])
            M = np.array([[x, c], [-y * y / c, x]])
            Sb = np.diag([p1, p2]) @ M
            S[k:k + 2, k:k + 2] = Sb
            P[k, k], P[k + 1, k + 1], P[k, k + 1] = p1, p2, 0.0
            b = np.sqrt(p1 * p2)
            ar[k] = ar[k + 1] = x * b
            ai[k], ai[k + 1] = y * b, -y * b
            be[k] = be[k + 1] = b
            k += 2
    S = np.asfortranarray(S.astype(dtype))
    P = np.asfortranarray(P.astype(dtype))
    out = (S, P, ar.astype(dtype), ai.astype(dtype), be.astype(dtype))
    if with_qz:
        Q, _ = np.linalg.qr(rng.standard_normal((n, n)))
        Z, _ = np.linalg.qr(rng.standard_normal((n, n)))
        out = out + (np.asfortranarray(Q.astype(dtype)), np.asfortranarray(Z.astype(dtype)))
    return out



def schur_blocks(n, rng):
    """Diagonal blocks of a gen_schur_like pencil of order n (same statistics), drawn with
    vectorised calls: returns (k1, s1, p1, k2, s2, p2, alphar, alphai, beta) where k1 are
    the rows of the 1x1 blocks with S[k,k] = s1, P[k,k] = p1, and k2 the first rows of the
    2x2 blocks with S[k:k+2, k:k+2] = s2[:, 2x2] (row-major 4-vectors) and P = diag(p2)
    (P[k, k+1] = 0)."""
    n_real = int(round(np.sqrt(2.0 * n / np.pi)))
    if (n - n_real) % 2:
        n_real += 1
    n_real = min(n_real, n)
    n_pairs = (n - n_real) // 2
    kinds = np.array([1] * n_real + [2] * n_pairs, dtype=np.int64)
    rng.shuffle(kinds)
    starts = np.concatenate([[0], np.cumsum(kinds)[:-1]]).astype(np.int64) if n else np.zeros(0, np.int64)
    scale = 0.67 * np.sqrt(n)
    ar, ai, be = np.zeros(n), np.zeros(n), np.zeros(n)
    k1 = starts[kinds == 1]
    p1 = scale * rng.uniform(0.2, 1.5, k1.size) * rng.choice([-1.0, 1.0], k1.size)
    lam = rng.standard_normal(k1.size) / rng.standard_normal(k1.size)
    s1 = lam * p1
    ar[k1], be[k1] = s1, p1
    k2 = starts[kinds == 2]
    m = k2.size
    g = (rng.standard_normal(m) + 1j * rng.standard_normal(m)) / (rng.standard_normal(m) +
                                                                  1j * rng.standard_normal(m))
    x, y = g.real, np.abs(g.imag) + 1e-3
    q1, q2 = scale * rng.uniform(0.2, 1.5, m), scale * rng.uniform(0.2, 1.5, m)
    c = y * np.exp(0.5 * rng.standard_normal(m)) * rng.choice([-1.0, 1.0], m)
    s2 = np.stack([q1 * x, q1 * c, q2 * (-y * y / c), q2 * x], axis=1)
    p2 = np.stack([q1, q2], axis=1)
    b = np.sqrt(q1 * q2)
    ar[k2] = ar[k2 + 1] = x * b
    ai[k2], ai[k2 + 1] = y * b, -y * b
    be[k2] = be[k2 + 1] = b
    return k1, s1, p1, k2, s2, p2, ar, ai, be


def gen_schur_batch(sizes, seed=0, dtype=np.float64):
    """Many pencils with the statistics of gen_schur_like (diagonal blocks from
    schur_blocks, strictly upper parts N(0,1)).  Returns a list of (S, P, alphar, alphai,
    beta), Fortran-ordered."""
    rng = np.random.default_rng(seed)
    out = []
    for n in sizes:
        n = int(n)
        S = np.asfortranarray(np.triu(rng.standard_normal((n, n)), 1).astype(dtype))
        P = np.asfortranarray(np.triu(rng.standard_normal((n, n)), 1).astype(dtype))
        k1, s1, p1, k2, s2, p2, ar, ai, be = schur_blocks(n, rng)
        S[k1, k1], P[k1, k1] = s1, p1
        S[k2, k2], S[k2, k2 + 1], S[k2 + 1, k2], S[k2 + 1, k2 + 1] = s2[:, 0], s2[:, 1], s2[:, 2], s2[:, 3]
        P[k2, k2], P[k2 + 1, k2 + 1], P[k2, k2 + 1] = p2[:, 0], p2[:, 1], 0.0
        out.append((S, P, ar.astype(dtype), ai.astype(dtype), be.astype(dtype)))
    return out
