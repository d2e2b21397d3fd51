"""Dense reference for the adjoint: the right-eigenvector forward (SIDE='R', HOWMNY='A')
restated with torch dense solves, differentiated by torch autograd (float64 / complex128
on the CPU).

The forward it restates (src/dtgevc3.cpp:616-822, 1254-1270, 1281-1470; src/ztgevc3.cpp
116-211, 528-542), per eigenvalue k with the column's shifted operator W = ac S - b P:
  coefficients: anorm, bnorm = max column sums of |S|, |P| over rows <= col + 1 (real) or
  rows <= col (complex); ascale = 1/anorm, bscale = 1/bnorm;
  real:  t = 1 / max((|ar| + |ai|) ascale, |beta| bscale, safemin), ac = t beta bscale
         ascale, b = t (ar + i ai) ascale bscale;
  complex: t = 1 / max(|alpha| ascale, |beta| bscale, safemin), ac = t ascale beta bscale,
         b = t bscale alpha ascale;
  x = [solve(W[:k,:k], -W[:k, k]); 1; 0]  (real eigenvalue / complex arithmetic),
  x = [solve(W[:k,:k], -W[:k, k:k+2] s); s; 0],  s = (-W[k,k+1], W[k,k])  (real pair).
W[:k, :k] is used only on the entries the forward reads (the upper Hessenberg band of a
real S, zeros on the subdiagonal included; the upper triangle of P and of complex
pencils), so the gradient of every other entry is zero.  Test
infrastructure only: the product never imports this module.
"""
import numpy as np
import torch


def structure_mask(S, real, band):
    """Entries the forward reads: the upper Hessenberg band of a real S (the shifted
    systems are solved as Hessenberg systems, subdiagonal zeros included), the upper
    triangle of P (triangular by contract) and of complex pencils."""
    n = S.shape[0]
    i = torch.arange(n)
    return i[:, None] <= i[None, :] + (1 if real and band else 0)


def forward(S, P, alpha, beta, alphai=None):
    """X (n x n) as torch tensors differentiable in S and P."""
    real = not torch.is_complex(S)
    n = S.shape[0]
    safemin = torch.finfo(S.real.dtype if not real else S.dtype).tiny
    i = torch.arange(n)
    nmask = (i[:, None] <= i[None, :] + (1 if real else 0))
    anorm = (S.abs() * nmask).sum(0).max()
    bnorm = (P.abs() * nmask).sum(0).max()
    ascale = 1.0 / torch.clamp(anorm, min=safemin)
    bscale = 1.0 / torch.clamp(bnorm, min=safemin)
    Sm = S * structure_mask(S, real, True)
    Pm = P * structure_mask(S, real, False)
    cols = []
    k = 0
    while k < n:
        pair = real and alphai is not None and alphai[k] != 0 and k + 1 < n
        if real:
            ar, be = float(alpha[k]), float(beta[k])
            ai = float(alphai[k]) if pair else 0.0
            den = torch.maximum(torch.maximum((abs(ar) + abs(ai)) * ascale, abs(be) * bscale),
                                torch.tensor(safemin, dtype=S.dtype))
            t = 1.0 / den
            ac = t * be * bscale * ascale
            br = t * ar * ascale * bscale
            bi = t * ai * ascale * bscale
            if abs(be) <= safemin and abs(ar) + abs(ai) > safemin:
                ac, br, bi = ac * 0, ac * 0 + 1, ac * 0
            if not pair:
                W = ac * Sm - br * Pm
                x = torch.zeros(n, dtype=S.dtype)
                if k > 0:
                    xh = torch.linalg.solve(W[:k, :k], -W[:k, k])
                    x = torch.cat([xh, torch.ones(1, dtype=S.dtype), torch.zeros(n - k - 1, dtype=S.dtype)])
                else:
                    x = torch.cat([torch.ones(1, dtype=S.dtype), torch.zeros(n - 1, dtype=S.dtype)])
                cols.append(x)
                k += 1
            else:
                b = torch.complex(br, bi)
                W = ac * Sm.to(torch.complex128) - b * Pm.to(torch.complex128)
                s = torch.stack([-W[k, k + 1], W[k, k]])
                if k > 0:
                    xh = torch.linalg.solve(W[:k, :k], -(W[:k, k:k + 2] @ s))
                    x = torch.cat([xh, s, torch.zeros(n - k - 2, dtype=torch.complex128)])
                else:
                    x = torch.cat([s, torch.zeros(n - 2, dtype=torch.complex128)])
                cols.append(x.real)
                cols.append(x.imag)
                k += 2
        else:
            a = complex(alpha[k])
            be = complex(beta[k])
            den = torch.maximum(torch.maximum(abs(a) * ascale, abs(be) * bscale),
                                torch.tensor(safemin, dtype=S.real.dtype))
            t = 1.0 / den
            ac = (t * ascale) * be * bscale
            bc = (t * bscale) * a * ascale
            if abs(be) <= safemin and abs(a) > safemin:
                ac, bc = ac * 0, ac * 0 + 1
            W = ac * Sm - bc * Pm
            if k > 0:
                xh = torch.linalg.solve(W[:k, :k], -W[:k, k])
                x = torch.cat([xh, torch.ones(1, dtype=S.dtype), torch.zeros(n - k - 1, dtype=S.dtype)])
            else:
                x = torch.cat([torch.ones(1, dtype=S.dtype), torch.zeros(n - 1, dtype=S.dtype)])
            cols.append(x)
            k += 1
    return torch.stack(cols, 1)


def gradient(S, P, alpha, beta, G, alphai=None):
    """(dL/dS, dL/dP) of L = sum(Re(conj(G) X)) as numpy arrays, by autograd."""
    St = torch.tensor(np.asarray(S), requires_grad=True)
    Pt = torch.tensor(np.asarray(P), requires_grad=True)
    X = forward(St, Pt, alpha, beta, alphai)
    Gt = torch.tensor(np.asarray(G))
    if torch.is_complex(X):
        L = (Gt.real * X.real + Gt.imag * X.imag).sum()
    else:
        L = (Gt * X).sum()
    L.backward()
    return St.grad.numpy(), Pt.grad.numpy(), X.detach().numpy()
