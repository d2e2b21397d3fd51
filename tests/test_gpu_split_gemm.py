"""The split-precision GEMMs alone (xtgevc3_split_gemm_dev) against FP64 matrix products.

C (+)= A B with FP64 operands through the tensor-core paths of the split forms: BF16 slices,
INT8 digit slices, INT8 residues (Chinese remainder theorem).  Each element's error is
measured against the scale of its exact terms, ||A(i, :)||_2 ||B(:, j)||_2 (the rounding of
the operands to t bits bounds the error by a small multiple of 2^-t times that); the
reference product is torch's FP64 matmul (itself ~1e-16 of that scale).  Shapes include
ragged edges of every tile, K at and past a stage boundary, and the accumulate mode.
Tolerance 1e-13 (t ~ 47 bits for 14 residues, ~48-49 for the slices)."""
import numpy as np
import pytest

import xtgevc3_b200 as X

pytestmark = pytest.mark.gpu


def _cm(a, torch):
    return torch.from_numpy(np.ascontiguousarray(a.T)).cuda().t()


SHAPES = [(300, 500, 700), (128, 256, 64), (129, 257, 65), (1024, 1024, 1024), (2048, 300, 4096), (33, 7, 5)]


@pytest.mark.parametrize("kind", [0, 1, 2], ids=["bf16", "int8", "crt"])
@pytest.mark.parametrize("shape", SHAPES, ids=lambda s: "x".join(map(str, s)))
def test_split_gemm_matches_fp64(cuda_ok, kind, shape):
    import torch
    M, N, K = shape
    rng = np.random.default_rng(M * 7 + N * 3 + K)
    A = rng.standard_normal((M, K)) * np.exp(rng.uniform(-3, 3, (M, 1)))  # rows of different scales
    B = rng.standard_normal((K, N)) * np.exp(rng.uniform(-3, 3, (1, N)))
    C0 = rng.standard_normal((M, N))
    dA, dB = _cm(A, torch), _cm(B, torch)
    scale = (torch.linalg.vector_norm(dA, dim=1)[:, None] * torch.linalg.vector_norm(dB, dim=0)[None, :])
    ref = dA @ dB
    C = X.split_gemm(kind, dA, dB)
    torch.cuda.synchronize()
    err = float(((C - ref).abs() / scale).max())
    assert err < 1e-13, err
    # accumulate into an existing C
    dC = _cm(C0, torch)
    X.split_gemm(kind, dA, dB, C=dC, accumulate=True)
    err2 = float(((dC - (ref + _cm(C0, torch))).abs() / (scale + 1e-300)).max())
    assert err2 < 1e-13, err2


def test_split_gemm_crt_modulus_counts(cuda_ok):
    """Fewer moduli give fewer operand bits and a larger (but bounded) error; more give less."""
    import torch
    rng = np.random.default_rng(3)
    M, N, K = 512, 512, 2048
    A, B = rng.standard_normal((M, K)), rng.standard_normal((K, N))
    dA, dB = _cm(A, torch), _cm(B, torch)
    scale = torch.linalg.vector_norm(dA, dim=1)[:, None] * torch.linalg.vector_norm(dB, dim=0)[None, :]
    ref = dA @ dB
    errs = {}
    for L in (8, 11, 14, 16):
        C = X.split_gemm(2, dA, dB, slices=L)
        errs[L] = float(((C - ref).abs() / scale).max())
    assert errs[8] < 1e-6 and errs[11] < 1e-9 and errs[14] < 1e-13 and errs[16] < 1e-14, errs
    assert errs[8] > errs[11] > errs[14], errs


def test_split_gemm_rejects_bad_arguments():
    import ctypes as ct
    lib = X.lib()
    rc = lib.xtgevc3_split_gemm_dev(None, 3, 0, 4, 4, 4, None, 4, None, 4, None, 4, 0)
    assert rc == -1 and "bad argument" in X.last_error()


def test_split_gemm_crt_pair_kernel(cuda_ok):
    """The SM-pair form of the residue GEMM (XTGEVC3_CRT_PAIR=1, tcgen05 cta_group::2) against
    FP64 on ragged and square shapes, in a child process (the kernel choice is read once per
    process)."""
    import subprocess
    import sys
    import os
    code = (
        "import numpy as np, torch, xtgevc3_b200 as X\n"
        "rng = np.random.default_rng(9)\n"
        "for M, N, K in ((300, 500, 700), (129, 257, 65), (1024, 1024, 1024), (33, 7, 5)):\n"
        "    A = torch.from_numpy(np.ascontiguousarray(rng.standard_normal((M, K)).T)).cuda().t()\n"
        "    B = torch.from_numpy(np.ascontiguousarray(rng.standard_normal((K, N)).T)).cuda().t()\n"
        "    C = X.split_gemm(2, A, B)\n"
        "    s = torch.linalg.vector_norm(A, dim=1)[:, None] * torch.linalg.vector_norm(B, dim=0)[None, :]\n"
        "    e = float(((C - A @ B).abs() / s).max())\n"
        "    assert e < 1e-13, (M, N, K, e)\n"
        "print('pair ok')\n")
    env = dict(os.environ, XTGEVC3_CRT_PAIR="1")
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, env=env, timeout=300,
                       cwd=os.path.join(os.path.dirname(__file__), ".."))
    assert r.returncode == 0 and "pair ok" in r.stdout, r.stdout + r.stderr
