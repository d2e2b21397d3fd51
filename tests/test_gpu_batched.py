"""Batched form (xtgevc3_{d,s}tgevc3_batched_*, one persistent kernel in a CUDA graph)
against the oracle, pencil by pencil.

Every pencil of a batch must match the oracle run on that pencil alone, with the
tolerances of the single-pencil parity tests: after both sides are scaled by the oracle's
value at its largest component, elementwise difference relative to the column max below
1e-11 (FP64) / 2e-4 (FP32) on xGGES pencils, 1e-8 / 5e-3 on the ill-conditioned
Schur-form stand-in pencils.
"""
import numpy as np
import pytest

import oracle
import xtgevc3_b200 as X
from xtgevc3_b200 import pencils

pytestmark = pytest.mark.gpu

TOL = {("gges", np.float64): 1e-11, ("gges", np.float32): 2e-4,
       ("schur", np.float64): 1e-8, ("schur", np.float32): 5e-3}


def dev(a):
    """Column-major CUDA tensor holding a (copy)."""
    import torch
    t = torch.from_numpy(np.ascontiguousarray(np.asarray(a).T)).cuda().t()
    assert t.stride(0) == 1
    return t


def host_pencil(kind, n, seed, dt):
    if kind == "gges":
        S, P, ar, ai, be, Q, Z = pencils.gen_gges(n, seed, dtype=dt)
    else:
        S, P, ar, ai, be, Q, Z = pencils.gen_schur_like(n, seed, dtype=dt, with_qz=True)
    return dict(kind=kind, n=n, S=S, P=P, alphar=ar, alphai=ai, beta=be, Q=Q, Z=Z)


def device_batch(hp, side, howmny):
    import torch
    out = []
    for h in hp:
        n = h["n"]
        d = dict(S=dev(h["S"]), P=dev(h["P"]), alphar=torch.from_numpy(h["alphar"]).cuda(),
                 alphai=torch.from_numpy(h["alphai"]).cuda(), beta=torch.from_numpy(h["beta"]).cuda())
        if howmny == "B":
            d["Q"], d["Z"] = dev(h["Q"]), dev(h["Z"])
        if side in ("L", "B"):
            d["VL"] = dev(np.full((n, n), np.nan, dtype=h["S"].dtype))
        if side in ("R", "B"):
            d["VR"] = dev(np.full((n, n), np.nan, dtype=h["S"].dtype))
        out.append(d)
    return out


def check(h, d, side, howmny):
    dt = h["S"].dtype.type
    key = (side, howmny)
    cache = h.setdefault("_ref", {})
    if key not in cache:
        cache[key] = oracle.tgevc3(side, howmny, h["S"], h["P"], h["alphar"], h["beta"], alphai=h["alphai"],
                                   VL=h["Q"].copy(order="F"), VR=h["Z"].copy(order="F"))
    ref = cache[key]
    assert ref[3] == 0 and ref[2] == h["n"]
    tol = TOL[(h["kind"], dt)]
    for s, key, r in (("L", "VL", ref[0]), ("R", "VR", ref[1])):
        if side not in (s, "B"):
            continue
        V = d[key].t().cpu().numpy().T
        assert np.isfinite(V).all(), (h["n"], s)
        a = oracle.to_complex_real_storage(V, h["alphai"])
        b = oracle.to_complex_real_storage(r[:, :h["n"]], h["alphai"])
        err, cols = oracle.max_rel_diff(a, b)
        assert err <= tol, (h["n"], s, err, int(np.nanargmax(cols)))


SIZES = [1, 2, 3, 16, 31, 32, 33, 47, 64, 65, 97, 128, 150, 200, 257]


@pytest.mark.parametrize("dt", [np.float64, np.float32], ids=["d", "s"])
def test_batched_matches_oracle_per_pencil(cuda_ok, dt):
    import torch
    hp = [host_pencil("gges", n, 500 + i, dt) for i, n in enumerate(SIZES)]
    db = device_batch(hp, "B", "B")
    b = X.Batch("B", "B", db)
    b.run()
    b.wait()
    info = b.info()
    assert info["grid"] >= 1 and info["units"] >= len(hp)
    torch.cuda.synchronize()
    for h, d in zip(hp, db):
        check(h, d, "B", "B")
    b.close()


@pytest.mark.parametrize("side,howmny", [("R", "A"), ("L", "A"), ("B", "A"), ("L", "B"), ("R", "B")])
def test_batched_sides_and_howmny(cuda_ok, side, howmny):
    hp = [host_pencil("gges", n, 600 + n, np.float64) for n in (5, 40, 77, 131)]
    db = device_batch(hp, side, howmny)
    b = X.Batch(side, howmny, db)
    b.run()
    b.wait()
    for h, d in zip(hp, db):
        check(h, d, side, howmny)


@pytest.mark.parametrize("dt", [np.float64, np.float32], ids=["d", "s"])
def test_batched_every_tile_configuration_at_order_512(cuda_ok, dt):
    """Orders up to 512 (the largest of the batched workload) with every tile
    configuration; a configuration whose shared memory does not fit must be refused with
    a message, not run."""
    hp = [host_pencil("schur", n, 700 + n, dt) for n in (512, 300, 33)]
    done = 0
    for nt in (16, 32):
        for h in (32, 64):
            db = device_batch(hp, "B", "B")
            try:
                b = X.Batch("B", "B", db, config=X.batch_config(nt, h))
            except RuntimeError as e:
                assert "shared memory" in str(e), str(e)
                continue
            b.run()
            b.wait()
            for hh, d in zip(hp, db):
                check(hh, d, "B", "B")
            b.close()
            done += 1
    assert done >= 2


def test_batched_graph_relaunch_with_new_data(cuda_ok):
    """The plan binds buffers, not values: relaunching after new pencils were copied into
    the same buffers computes the new eigenvectors."""
    import torch
    sizes = (70, 129, 20)
    hp1 = [host_pencil("gges", n, 800 + n, np.float64) for n in sizes]
    hp2 = [host_pencil("gges", n, 900 + n, np.float64) for n in sizes]
    db = device_batch(hp1, "B", "B")
    b = X.Batch("B", "B", db)
    b.run()
    b.wait()
    first = [d["VR"].clone() for d in db]
    b.run()
    b.wait()
    for d, f in zip(db, first):
        assert torch.equal(d["VR"], f)  # deterministic relaunch
    for h, d in zip(hp2, db):
        for key in ("S", "P", "Q", "Z"):
            d[key].copy_(dev(h[key]))
        for key in ("alphar", "alphai", "beta"):
            d[key].copy_(torch.from_numpy(h[key]))
    b.run()
    b.wait()
    for h, d in zip(hp2, db):
        check(h, d, "B", "B")


def test_batched_tuner_sets_default(cuda_ok):
    hp = [host_pencil("gges", n, 1000 + n, np.float64) for n in (90, 180, 45, 260)]
    db = device_batch(hp, "B", "B")
    old = X.batched_get_default("d")
    try:
        cfg, ms = X.batched_tune("B", "B", db, reps=2)
        assert cfg in {X.batch_config(nt, h) for nt in (16, 32) for h in (32, 64)}
        assert ms > 0
        assert X.batched_get_default("d") == cfg
        b = X.Batch("B", "B", db)  # config 0 takes the tuned default
        assert (b.info()["nt"] << 8 | b.info()["h"]) == cfg
        b.run()
        b.wait()
        for h, d in zip(hp, db):
            check(h, d, "B", "B")
    finally:
        X.batched_set_default("d", old)


def test_batched_fp32_graded_pencils_stay_finite(cuda_ok):
    """FP32 batch of random quasi-triangular pencils of order 401-512 with the rows of P
    graded by 10^U(-8,8) (a 2x2 block's rows share one factor): consecutive rows can differ
    by 1e16, beyond what float's range allows between two overflow checks, so blocks whose
    substitution passes the per-row cap are solved again with it.  Every column must be
    finite with a DGET52-style residual below 100 (in single-precision eps)."""
    import torch
    dt = np.float32
    hp, db = [], []
    for i, n in enumerate((512, 475, 438, 401)):
        S, P, ar, ai, be = pencils.gen_quasi_triangular(n, 900 + i, dtype=dt)
        g = 10.0 ** np.random.default_rng(901 + i).uniform(-8, 8, n)
        k = 0
        while k < n:
            if ai[k] != 0 and k + 1 < n:
                g[k + 1] = g[k]
                k += 2
            else:
                k += 1
        P = np.asfortranarray((g[:, None] * P).astype(dt))
        be = np.diag(P).copy()
        hp.append(dict(n=n, S=S, P=P, ar=ar, ai=ai, be=be))
        db.append(dict(S=dev(S), P=dev(P), alphar=torch.from_numpy(ar).cuda(), alphai=torch.from_numpy(ai).cuda(),
                       beta=torch.from_numpy(be).cuda(), VL=dev(np.full((n, n), np.nan, dtype=dt)),
                       VR=dev(np.full((n, n), np.nan, dtype=dt))))
    b = X.Batch("B", "A", db)
    b.run()
    b.wait()
    torch.cuda.synchronize()
    scale = np.finfo(np.float64).eps / np.finfo(np.float32).eps
    for h, d in zip(hp, db):
        a_c, b_c = oracle.column_eigenvalues(h["ar"], h["be"], alphai=h["ai"])
        for side, key in (("R", "VR"), ("L", "VL")):
            V = d[key].t().cpu().numpy().T
            assert np.isfinite(V).all(), (h["n"], side)
            r = oracle.residual_ratio(h["S"], h["P"], oracle.to_complex_real_storage(V, h["ai"]), a_c, b_c,
                                      left=side == "L") * scale
            assert r.max() < 100, (h["n"], side, r.max())
    b.close()


def test_batched_ready_wait_expires_and_reports(cuda_ok, monkeypatch):
    """The bounded wait of a compute unit for its pencil's ready flag runs out: pencil 1's
    prep unit is left out of the plan (XTGEVC3_BATCH_WITHHOLD_READY), so its flag is never
    set, and the poll limit is shortened (XTGEVC3_BATCH_SPIN_LIMIT).  The kernel must end,
    xtgevc3_batched_wait must return 3 with its message, the other pencils must still be
    right, and a normal plan in the same process must then run cleanly."""
    hp = [host_pencil("gges", n, 1100 + n, np.float64) for n in (70, 120, 40)]
    db = device_batch(hp, "B", "B")
    monkeypatch.setenv("XTGEVC3_BATCH_SPIN_LIMIT", "2000")
    monkeypatch.setenv("XTGEVC3_BATCH_WITHHOLD_READY", "1")
    b = X.Batch("B", "B", db)
    monkeypatch.delenv("XTGEVC3_BATCH_SPIN_LIMIT")
    monkeypatch.delenv("XTGEVC3_BATCH_WITHHOLD_READY")
    b.run()
    with pytest.raises(RuntimeError, match=r"batched wait \(3\).*bounded wait"):
        b.wait()
    b.close()
    for i in (0, 2):
        check(hp[i], db[i], "B", "B")
    db2 = device_batch(hp, "B", "B")
    b2 = X.Batch("B", "B", db2)
    b2.run()
    b2.wait()
    for h, d in zip(hp, db2):
        check(h, d, "B", "B")
    b2.close()
