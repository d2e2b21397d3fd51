"""bench.py's reference arm on the CPU: the upstream library (oracle/_ref) on the bench's own
workload, here at n = 256, printing one JSON line with the contract's keys.  The reference
arm's `cpu_baseline` and `e2e` describe the line itself (same value and unit; no host-device
copies).  Skipped where the upstream library has not been built."""
import json
import os
import subprocess
import sys

import pytest

import oracle

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.skipif(not oracle.ref_available(), reason="upstream library (oracle/_ref) not built")
def test_reference_arm_json_line():
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--n", "256",
                          "--steps", "2", "--warmup", "1"], capture_output=True, text=True, timeout=300, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [ln for ln in out.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, out.stdout[-2000:]
    d = json.loads(lines[0])
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
                "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert key in d, key
    assert d["impl"] == "reference"
    assert d["higher_is_better"] is True and d["value"] > 0
    assert d["config"]["workload"].endswith("n=256")
    cb, e2e = d["cpu_baseline"], d["e2e"]
    assert cb["kind"] == "reference" and cb["cores"] >= 1 and cb["sample"]
    assert cb["value"] == d["value"] and cb["unit"] == d["unit"]
    assert e2e["value"] == d["value"] and e2e["unit"] == d["unit"]
    assert e2e["h2d_bytes_per_step"] == 0 and e2e["d2h_bytes_per_step"] == 0


def test_neighbours_brief_tolerates_missing_and_odd_legs():
    """The compact per-leg summary in `config`: ms, LAPACK's seconds and the ratio where a leg
    has them; absent (None), failed or oddly shaped legs are left out instead of raising."""
    import importlib.util
    spec = importlib.util.spec_from_file_location("bench_mod", os.path.join(ROOT, "bench.py"))
    bench = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(bench)
    legs = {"dtgexc": {"ms": 80.0, "cpu_lapack": {"seconds": 0.46}},
            "adjoint": {"d": {"ms": 12.5}},
            "dtrevc3": {"ms": 30.0},
            "ztgexc": None,
            "odd": {"ms": "x"},
            "zero": {"ms": 0.0, "cpu_lapack": {"seconds": 1.0}},
            "list": [1, 2]}
    out = bench.neighbours_brief(legs)
    assert out["dtgexc"] == {"ms": 80.0, "lapack_s": 0.46, "x_lapack": 5.75}
    assert out["adjoint"] == {"ms": 12.5} and out["dtrevc3"] == {"ms": 30.0}
    assert "ztgexc" not in out and "odd" not in out and "zero" not in out and "list" not in out


def _bench_module():
    import importlib.util
    spec = importlib.util.spec_from_file_location("bench_mod", os.path.join(ROOT, "bench.py"))
    bench = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(bench)
    return bench


def test_bench_table_pencils_follow_the_upstream_generators():
    """pencils.gen_bench_triangular, the inputs of `bench.py --reference-table`: upper
    triangular S and P with entries in [-1, 1) (complex: both parts), P's diagonal real with
    magnitude in [1, 2); alpha, beta its diagonals; seeded."""
    import numpy as np
    from xtgevc3_b200 import pencils
    for dt in (np.float64, np.float32, np.complex128, np.complex64):
        S, P, al, be = pencils.gen_bench_triangular(60, seed=3, dtype=dt)
        assert S.dtype == dt and P.dtype == dt and S.flags.f_contiguous
        assert not np.tril(S, -1).any() and not np.tril(P, -1).any()
        for M in (S, P):
            off = M[np.triu_indices(60, 1)]
            assert np.abs(off.real).max() <= 1 and np.abs(off.imag).max() <= 1
        d = np.diag(P)
        assert not d.imag.any() and (np.abs(d) >= 1).all() and (np.abs(d) < 2).all()
        assert np.array_equal(al, np.diag(S)) and np.array_equal(be, d)
        S2 = pencils.gen_bench_triangular(60, seed=3, dtype=dt)[0]
        assert np.array_equal(S, S2)


@pytest.mark.skipif(not oracle.ref_available(), reason="upstream library (oracle/_ref) not built")
def test_bench_table_reference_rows():
    """The CPU column of the table: one upstream SIDE='B', HOWMNY='A' call per type on the
    table's pencil, every eigenvector within 1e-10 (double) / 5e-3 (single) of its column's
    largest entry of the oracle's C restatement on the same input (the pencils are
    ill-conditioned: columns grow to 1e14 and more)."""
    import numpy as np
    bench = _bench_module()
    oracle.set_ref_threads(2)
    for prec, tol in (("d", 1e-10), ("s", 5e-3), ("z", 1e-10), ("c", 5e-3)):  # ill-conditioned triangular pencils
        t, VL, VR = bench.table_reference_row(prec, 48, 5)
        S, P, al, ai, be = bench.table_inputs(prec, 48, 5)
        OL, OR = (np.zeros((48, 48), dtype=S.dtype, order="F") for _ in range(2))
        OL, OR, m, info = oracle.tgevc3("B", "A", S, P, al, be, alphai=ai, VL=OL, VR=OR, impl="oracle")
        assert (m, info) == (48, 0) and t > 0
        for V, R in ((VL, OL), (VR, OR)):
            assert (np.abs(V - R).max(0) / np.abs(R).max(0)).max() < tol, prec
