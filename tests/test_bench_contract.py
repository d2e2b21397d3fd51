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
