#!/usr/bin/env python
"""Benchmark: dtgevc3 SIDE='B' HOWMNY='B' (left and right eigenvectors, back-transformed
by Q and Z) on an n = 8192 real pencil in generalized Schur form, on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--n 8192]

One "step" = one full dtgevc3 call (all 2n eigenvectors) on one pencil.  With N > 1
(torchrun, one process per GPU) every rank solves its own pencil: the units (pencils)
are independent, there is no data-path collective, scaling is weak.

Prints one JSON line (rank 0).  value = eigenvectors/s of the whole job with inputs
resident in HBM; e2e = the same through the host-pointer C ABI (xtgevc3_dtgevc3) from
pinned host buffers, copies included.  roofline = the dominant kernel class from the
library's CUDA-event trace against the FP64 GEMM peak measured in this run (cuBLAS
DGEMM, MEASURED_PEAKS.json has no FP64 figure).  cpu_baseline = one full call of the
upstream CPU library (oracle/_ref, OpenBLAS on all host cores) on the same pencil, Q and Z;
its result is also the reference every form is compared with elementwise
(config.max_rel_diff_vs_reference, config.forms).  --impl reference times that CPU library
alone (rank 0): one full call of the same workload per step.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "dtgevc3 n=8192 eigvecs/s vs plain FP64 GPU at resid<=1e-12; batched pencils/s"
UNIT = "eigvecs/s"
DATA = ("synthetic: seeded real generalized-Schur-form pencil with the statistics of xGGES output "
        "of N(0,1) A,B (stand-in: xGGES at n=8192 takes ~1.5 h); random orthogonal Q, Z")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=8192)
    ap.add_argument("--seed", type=int, default=8192)
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--ref-budget-s", type=float, default=240.0,
                    help="--impl reference: stop timing further full calls once this many seconds are spent")
    ap.add_argument("--form", default="all", choices=["plain", "split", "split_i8", "split_crt", "all"],
                    help="plain FP64, split precision with BF16 slices, INT8 slices or INT8 residues, or all (the "
                         "fastest one meeting the residual bound is the headline)")
    ap.add_argument("--slices", type=int, default=6, help="BF16 slices of the split form")
    ap.add_argument("--slices-i8", type=int, default=7, help="INT8 slices of the split_i8 form")
    ap.add_argument("--moduli", type=int, default=14, help="moduli of the split_crt (residue) form")
    ap.add_argument("--gemm-only", action="store_true",
                    help="time the split GEMM kinds and cuBLAS DGEMM on one n x n x n product and exit")
    ap.add_argument("--batch-count", type=int, default=2048,
                    help="pencils of the batched workload (0 skips it)")
    ap.add_argument("--batch-seed", type=int, default=2048)
    ap.add_argument("--adjoint-n", type=int, default=2048, help="order of the dtgevc3 adjoint case (0 skips)")
    ap.add_argument("--adjoint-c-count", type=int, default=256, help="complex64 pencils of the ctgevc3 adjoint case")
    ap.add_argument("--adjoint-c-n", type=int, default=128)
    ap.add_argument("--z-n", type=int, default=4096, help="order of the ztgevc3 SIDE=R HOWMNY=A leg (0 skips)")
    ap.add_argument("--trevc3-n", type=int, default=8192, help="order of the dtrevc3 SIDE=B HOWMNY=B leg (0 skips)")
    ap.add_argument("--tgexc-n", type=int, default=4096, help="order of the ztgexc and dtgexc reordering legs (0 skips)")
    ap.add_argument("--tgsen-n", type=int, default=0,
                    help="order of the dtgsen IJOB=4 leg beside LAPACK dtgsen; 0 (the default) skips it")
    ap.add_argument("--tgsna-n", type=int, default=0,
                    help="order of the dtgsna DIF leg beside LAPACK dtgsna JOB='V'; 0 (the default) skips it")
    ap.add_argument("--reference-table", action="store_true",
                    help="only the upstream benchmark table (BM_xtgevc3 rows: SIDE=B, HOWMNY=A over --table-sizes)")
    ap.add_argument("--table-sizes", default="", help="comma-separated orders (default: the upstream list)")
    ap.add_argument("--table-prec", default="dszc", help="types of the table, any of d s z c")
    ap.add_argument("--gges-sort", action="store_true",
                    help="the dgges leg orders the eigenvalues (SORT = 'S', left half-plane first)")
    ap.add_argument("--gges-n", type=int, default=0,
                    help="order of the dgges (QZ step) leg beside LAPACK dgges; 0 (the default) skips it")
    ap.add_argument("--profile-case", default=None,
                    help="run one small case for an ncu capture and exit (no JSON line): plain:N (two dtgevc3 "
                         "B/B calls, FP64; plain_norm:N with the normalisation), split_i8:N / split_crt:N (the same, INT8 digit / residue split "
                         "form), crt_gemm:N (two N^3 residue GEMMs), batch:COUNT (two launches of the batched "
                         "dtgevc3 B/B kernel, tiles 32x32)")
    return ap.parse_args()


# ----------------------------------------------------------------------------------------
# clocks during the timed region
# ----------------------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.idx = gpu_index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "100",
                 "-i", str(self.idx)], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        time.sleep(0.3)

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.2)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        rows = []
        for line in open(self.path):
            p = [x.strip() for x in line.split(",")]
            if len(p) < 9:
                continue
            try:
                rows.append((float(p[1]), float(p[2]), float(p[3]) if p[3] not in ("[N/A]", "N/A") else 0.0, p[5:9]))
            except ValueError:
                continue
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        maxmhz = max(r[1] for r in rows)
        load = [r for r in rows if r[2] > 200.0] or rows
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        reasons = sorted({names[i] for r in load for i, v in enumerate(r[3]) if v.lower() == "active"})
        return {"sm_mhz": float(np.median([r[0] for r in load])), "sm_max_mhz": maxmhz, "reasons": reasons,
                "samples": len(rows), "power_w_max": max(r[2] for r in rows)}


# ----------------------------------------------------------------------------------------
# inputs
# ----------------------------------------------------------------------------------------
def host_pencil(n, seed):
    from xtgevc3_b200 import pencils
    return pencils.gen_schur_like(n, seed)


def colmajor_cuda(a, torch):
    """numpy Fortran matrix -> column-major CUDA tensor (stride(0) == 1)."""
    return torch.from_numpy(np.ascontiguousarray(a.T)).cuda().t()


def orthogonal(n, seed, torch):
    g = torch.Generator(device="cuda")
    g.manual_seed(seed)
    A = torch.randn(n, n, device="cuda", dtype=torch.float64, generator=g)
    Q, _ = torch.linalg.qr(A)
    return Q.t().contiguous().t()  # column-major copy


def dgemm_peak(torch):
    """cuBLAS DGEMM 8192^3, best of 5 (burst), TFLOP/s: the FP64 denominator."""
    n = 8192
    a = torch.randn(n, n, device="cuda", dtype=torch.float64)
    b = torch.randn_like(a)
    for _ in range(2):
        a @ b
    torch.cuda.synchronize()
    best = 1e30
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for _ in range(5):
        e0.record()
        a @ b
        e1.record()
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1))
    del a, b
    return 2.0 * n ** 3 / (best * 1e-3) / 1e12


def int8_peak(torch):
    """cuBLASLt INT8 GEMM (torch._int_mm, INT32 accumulation) 8192^3, best of 5: the INT8
    denominator (MEASURED_PEAKS.json has none).  None if torch lacks the path."""
    n = 8192
    try:
        a = torch.randint(-128, 128, (n, n), device="cuda", dtype=torch.int8)
        b = torch.randint(-128, 128, (n, n), device="cuda", dtype=torch.int8)
        for _ in range(2):
            torch._int_mm(a, b)
        torch.cuda.synchronize()
        best = 1e30
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        for _ in range(5):
            e0.record()
            torch._int_mm(a, b)
            e1.record()
            torch.cuda.synchronize()
            best = min(best, e0.elapsed_time(e1))
        del a, b
        return 2.0 * n ** 3 / (best * 1e-3) / 1e12
    except (RuntimeError, AttributeError):
        return None


def residual_max(torch, S, P, ar, ai, be, Q, Z, VL, VR):
    """max over eigenvectors of ||beta S x - alpha P x||_1 / ((|beta| ||S||_1 + |alpha| ||P||_1) ||x||_1)
    in Schur coordinates (x = Z^T v, y = Q^T u; Q, Z orthogonal)."""
    dev = S.device
    ar_t = torch.as_tensor(ar, device=dev)
    ai_t = torch.as_tensor(ai, device=dev)
    be_t = torch.as_tensor(be, device=dev)
    nS = S.abs().sum(0).max()
    nP = P.abs().sum(0).max()
    out = []
    for left, V, B in ((False, VR, Z), (True, VL, Q)):
        W = B.t() @ V
        Sm, Pm = (S.t(), P.t()) if left else (S, P)
        SW = Sm @ W
        PW = Pm @ W
        n = W.shape[1]
        re_c = torch.zeros(n, dtype=torch.bool, device=dev)
        k = 0
        pairs = []
        ai_h = ai
        while k < n:
            if ai_h[k] != 0 and k + 1 < n:
                pairs.append(k)
                k += 2
            else:
                k += 1
        idx = torch.as_tensor(pairs, device=dev, dtype=torch.long)
        R = SW * be_t[None, :] - PW * ar_t[None, :]
        num = R.abs().sum(0)
        if len(pairs):
            sg = 1.0 if not left else -1.0
            xr, xi = idx, idx + 1
            b = be_t[xr][None, :]
            a_r, a_i = ar_t[xr][None, :], ai_t[xr][None, :]
            rr = SW[:, xr] * b - PW[:, xr] * a_r + sg * a_i * PW[:, xi]
            ri = SW[:, xi] * b - PW[:, xi] * a_r - sg * a_i * PW[:, xr]
            pn = rr.abs().sum(0) + ri.abs().sum(0)
            num[xr] = pn
            num[xi] = pn
            re_c[xr] = True
        vn = W.abs().sum(0)
        if len(pairs):
            vv = vn[idx] + vn[idx + 1]
            vn[idx] = vv
            vn[idx + 1] = vv
        amag = ar_t.abs() + ai_t.abs()
        den = (be_t.abs() * nS + amag * nP) * vn
        out.append(float((num / den).max()))
    return max(out)


# ----------------------------------------------------------------------------------------
# CPU: the upstream library on the whole workload
# ----------------------------------------------------------------------------------------
def cpu_full(S, P, ar, ai, be, Q, Z, threads):
    """One upstream dtgevc3 call with the bench's arguments (SIDE='B', HOWMNY='B', VL = Q,
    VR = Z on entry): the library built from the upstream sources (oracle/_ref) with its
    OpenBLAS on `threads` host threads, or this repository's C restatement where that
    library is absent.  Returns (VL, VR, seconds, kind)."""
    import oracle
    impl = "ref" if oracle.ref_available() else "oracle"
    if impl == "ref":
        oracle.set_ref_threads(threads)
    VL = np.array(Q, order="F", dtype=np.float64)
    VR = np.array(Z, order="F", dtype=np.float64)
    t0 = time.perf_counter()
    VL, VR, m, info = oracle.tgevc3("B", "B", S, P, ar, be, alphai=ai, VL=VL, VR=VR, impl=impl)
    t = time.perf_counter() - t0
    assert (m, info) == (S.shape[0], 0), (m, info)
    return VL, VR, t, ("reference" if impl == "ref" else "port")


def householder(n, seed):
    """A dense orthogonal n x n matrix I - 2 v v^T / (v^T v), v ~ N(0,1) seeded (host,
    Fortran order): Q / Z of the CPU arm, whose run time does not depend on their values."""
    v = np.random.default_rng(seed).standard_normal(n)
    H = -(2.0 / (v @ v)) * np.outer(v, v)
    H[np.diag_indices(n)] += 1.0
    return np.asfortranarray(H)


def host_threads():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def reference_arm(args):
    """The upstream library (the reference's CPU implementation of the path) on the bench's
    own workload: one full dtgevc3 SIDE='B' HOWMNY='B' call on the n = --n pencil per step,
    on every host thread.  Warm-up steps run the same call at n = 1024 (library, OpenBLAS
    threads and page-ins warm); timed steps stop early once --ref-budget-s is spent, so that
    the run ends within minutes (steps reports the calls timed)."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    n = args.n
    thr = host_threads()
    S, P, ar, ai, be = host_pencil(n, args.seed)
    Q, Z = householder(n, args.seed + 1), householder(n, args.seed + 2)
    nw = min(n, 1024)
    Sw, Pw, arw, aiw, bew = host_pencil(nw, args.seed + 3)
    Iw = np.eye(nw, order="F")
    for _ in range(args.warmup):
        cpu_full(Sw, Pw, arw, aiw, bew, Iw, Iw, thr)
    times, kind = [], "reference"
    t_start = time.perf_counter()
    for _ in range(args.steps):
        _, _, t, kind = cpu_full(S, P, ar, ai, be, Q, Z, thr)
        times.append(t)
        if time.perf_counter() - t_start + t > args.ref_budget_s:
            break
    t_mean = float(np.mean(times))
    v = 2 * n / t_mean
    sample = (f"upstream dtgevc3 SIDE=B HOWMNY=B, the whole n={n} job (all {2 * n} eigenvectors, "
              f"back-transform included) per step, {thr} threads")
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
            "steps": len(times), "steps_requested": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * t_mean, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": DATA,
            "config": {"workload": f"dtgevc3 SIDE=B HOWMNY=B n={n}", "n": n, "side": "B", "howmny": "B",
                       "form": "upstream CPU (OpenBLAS)", "same_config": True,
                       "warmup_calls": f"n={nw} B/B", "budget_s": args.ref_budget_s},
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": thr, "kind": kind, "sample": sample},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


# ----------------------------------------------------------------------------------------
# GPU arm
# ----------------------------------------------------------------------------------------
def load_traffic():
    """Per-launch DRAM bytes of the dominant kernel from the committed ncu summary, as bytes
    per algorithmic flop (scaled to a launch of the bench by its flops)."""
    p = os.path.join(ROOT, "profiles", "ncu_traffic.json")
    if not os.path.exists(p):
        return None
    try:
        return json.load(open(p))
    except (OSError, ValueError):
        return None




def max_over_ranks(value, dist, torch, device="cuda"):
    """The largest of the ranks' values (a time in ms, say); every rank gets it.  With no
    process group (one GPU) the value itself."""
    if not dist:
        return float(value)
    t = torch.tensor([float(value)], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def rank_seeds(seed, batch_seed, rank):
    """Seeds of one rank's inputs: each rank solves its own pencils (weak scaling)."""
    return {"pencil": seed + rank, "q": 2 * seed + 1 + 7 * rank, "z": 2 * seed + 2 + 7 * rank,
            "batch": batch_seed + 7919 * rank}


def max_rel_diff_vs(torch, V, R, ai):
    """Elementwise agreement of two real eigenvector matrices in (Re, Im) pair storage (all
    eigenvalues, ascending), on the device: both are turned into one complex eigenvector per
    column, scaled by their value at the row where |R| is largest (the comparison
    normalisation of the oracle package), and the largest |v - r| over the column's largest
    |r| is returned (max over columns).  Columns go in chunks that never split a pair."""
    n, m = V.shape
    starts, k = set(), 0
    while k < m:
        if ai[k] != 0 and k + 1 < m:
            starts.add(k)
            k += 2
        else:
            k += 1
    worst, c0 = 0.0, 0
    while c0 < m:
        c1 = min(m, c0 + 2048)
        if c1 < m and (c1 - 1) in starts:
            c1 += 1
        loc = [c - c0 for c in range(c0, c1) if c in starts]
        ix = torch.as_tensor(loc, device=V.device, dtype=torch.long)

        def cplx(W):
            C = torch.complex(W, torch.zeros_like(W))
            if loc:
                re, im = W[:, ix], W[:, ix + 1]
                C[:, ix] = torch.complex(re, im)
                C[:, ix + 1] = torch.complex(re, -im)
            return C

        Vc, Rc = cplx(V[:, c0:c1]), cplx(R[:, c0:c1])
        row = Rc.abs().argmax(0)
        cols = torch.arange(c1 - c0, device=V.device)
        a, b = Vc[row, cols], Rc[row, cols]
        a = torch.where(a == 0, torch.ones_like(a), a)
        b = torch.where(b == 0, torch.ones_like(b), b)
        Vn, Rn = Vc / a[None, :], Rc / b[None, :]
        den = Rn.abs().amax(0).clamp_min(1e-300)
        worst = max(worst, float(((Vn - Rn).abs().amax(0) / den).max()))
        del Vc, Rc, Vn, Rn
        c0 = c1
    return worst


def measure_form(name, flags, args, X, torch, data, dist, local, world, ref=None):
    """Time K steps of one form (device-resident inputs), check the residual of the result,
    then trace K more steps for the per-kernel breakdown."""
    S, P, ar, ai, be, Q, Z, VL, VR = data
    n = S.shape[0]

    def step():
        VL.copy_(Q)
        VR.copy_(Z)
        X.tgevc3_dev("B", "B", S, P, ar, be, alphai=ai, VL=VL, VR=VR, flags=flags)

    for _ in range(max(args.warmup, 1)):
        step()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    l0 = X.launch_count()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        step()
    e1.record()
    torch.cuda.synchronize()
    launches = X.launch_count() - l0
    clk = clocks.stop()
    ms = max_over_ranks(e0.elapsed_time(e1) / args.steps, dist, torch)
    resid = residual_max(torch, S, P, ar, ai, be, Q, Z, VL, VR)
    # elementwise error against the upstream library's result on the same inputs
    err = None
    if ref is not None:
        err = max(max_rel_diff_vs(torch, VL, ref[0], ai), max_rel_diff_vs(torch, VR, ref[1], ai))
    X.trace_reset()
    X.trace_enable(True)
    for _ in range(args.steps):
        step()
    torch.cuda.synchronize()
    X.trace_enable(False)
    kernels = {k: dict(v, ms_per_step=v["ms"] / args.steps) for k, v in X.trace().items() if v["launches"]}
    refined = X.split_refined() if flags & X.SPLIT else 0  # columns the last (traced) call refined
    return {"name": name, "flags": flags, "ms": ms, "value": world * 2 * n / (ms * 1e-3), "resid": resid,
            "err_vs_ref": err, "refined_columns": refined, "clocks": clk, "launches": launches, "kernels": kernels}


def measure_normalize(args, X, torch, data, peak_hbm):
    """XTGEVC3_NORMALIZE on the plain form: the one-pass normalisation kernel's time per call
    from the library trace (both sides), and its rate against the HBM peak: each entry of
    VL and VR read once and written once, 2 x 2 n^2 x 8 bytes per call."""
    S, P, ar, ai, be, Q, Z, VL, VR = data
    n = S.shape[0]
    for _ in range(max(args.warmup, 1)):
        VL.copy_(Q)
        VR.copy_(Z)
        X.tgevc3_dev("B", "B", S, P, ar, be, alphai=ai, VL=VL, VR=VR, flags=X.NORMALIZE)
    torch.cuda.synchronize()
    X.trace_reset()
    X.trace_enable(True)
    for _ in range(args.steps):
        VL.copy_(Q)
        VR.copy_(Z)
        X.tgevc3_dev("B", "B", S, P, ar, be, alphai=ai, VL=VL, VR=VR, flags=X.NORMALIZE)
    torch.cuda.synchronize()
    X.trace_enable(False)
    t = X.trace()["normalize"]
    ms = t["ms"] / args.steps
    byts = t["bytes"] / args.steps
    mx = max(float(VL.abs().amax(0).max()), float(VR.abs().amax(0).max()))
    return {"ms_per_call": ms, "bytes_per_call": byts, "gbs": byts / (ms * 1e-3) / 1e9,
            "frac_of_hbm": byts / (ms * 1e-3) / 1e9 / peak_hbm, "launches_per_call": t["launches"] / args.steps,
            "largest_entry_after": mx}


def batched_inputs(count, seed, torch):
    """The batched workload on the device: `count` pencils of orders n ~ U{16..512}
    (seeded), each in generalized Schur form with the block statistics of the single-pencil
    workload (strictly upper parts N(0,1) drawn on the device), Householder Q and Z; the
    FP32 batch is the same pencils rounded to FP32.  Returns (sizes, batches) with batches
    = {"d": [...], "s": [...]}, each pencil a dict of device tensors plus host eigenvalues."""
    from xtgevc3_b200 import pencils as gen
    rng = np.random.default_rng(seed)
    sizes = rng.integers(16, 513, size=count).astype(np.int64)
    offs = np.concatenate([[0], np.cumsum(sizes ** 2)])
    tot = int(offs[-1])
    g = torch.Generator(device="cuda")
    g.manual_seed(seed)
    out = {}
    for prec, tdt in (("d", torch.float64), ("s", torch.float32)):
        out[prec] = {k: torch.empty(tot, device="cuda", dtype=tdt) for k in ("S", "P", "Q", "Z", "VL", "VR")}
    bd, bs = out["d"], out["s"]
    plist = {"d": [], "s": []}
    for i, n in enumerate(sizes):
        n = int(n)
        o = int(offs[i])

        def view(buf):
            return buf[o:o + n * n].view(n, n).t()  # column-major n x n

        S, P, Q, Z = view(bd["S"]), view(bd["P"]), view(bd["Q"]), view(bd["Z"])
        S.copy_(torch.triu(torch.randn(n, n, generator=g, device="cuda", dtype=torch.float64), 1))
        P.copy_(torch.triu(torch.randn(n, n, generator=g, device="cuda", dtype=torch.float64), 1))
        k1, s1, p1, k2, s2, p2, ar, ai, be = gen.schur_blocks(n, rng)
        t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
        k1t, k2t = t(k1), t(k2)
        S[k1t, k1t] = t(s1)
        P[k1t, k1t] = t(p1)
        if k2.size:
            S[k2t, k2t], S[k2t, k2t + 1] = t(s2[:, 0]), t(s2[:, 1])
            S[k2t + 1, k2t], S[k2t + 1, k2t + 1] = t(s2[:, 2]), t(s2[:, 3])
            P[k2t, k2t], P[k2t + 1, k2t + 1], P[k2t, k2t + 1] = t(p2[:, 0]), t(p2[:, 1]), 0.0
        for M in (Q, Z):
            v = torch.randn(n, 1, generator=g, device="cuda", dtype=torch.float64)
            M.copy_(torch.eye(n, device="cuda", dtype=torch.float64) - (2.0 / (v.t() @ v)) * (v @ v.t()))
        for prec, b in (("d", bd), ("s", bs)):
            dt = np.float64 if prec == "d" else np.float32
            ph = dict(n=n, ar=ar.astype(dt), ai=ai.astype(dt), be=be.astype(dt))
            pd = dict(S=view(b["S"]), P=view(b["P"]), Q=view(b["Q"]), Z=view(b["Z"]), VL=view(b["VL"]),
                      VR=view(b["VR"]))
            for key in ("alphar", "alphai", "beta"):
                pd[key] = torch.from_numpy(ph[{"alphar": "ar", "alphai": "ai", "beta": "be"}[key]]).cuda()
            pd["host"] = ph
            plist[prec].append(pd)
    for k in ("S", "P", "Q", "Z"):
        bs[k].copy_(bd[k])
    return sizes, plist, out


def measure_batched(args, X, torch, dist, world):
    """The batched form (one persistent kernel in a CUDA graph per precision, tile
    configuration from the project's tuner) against a loop of per-pencil plain launches
    (xtgevc3_{d,s}tgevc3_dev) over the same pencils; both on device-resident inputs."""
    rank = int(os.environ.get("RANK", "0"))
    sizes, plist, bufs = batched_inputs(args.batch_count, rank_seeds(args.seed, args.batch_seed, rank)["batch"], torch)
    count = len(sizes)
    flops = float(np.sum(10.0 / 3.0 * sizes.astype(np.float64) ** 3))
    res = {}
    for prec in ("d", "s"):
        pens = [{k: v for k, v in p.items() if k != "host"} for p in plist[prec]]
        cfg, tune_ms = X.batched_tune("B", "B", pens, reps=2)
        plan = X.Batch("B", "B", pens)
        for _ in range(max(args.warmup, 1)):
            plan.run()
        plan.wait()
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        l0 = X.launch_count()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(args.steps):
            plan.run()
        e1.record()
        plan.wait()
        ms = e0.elapsed_time(e1) / args.steps
        launches = X.launch_count() - l0
        ms = max_over_ranks(ms, dist, torch)
        info = plan.info()
        # loop of plain per-pencil launches (in place, so VL/VR start as Q/Z each call)
        VLl = torch.empty_like(bufs[prec]["VL"])
        VRl = torch.empty_like(bufs[prec]["VR"])
        offs = np.concatenate([[0], np.cumsum(sizes ** 2)])

        def loop(idx):
            for i in idx:
                p, h = plist[prec][i], plist[prec][i]["host"]
                n, o = h["n"], int(offs[i])
                vl = VLl[o:o + n * n].view(n, n).t()
                vr = VRl[o:o + n * n].view(n, n).t()
                vl.copy_(p["Q"])
                vr.copy_(p["Z"])
                X.tgevc3_dev("B", "B", p["S"], p["P"], h["ar"], h["be"], alphai=h["ai"], VL=vl, VR=vr)

        loop(range(min(16, count)))
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        f0.record()
        loop(range(count))
        f1.record()
        torch.cuda.synchronize()
        loop_ms = f0.elapsed_time(f1)
        loop_wall = time.perf_counter() - t0
        # agreement of the two on every pencil (elementwise, relative to the column max)
        worst = 0.0
        for V, W in ((bufs[prec]["VL"], VLl), (bufs[prec]["VR"], VRl)):
            for i in range(count):
                n, o = int(sizes[i]), int(offs[i])
                a, b = V[o:o + n * n].view(n, n), W[o:o + n * n].view(n, n)  # rows = columns of V
                den = b.abs().amax(1).clamp_min(1e-300)
                worst = max(worst, float(((a - b).abs().amax(1) / den).max()))
        big = np.argsort(-sizes)[:2]
        resid = []
        for i in big:
            p, h = plist[prec][i], plist[prec][i]["host"]
            S64, P64, Q64, Z64, VL64, VR64 = (p[k].double() for k in ("S", "P", "Q", "Z", "VL", "VR"))
            resid.append(residual_max(torch, S64, P64, h["ar"].astype(np.float64), h["ai"].astype(np.float64),
                                      h["be"].astype(np.float64), Q64, Z64, VL64, VR64))
        res[prec] = {"ms": ms, "pencils_per_s": count / (ms * 1e-3), "tflops": flops / (ms * 1e-3) / 1e12,
                     "config": {"nt": info["nt"], "h": info["h"], "grid_ctas": info["grid"],
                                "units": info["units"], "tuner_ms": tune_ms},
                     "graph_launches": launches,
                     "loop_ms": loop_ms, "loop_wall_s": loop_wall, "loop_pencils_per_s": count / (loop_ms * 1e-3),
                     "speedup_vs_loop": loop_ms / ms, "max_rel_diff_vs_loop": worst,
                     "resid_max_two_largest": max(resid)}
        plan.close()
        del VLl, VRl
    tot_ms = res["d"]["ms"] + res["s"]["ms"]
    tot_loop = res["d"]["loop_ms"] + res["s"]["loop_ms"]
    return {"value": world * 2 * count / (tot_ms * 1e-3), "unit": "pencils/s",
            "workload": (f"{count} pencils per GPU, n ~ U{{16..512}} (seed {args.batch_seed}), dtgevc3 and "
                         f"stgevc3 SIDE=B HOWMNY=B, each pencil in both precisions"),
            "sum_n3_flops_per_precision": flops, "ms_per_step_both_precisions": tot_ms,
            "loop_ms_both_precisions": tot_loop, "speedup_vs_loop": tot_loop / tot_ms,
            "d": res["d"], "s": res["s"],
            "data": "synthetic Schur-form pencils (device-drawn strictly upper parts, seeded diagonal blocks), "
                    "Householder Q, Z; inputs larger than L2 (no flush)"}


def measure_adjoint(args, X, torch):
    """xtgevc3_adjoint: dL/dS, dL/dP of the right eigenvectors (SIDE='R', HOWMNY='A') for a
    seeded upstream gradient dL/dX ~ N(0,1); d at order --adjoint-n, and c on
    --adjoint-c-count complex64 pencils of order --adjoint-c-n (one call per pencil).  The
    forward runs once, outside the timed region."""
    from xtgevc3_b200 import pencils as gen
    out = {}
    n = args.adjoint_n
    S_h, P_h, ar, ai, be = gen.gen_schur_like(n, args.seed + 11)
    S, P = colmajor_cuda(S_h, torch), colmajor_cuda(P_h, torch)
    VR = torch.zeros(n, n, device="cuda", dtype=torch.float64).t()
    X.tgevc3_dev("R", "A", S, P, ar, be, alphai=ai, VR=VR)
    g = torch.Generator(device="cuda")
    g.manual_seed(args.seed + 12)
    G = torch.randn(n, n, device="cuda", dtype=torch.float64, generator=g).t()
    for _ in range(max(args.warmup, 1)):
        X.adjoint(S, P, ar, be, VR, G, alphai=ai)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        dS, dP = X.adjoint(S, P, ar, be, VR, G, alphai=ai)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / args.steps
    # masked gradient GEMMs (2 x 2 n^3) plus the transposed solves (~ n^3 / 3 x 2)
    fl = 2 * 2.0 * n ** 3 + 2.0 * n ** 3 / 3.0
    out["d"] = {"n": n, "ms": ms, "gradients_per_s": 1e3 / ms, "tflops_nominal": fl / (ms * 1e-3) / 1e12,
                "finite": bool(torch.isfinite(dS).all() and torch.isfinite(dP).all())}
    cnt, nc = args.adjoint_c_count, args.adjoint_c_n
    cases = []
    for i in range(cnt):
        Sc, Pc, al, bc = gen.gen_upper_triangular_complex(nc, args.seed + 100 + i, dtype=np.complex64)
        Sd, Pd = colmajor_cuda(Sc, torch), colmajor_cuda(Pc, torch)
        V = torch.zeros(nc, nc, device="cuda", dtype=torch.complex64).t()
        X.tgevc3_dev("R", "A", Sd, Pd, al, bc, VR=V)
        Gc = torch.randn(nc, nc, device="cuda", dtype=torch.complex64, generator=g).t()
        cases.append((Sd, Pd, al, bc, V, Gc))
    for c in cases[:4]:
        X.adjoint(c[0], c[1], c[2], c[3], c[4], c[5])
    torch.cuda.synchronize()
    e0.record()
    for c in cases:
        X.adjoint(c[0], c[1], c[2], c[3], c[4], c[5])
    e1.record()
    torch.cuda.synchronize()
    msc = e0.elapsed_time(e1)
    out["c"] = {"pencils": cnt, "n": nc, "ms_all": msc, "gradients_per_s": cnt / (msc * 1e-3),
                "path": "one xtgevc3_adjoint call per pencil"}
    return out


def measure_ztgevc3(args, X, torch):
    """ztgevc3 SIDE='R', HOWMNY='A' on a complex upper-triangular pencil of order --z-n
    (the structure of the upstream complex test generator), plus a graded variant whose
    rows of P are scaled by 10^U(-8, 8) so that eigenvalues span many orders of magnitude
    and the overflow guards rescale columns.  Device-resident inputs, CUDA-event timing."""
    from xtgevc3_b200 import pencils as gen
    n = args.z_n
    out = {}
    for name in ("standard", "graded"):
        S_h, P_h, al, be = gen.gen_upper_triangular_complex(n, args.seed + 21)
        if name == "graded":
            rng = np.random.default_rng(args.seed + 22)
            P_h = np.asfortranarray((10.0 ** rng.uniform(-8, 8, n))[:, None] * P_h)
            be = np.diag(P_h).copy()
        S, P = colmajor_cuda(S_h, torch), colmajor_cuda(P_h, torch)
        VR = torch.zeros(n, n, dtype=torch.complex128, device="cuda").t()
        for _ in range(max(args.warmup, 1)):
            X.tgevc3_dev("R", "A", S, P, al, be, VR=VR)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(args.steps):
            X.tgevc3_dev("R", "A", S, P, al, be, VR=VR)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / args.steps
        # residual max_c ||beta S x - alpha P x||_1 / ((|beta| ||S||_1 + |alpha| ||P||_1) ||x||_1)
        a_t = torch.as_tensor(al, device="cuda")
        b_t = torch.as_tensor(be, device="cuda")
        R = (S @ VR) * b_t[None, :] - (P @ VR) * a_t[None, :]
        den = (b_t.abs() * S.abs().sum(0).max() + a_t.abs() * P.abs().sum(0).max()) * VR.abs().sum(0)
        resid = float((R.abs().sum(0) / den).max())
        guarded = int((torch.diagonal(VR).abs() < 1).sum())
        out[name] = {"ms": ms, "eigvecs_per_s": n / (ms * 1e-3), "tflops": 8.0 / 3.0 * n ** 3 / (ms * 1e-3) / 1e12,
                     "resid_max": resid, "columns_rescaled_by_guards": guarded,
                     "finite": bool(torch.isfinite(torch.view_as_real(VR)).all())}
        del S, P, VR, R
    return {"n": n, "side": "R", "howmny": "A",
            "data": "complex upper-triangular stand-in pencils (U(-1,1) parts, |P_kk| kept away from 0); "
                    "graded: rows of P scaled by 10^U(-8,8)", **out}


def measure_tgexc(args, X, torch, real=False):
    """ztgexc (or dtgexc with `real`): the last eigenvalue of an upper-triangular pencil of
    order --tgexc-n moves to the top (n - 1 swaps), Q and Z updated (Q = Z = I: the rotations
    cost the same whatever their values); device-resident inputs restored before each step
    outside the timed region, CUDA-event timing; LAPACK Z/DTGEXC (SciPy's OpenBLAS) on the
    same input and move beside it, with the largest difference between the two results."""
    from xtgevc3_b200 import pencils as gen
    n = args.tgexc_n
    if real:  # real eigenvalues only (1x1 blocks): the pencil class the real entry points take
        rng = np.random.default_rng(args.seed + 43)
        S_h = np.asfortranarray(np.triu(rng.standard_normal((n, n))))
        P_h = np.triu(rng.standard_normal((n, n)))
        P_h[np.diag_indices(n)] = np.abs(P_h[np.diag_indices(n)]) + 0.5
        P_h = np.asfortranarray(P_h)
    else:
        S_h, P_h, _, _ = gen.gen_upper_triangular_complex(n, args.seed + 41)
    dt_t, dt_n = (torch.float64, np.float64) if real else (torch.complex128, np.complex128)
    S0, P0 = colmajor_cuda(S_h, torch), colmajor_cuda(P_h, torch)
    I0 = torch.eye(n, dtype=dt_t, device="cuda")
    A, B, Q, Z = (torch.empty_like(S0) for _ in range(4))
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ts, res = [], None
    warm = max(args.warmup, 1)
    for it in range(warm + args.steps):
        A.copy_(S0)
        B.copy_(P0)
        Q.copy_(I0)
        Z.copy_(I0)
        torch.cuda.synchronize()
        e0.record()
        res = X.tgexc_dev(A, B, Q, Z, n, 1)
        e1.record()
        torch.cuda.synchronize()
        if it >= warm:
            ts.append(e0.elapsed_time(e1))
    ms = float(np.mean(ts))
    out = {"n": n, "move": f"{n} -> 1", "swaps": n - 1, "ilst_info": list(res), "ms": ms,
           "swaps_per_s": (n - 1) / (ms * 1e-3),
           "data": ("real upper-triangular pencil (N(0,1) parts, |P_kk| >= 0.5), Q = Z = I" if real else
                    "complex upper-triangular stand-in pencil (U(-1,1) parts, |P_kk| kept away from 0), Q = Z = I")}
    if not args.no_cpu:
        import oracle
        Ih = np.eye(n, dtype=dt_n, order="F")
        t0 = time.perf_counter()
        ra, rb, rq, rz, rinfo = oracle.lapack_tgexc(S_h, P_h, Ih, Ih.copy(order="F"), n, 1)
        tc = time.perf_counter() - t0
        diff = 0.0
        for D, R in ((A, ra), (B, rb), (Q, rq), (Z, rz)):
            diff = max(diff, float(np.abs(D.cpu().numpy() - R).max() / np.abs(R).max()))
        out["cpu_lapack"] = {"seconds": tc, "swaps_per_s": (n - 1) / tc, "cores": host_threads(), "info": int(rinfo),
                             "kind": f"LAPACK {'d' if real else 'z'}tgexc (SciPy OpenBLAS), one call"}
        out["max_rel_diff_vs_lapack"] = diff
    del S0, P0, I0, A, B, Q, Z
    return out


def measure_tgexc_blocks(args, X, torch):
    """dtgexc across 2x2 blocks: the last diagonal block of a real generalized Schur pencil of
    order --tgexc-n (the xGGES-statistics stand-in: about n - sqrt(2n/pi) eigenvalues in
    standardised 2x2 blocks) moves to the top, Q and Z updated (Q = Z = I); one swap of two
    2x2 blocks solves a 4 x 4 pair of Sylvester equations (an 8 x 8 Kronecker system) on one
    thread and updates 4 rows and columns.  Device-resident inputs restored before each
    step outside the timed region, CUDA-event timing; LAPACK DTGEXC (SciPy's OpenBLAS) on the
    same input and move beside it, results compared up to the sign of each column of Q and Z
    (LAPACK's choice between two re-triangularisations of a swapped 2x2 block follows its
    rounding noise)."""
    from xtgevc3_b200 import pencils as gen
    n = args.tgexc_n
    S_h, P_h = gen.gen_schur_like(n, args.seed + 47)[:2]
    S0, P0 = colmajor_cuda(S_h, torch), colmajor_cuda(P_h, torch)
    I0 = torch.eye(n, dtype=torch.float64, device="cuda")
    A, B, Q, Z = (torch.empty_like(S0) for _ in range(4))
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ts, res = [], None
    warm = max(args.warmup, 1)
    for it in range(warm + args.steps):
        A.copy_(S0)
        B.copy_(P0)
        Q.copy_(I0)
        Z.copy_(I0)
        torch.cuda.synchronize()
        e0.record()
        res = X.tgexc_dev(A, B, Q, Z, n, 1, with_ifst=True)
        e1.record()
        torch.cuda.synchronize()
        if it >= warm:
            ts.append(e0.elapsed_time(e1))
    ms = float(np.mean(ts))
    pairs = int((np.diag(S_h, -1) != 0).sum())
    out = {"n": n, "move": f"{n} -> 1", "pairs_in_pencil": pairs, "ifst_ilst_info": list(res), "ms": ms,
           "data": "real generalized Schur stand-in (xGGES statistics, standardised 2x2 blocks), Q = Z = I"}
    if not args.no_cpu:
        import oracle
        Ih = np.eye(n, order="F")
        t0 = time.perf_counter()
        r = oracle.lapack_tgexc_real(S_h, P_h, Ih, Ih.copy(order="F"), n, 1)
        tc = time.perf_counter() - t0
        qd, zd = Q.cpu().numpy(), Z.cpu().numpy()
        dq = np.where(np.einsum("ij,ij->j", qd, r[2]) < 0, -1.0, 1.0)
        dz = np.where(np.einsum("ij,ij->j", zd, r[3]) < 0, -1.0, 1.0)
        diff = 0.0
        for D, R in ((dq[:, None] * A.cpu().numpy() * dz[None, :], r[0]), (dq[:, None] * B.cpu().numpy() * dz[None, :], r[1]),
                     (qd * dq[None, :], r[2]), (zd * dz[None, :], r[3])):
            diff = max(diff, float(np.abs(D - R).max() / np.abs(R).max()))
        out["cpu_lapack"] = {"seconds": tc, "cores": host_threads(), "ifst_ilst_info": [int(v) for v in r[4:]],
                             "kind": "LAPACK dtgexc (SciPy OpenBLAS), one call"}
        out["speedup_vs_lapack"] = tc / (ms * 1e-3)
        out["max_rel_diff_vs_lapack_up_to_column_signs"] = diff
    del S0, P0, I0, A, B, Q, Z
    return out


def measure_gges(args, X, torch):
    """dgges (the QZ step) on an iid N(0,1) real pencil of order --gges-n, Q and Z formed:
    device-resident inputs restored before each step outside the timed region, CUDA-event
    timing; LAPACK DGGES (SciPy's OpenBLAS) on the same pencil beside it, the eigenvalues
    compared (each matched to its nearest).  With --gges-sort both order the eigenvalues of the
    left half-plane first (SORT = 'S', SELCTG alphar * beta < 0; xtgevc3_dgges_sort_dev, the
    reordering kernel inside the timed region) and SDIM is compared too."""
    n = args.gges_n
    sort = (lambda ar, ai, b: ar * b < 0) if args.gges_sort else None
    rng = np.random.default_rng(args.seed + 53)
    A_h, B_h = np.asfortranarray(rng.standard_normal((n, n))), np.asfortranarray(rng.standard_normal((n, n)))
    A0, B0 = colmajor_cuda(A_h, torch), colmajor_cuda(B_h, torch)
    A, B, Q, Z = (torch.empty_like(A0) for _ in range(4))
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ts, res = [], None
    for it in range(max(args.warmup, 1) + args.steps):
        A.copy_(A0)
        B.copy_(B0)
        torch.cuda.synchronize()
        e0.record()
        res = X.gges_dev(A, B, Q, Z, sort=sort)
        e1.record()
        torch.cuda.synchronize()
        if it >= max(args.warmup, 1):
            ts.append(e0.elapsed_time(e1))
    ms = float(np.mean(ts))
    ar, ai, be = (t.cpu().numpy() for t in res[:3])
    out = {"n": n, "ms": ms, "info": int(res[-1]), "sort": "S (left half-plane first)" if sort else "N",
           "data": "iid N(0,1) real pencil, Q and Z formed"}
    if sort:
        out["sdim"] = int(res[3])
    if not args.no_cpu:
        import scipy.linalg.lapack as la
        t0 = time.perf_counter()
        if sort:
            r = la.dgges(lambda x, y, z: int(x * z < 0), A_h.copy(order="F"), B_h.copy(order="F"), sort_t=1)
        else:
            r = la.dgges(lambda x, y, z: 0, A_h.copy(order="F"), B_h.copy(order="F"), sort_t=0)
        tc = time.perf_counter() - t0
        if sort:
            out["sdim_lapack"] = int(r[2])
        ref = (r[3] + 1j * r[4]) / r[5]
        fin = be != 0
        ev = (ar[fin] + 1j * ai[fin]) / be[fin]
        err = max([float(np.min(np.abs(ref - e)) / max(1.0, abs(e))) for e in ev] + [0.0])
        out["cpu_lapack"] = {"seconds": tc, "cores": host_threads(),
                             "kind": f"LAPACK dgges (SciPy OpenBLAS), SORT='{'S' if sort else 'N'}'"}
        out["speedup_vs_lapack"] = tc / (ms * 1e-3)
        out["max_eigenvalue_rel_diff_vs_lapack"] = err
    del A0, B0, A, B, Q, Z
    return out


def measure_tgsen(args, X, torch):
    """dtgsen IJOB = 4 (reordering with PL, PR and the Frobenius-norm DIF estimates) on a real
    generalized Schur stand-in of order --tgsen-n (xGGES statistics), the eigenvalues of the left
    half-plane selected, Q and Z updated: device-resident inputs restored before each step
    outside the timed region, CUDA-event timing of xtgevc3_dtgsen_dev; LAPACK DTGSEN (SciPy's
    OpenBLAS) on the same pencil beside it, with M, PL, PR and the DIF ratio compared."""
    from xtgevc3_b200 import pencils as gen
    import scipy.linalg.lapack as la
    n = args.tgsen_n
    S_h, P_h = gen.gen_schur_like(n, args.seed + 61)[:2]
    Q_h = Z_h = np.asfortranarray(np.eye(n))
    ar = np.diag(S_h).copy()
    for k in range(n - 1):  # the real parts of the pairs, from the 2x2 blocks' trace / 2
        if S_h[k + 1, k] != 0:
            ar[k] = ar[k + 1] = 0.5 * (S_h[k, k] / P_h[k, k] + S_h[k + 1, k + 1] / P_h[k + 1, k + 1])
    sel = (ar * np.sign(np.diag(P_h)) < 0).astype(np.int32)
    tensors = [colmajor_cuda(M, torch) for M in (S_h, P_h, Q_h, Z_h)]
    work = [torch.empty_like(t) for t in tensors]
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ts, res = [], None
    for it in range(max(args.warmup, 1) + args.steps):
        for w, t in zip(work, tensors):
            w.copy_(t)
        torch.cuda.synchronize()
        e0.record()
        res = X.tgsen_dev(sel, *work, ijob=4)
        e1.record()
        torch.cuda.synchronize()
        if it >= max(args.warmup, 1):
            ts.append(e0.elapsed_time(e1))
    ms = float(np.mean(ts))
    m, pl, pr, dif, info = res[3:]
    out = {"n": n, "ms": ms, "ijob": 4, "m": int(m), "info": int(info), "pl": pl, "pr": pr, "dif": [float(v) for v in dif],
           "data": "real generalized Schur stand-in (xGGES statistics), left half-plane selected, Q = Z = I"}
    if not args.no_cpu:
        lw = max(4 * n + 16, 2 * int(m) * (n - int(m))) + 64
        t0 = time.perf_counter()
        r = la.dtgsen(sel, S_h, P_h, Q_h, Z_h, ijob=4, lwork=lw, liwork=n + 64)
        tc = time.perf_counter() - t0
        out["cpu_lapack"] = {"seconds": tc, "cores": host_threads(), "kind": "LAPACK dtgsen IJOB=4 (SciPy OpenBLAS)"}
        out["speedup_vs_lapack"] = tc / (ms * 1e-3)
        out["m_equal"] = int(r[7]) == int(m)
        out["pl_pr_rel_diff"] = float(max(abs(pl - r[8]) / r[8], abs(pr - r[9]) / r[9])) if r[8] > 0 else None
        out["dif_ratio_to_lapack"] = [float(a / b) for a, b in zip(dif, r[10])]
    del tensors, work
    return out


def measure_tgsna_dif(args, X, torch):
    """dtgsna JOB='V' (DIF of every eigenvalue) on a real generalized Schur stand-in of order
    --tgsna-n (xGGES statistics): CUDA-event timing of xtgevc3_dtgsna_dif_dev on device-resident
    S, P; LAPACK DTGSNA (SciPy's OpenBLAS) on the same pencil beside it, with the share of DIFs
    equal to LAPACK's (1e-12) and the largest ratio between the two estimates."""
    from xtgevc3_b200 import pencils as gen
    import oracle
    n = args.tgsna_n
    S_h, P_h = gen.gen_schur_like(n, args.seed + 59)[:2]
    S0, P0 = colmajor_cuda(S_h, torch), colmajor_cuda(P_h, torch)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ts, dif = [], None
    for it in range(max(args.warmup, 1) + args.steps):
        torch.cuda.synchronize()
        e0.record()
        dif, m, info = X.tgsna_dif_dev(S0, P0)
        e1.record()
        torch.cuda.synchronize()
        if it >= max(args.warmup, 1):
            ts.append(e0.elapsed_time(e1))
    ms = float(np.mean(ts))
    out = {"n": n, "ms": ms, "eigenvalues": int(m), "info": int(info),
           "data": "real generalized Schur stand-in (xGGES statistics, standardised 2x2 blocks)"}
    if not args.no_cpu:
        t0 = time.perf_counter()
        _, d, _, _ = oracle.lapack_tgsna("A", S_h, P_h, None, None, job="V")
        tc = time.perf_counter() - t0
        h = dif.cpu().numpy()
        same = np.abs(h - d) <= 1e-12 * np.abs(d)
        ratio = np.maximum(h / d, d / h)
        out["cpu_lapack"] = {"seconds": tc, "cores": host_threads(), "kind": "LAPACK dtgsna JOB='V' (SciPy OpenBLAS)"}
        out["speedup_vs_lapack"] = tc / (ms * 1e-3)
        out["share_equal_to_lapack"] = float(same.mean())
        out["max_ratio_to_lapack"] = float(ratio[np.isfinite(ratio)].max()) if np.isfinite(ratio).any() else None
    del S0, P0
    return out


def neighbours_brief(legs):
    """One compact entry per LAPACK-neighbour leg for the `config` block (device ms; LAPACK's
    seconds on the host and the ratio where the leg timed it).  A leg that is absent, failed
    or shaped otherwise is left out: this summary must never stop the line from printing."""
    out = {}
    for name, leg in legs.items():
        try:
            if not isinstance(leg, dict):
                continue
            ms = leg.get("ms")
            if ms is None and isinstance(leg.get("d"), dict):
                ms = leg["d"].get("ms")
            if ms is None:
                continue
            e = {"ms": round(float(ms), 3)}
            cpu = leg.get("cpu_lapack")
            if isinstance(cpu, dict) and cpu.get("seconds"):
                e["lapack_s"] = round(float(cpu["seconds"]), 3)
                e["x_lapack"] = round(float(cpu["seconds"]) / (float(ms) * 1e-3), 2)
            out[name] = e
        except (TypeError, ValueError, KeyError, ZeroDivisionError):
            continue
    return out


def schur_stand_in(n, seed):
    """Stand-in for the real Schur factor T of an n x n iid N(0,1) matrix (host, Fortran):
    strictly upper part N(0,1); about sqrt(2n/pi) real eigenvalues, uniform on [-sqrt(n),
    sqrt(n)], and the rest complex pairs uniform in the disk of radius sqrt(n) (the circular
    law), in random order; each pair a LAPACK-standardised block [[a, b], [c, a]] with
    b c = -w^2 and |b| / |c| = exp(2 N(0,1)), so both of LAPACK xTREVC3's seed branches occur.
    xGEES of an 8192 matrix takes minutes on the host, hence the stand-in.  Returns (T,
    eigenvalue real parts, imaginary parts)."""
    rng = np.random.default_rng(seed)
    T = np.triu(rng.standard_normal((n, n)), 1)
    nreal = int(round(np.sqrt(2 * n / np.pi)))
    nreal += (n - nreal) % 2
    kinds = np.array([0] * nreal + [1] * ((n - nreal) // 2))
    rng.shuffle(kinds)
    wr, wi = np.zeros(n), np.zeros(n)
    r, k = np.sqrt(n), 0
    for kd in kinds:
        if kd == 0:
            wr[k] = rng.uniform(-r, r)
            T[k, k] = wr[k]
            k += 1
        else:
            rad, th = r * np.sqrt(rng.random()), rng.uniform(0, np.pi)
            a, w = rad * np.cos(th), rad * np.sin(th)
            t = np.exp(rng.standard_normal())
            T[k, k] = T[k + 1, k + 1] = a
            T[k, k + 1], T[k + 1, k] = w * t, -w / t
            wr[k] = wr[k + 1] = a
            wi[k], wi[k + 1] = w, -w
            k += 2
    return np.asfortranarray(T), wr, wi


def measure_trevc3(args, X, torch):
    """dtrevc3 (the standard problem, P = I) SIDE='B', HOWMNY='B' at n = --trevc3-n on the
    Schur-factor stand-in, device-resident, CUDA-event timing; residuals of both sides
    against A = Q T Q^T on the device; LAPACK dtrevc3 (SciPy's OpenBLAS, all host threads)
    on the same kind of input at n = 2048, beside this library at that size."""
    n = args.trevc3_n
    out = {"n": n, "side": "B", "howmny": "B"}

    def run(nn, seed, steps, warm):
        T_h, wr, wi = schur_stand_in(nn, seed)
        T = colmajor_cuda(T_h, torch)
        Q = orthogonal(nn, seed + 1, torch)
        VL, VR = torch.empty_like(Q), torch.empty_like(Q)
        ts = []
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        for it in range(warm + steps):
            VL.copy_(Q)
            VR.copy_(Q)
            torch.cuda.synchronize()
            e0.record()
            X.trevc3_dev("B", "B", T, VL=VL, VR=VR)
            e1.record()
            torch.cuda.synchronize()
            if it >= warm:
                ts.append(e0.elapsed_time(e1))
        return T_h, wr, wi, T, Q, VL, VR, float(np.mean(ts))

    T_h, wr, wi, T, Q, VL, VR, ms = run(n, args.seed + 31, args.steps, max(args.warmup, 1))
    A = Q @ T @ Q.t()
    # columns of a pair (a +- i w): Re col j, Im col j+1; partner index and coupling per column
    part = np.arange(n)
    cpl = np.zeros(n)
    k = 0
    while k < n:
        if wi[k] != 0:
            part[k], part[k + 1] = k + 1, k
            cpl[k], cpl[k + 1] = wi[k], -wi[k]
            k += 2
        else:
            k += 1
    a_t = torch.as_tensor(wr, device="cuda")
    c_t = torch.as_tensor(cpl, device="cuda")
    p_t = torch.as_tensor(part, device="cuda")
    nA = A.abs().sum(0).max()
    resid = {}
    for side, V, M, sg in (("R", VR, A, 1.0), ("L", VL, A.t(), -1.0)):
        R = M @ V - V * a_t[None, :] + sg * V[:, p_t] * c_t[None, :]
        den = nA * (V.abs().sum(0) + (c_t != 0) * V[:, p_t].abs().sum(0))
        resid[side] = float((R.abs().sum(0) / den).max())
        del R
    out.update({"ms": ms, "eigvecs_per_s": 2 * n / (ms * 1e-3),
                "algorithmic_flops": 2 * (n ** 3 / 3 + n ** 3), "tflops": 2 * (n ** 3 / 3 + n ** 3) / (ms * 1e-3) / 1e12,
                "resid_max_right": resid["R"], "resid_max_left": resid["L"],
                "finite": bool(torch.isfinite(VL).all() and torch.isfinite(VR).all()),
                "data": "stand-in real Schur factor (circular-law eigenvalues, N(0,1) strictly upper part, "
                        "LAPACK-standardised 2x2 blocks), Q from the QR of a Gaussian matrix",
                "resid": "max_c ||A v - lambda v||_1 / (||A||_1 ||v||_1), A = Q T Q^T (left: A^T, conj lambda)"})
    del A, T, Q, VL, VR
    if not args.no_cpu:
        import oracle
        nc = 2048
        T_h, _, _, _, Qc, _, _, msg = run(nc, args.seed + 32, 3, 1)
        Qh = Qc.cpu().numpy()
        thr = host_threads()
        if oracle.ref_available():
            oracle.set_ref_threads(thr)  # the same OpenBLAS instance as the LAPACK oracle
        t0 = time.perf_counter()
        _, _, mc, info = oracle.lapack_trevc3("B", "B", T_h, VL=Qh, VR=Qh)
        tc = time.perf_counter() - t0
        out["cpu_lapack_n2048"] = {"value": 2 * nc / tc, "unit": "eigvecs/s", "seconds": tc, "cores": thr,
                                   "info": info, "gpu_ms_same_n": msg,
                                   "gpu_eigvecs_per_s_same_n": 2 * nc / (msg * 1e-3),
                                   "kind": "LAPACK dtrevc3 (SciPy OpenBLAS), one call"}
    return out


def profile_case(args):
    """Small, fixed workloads for ncu captures (profiles/*.md name the exact command)."""
    import torch
    import xtgevc3_b200 as X
    kind, _, size = args.profile_case.partition(":")
    size = int(size)
    if kind == "crt_gemm":  # two residue GEMMs of size^3 (14 moduli)
        g = torch.Generator(device="cuda")
        g.manual_seed(1)
        A = torch.randn(size, size, device="cuda", dtype=torch.float64, generator=g).t()
        B = torch.randn(size, size, device="cuda", dtype=torch.float64, generator=g).t()
        for _ in range(2):
            C = X.split_gemm(2, A, B, slices=14)
        torch.cuda.synchronize()
        print(json.dumps({"case": args.profile_case, "fp64_flops": 2.0 * size ** 3,
                          "max_abs": float(C.abs().max())}))
        return 0
    if kind in ("plain", "plain_norm", "split_i8", "split_crt"):
        flags = {"plain": 0, "plain_norm": X.NORMALIZE, "split_i8": X.SPLIT | X.SPLIT_INT8 | X.slices(7),
                 "split_crt": X.SPLIT | X.SPLIT_CRT | X.slices(14)}[kind]
        S_h, P_h, ar, ai, be = host_pencil(size, 3)
        S, P = colmajor_cuda(S_h, torch), colmajor_cuda(P_h, torch)
        Q, Z = orthogonal(size, 4, torch), orthogonal(size, 5, torch)
        VL, VR = torch.empty_like(Q), torch.empty_like(Z)
        for _ in range(2):
            VL.copy_(Q)
            VR.copy_(Z)
            X.tgevc3_dev("B", "B", S, P, ar, be, alphai=ai, VL=VL, VR=VR, flags=flags)
        torch.cuda.synchronize()
        kext, k = [], 0
        while k < size:
            w = 2 if (ai[k] != 0 and k + 1 < size) else 1
            kext += [k + w] * w
            k += w
        print(json.dumps({"case": args.profile_case, "back_flops_per_side": 2.0 * size * sum(kext)}))
    elif kind == "batch":
        sizes, plist, _ = batched_inputs(size, 5, torch)
        pens = [{k: v for k, v in p.items() if k != "host"} for p in plist["d"]]
        b = X.Batch("B", "B", pens, config=X.batch_config(32, 32))
        for _ in range(2):
            b.run()
        b.wait()
        print(json.dumps({"case": args.profile_case, "flops": float(np.sum(10.0 / 3.0 * sizes.astype(float) ** 3))}))
    else:
        raise SystemExit(f"unknown profile case {args.profile_case}")
    return 0


def gemm_only(args):
    """Split GEMM kinds and cuBLAS DGEMM on one n x n x n FP64 product (no JSON line)."""
    import torch
    import xtgevc3_b200 as X
    n = min(args.n, 16384)
    g = torch.Generator(device="cuda")
    g.manual_seed(1)
    A = torch.randn(n, n, device="cuda", dtype=torch.float64, generator=g).t()
    B = torch.randn(n, n, device="cuda", dtype=torch.float64, generator=g).t()
    C = torch.empty(n, n, device="cuda", dtype=torch.float64).t()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    out = {}
    ref = A @ B
    for name, fn in (("dgemm", lambda: torch.matmul(A, B, out=C)),
                     ("bf16_6", lambda: X.split_gemm(0, A, B, C=C, slices=6)),
                     ("int8_7", lambda: X.split_gemm(1, A, B, C=C, slices=7)),
                     ("crt_14", lambda: X.split_gemm(2, A, B, C=C, slices=14))):
        for _ in range(2):
            fn()
        torch.cuda.synchronize()
        e0.record()
        for _ in range(3):
            fn()
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / 3
        err = float((C - ref).abs().max() / ref.abs().max())
        out[name] = {"ms": ms, "fp64_equiv_tflops": 2.0 * n ** 3 / (ms * 1e-3) / 1e12, "max_err_rel": err}
    print(json.dumps({"n": n, "gemm": out}), flush=True)
    return 0


# the upstream benchmark's sizes (benchmarks/bench_dtgevc3.cpp:18)
REF_TABLE_SIZES = (500, 707, 1000, 1414, 2000, 2828, 4000, 5657, 8000)
_TABLE_TYPES = {"d": np.float64, "s": np.float32, "z": np.complex128, "c": np.complex64}


def table_inputs(prec, n, seed):
    """The pencil of one row of the upstream benchmark table: (S, P, alpha, alphai, beta) on
    the host (alphai zeros for real types, None for complex)."""
    from xtgevc3_b200 import pencils as gen
    dt = _TABLE_TYPES[prec]
    S, P, al, be = gen.gen_bench_triangular(n, seed=seed, dtype=dt)
    ai = np.zeros(n, dtype=dt) if prec in "ds" else None
    return S, P, al, ai, be


def table_reference_row(prec, n, seed):
    """One upstream xtgevc3 call (SIDE='B', HOWMNY='A') on the row's pencil, the library built
    from the upstream sources (oracle/_ref) on the threads set by oracle.set_ref_threads:
    returns (seconds, VL, VR)."""
    import oracle
    S, P, al, ai, be = table_inputs(prec, n, seed)
    dt = S.dtype
    VL, VR = (np.zeros((n, n), dtype=dt, order="F") for _ in range(2))
    t0 = time.perf_counter()
    VL, VR, m, info = oracle.tgevc3("B", "A", S, P, al, be, alphai=ai, VL=VL, VR=VR, impl="ref")
    t = time.perf_counter() - t0
    assert (m, info) == (n, 0), (prec, n, m, info)
    return t, VL, VR


def reference_table(args):
    """The upstream benchmark table on this GPU.  benchmarks/bench_{d,s,z,c}tgevc3.cpp time
    xtgevc3 (BM_xtgevc3) at n = 500, 707, ..., 8000 with SIDE='B', HOWMNY='A' on triangular
    pencils (pencils.gen_bench_triangular: their distributions, seeded numpy draws).  Per type
    (--table-prec) and n (--table-sizes): the device form on resident inputs (CUDA events,
    mean of --steps after --warmup), the host-pointer call as the upstream benchmark makes it
    (host arrays in and out, every copy inside; wall clock, best of --steps), and beside them
    the upstream library (oracle/_ref) on every host thread, one call per row until
    --ref-budget-s is spent (later rows: null), with the largest column difference between its
    output and the host-pointer call's (both in the upstream scaling).  Prints one JSON line."""
    import torch
    import oracle
    import xtgevc3_b200 as X
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    if int(os.environ.get("RANK", "0")) != 0:
        return 0
    sizes = [int(v) for v in args.table_sizes.split(",")] if args.table_sizes else list(REF_TABLE_SIZES)
    thr = host_threads()
    have_ref = not args.no_cpu and oracle.ref_available()
    if have_ref:
        oracle.set_ref_threads(thr)
        table_reference_row("d", 256, args.seed)  # library, OpenBLAS threads and page-ins warm
    tdt = {"d": torch.float64, "s": torch.float32, "z": torch.complex128, "c": torch.complex64}
    rows, spent = [], 0.0
    for prec in args.table_prec:
        for n in sizes:
            S_h, P_h, al, ai, be = table_inputs(prec, n, args.seed)
            S, P = colmajor_cuda(S_h, torch), colmajor_cuda(P_h, torch)
            VL, VR = (torch.zeros(n, n, dtype=tdt[prec], device="cuda").t() for _ in range(2))
            for _ in range(max(args.warmup, 1)):
                X.tgevc3_dev("B", "A", S, P, al, be, alphai=ai, VL=VL, VR=VR)
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            for _ in range(args.steps):
                X.tgevc3_dev("B", "A", S, P, al, be, alphai=ai, VL=VL, VR=VR)
            e1.record()
            torch.cuda.synchronize()
            dev_ms = e0.elapsed_time(e1) / args.steps
            del S, P, VL, VR
            VLh, VRh = (np.zeros((n, n), dtype=S_h.dtype, order="F") for _ in range(2))
            X.tgevc3("B", "A", S_h, P_h, al, be, alphai=ai, VL=VLh, VR=VRh)
            host_s = float("inf")
            for _ in range(args.steps):
                t0 = time.perf_counter()
                X.tgevc3("B", "A", S_h, P_h, al, be, alphai=ai, VL=VLh, VR=VRh)
                host_s = min(host_s, time.perf_counter() - t0)
            row = {"prec": prec, "n": n, "device_ms": dev_ms, "host_ms": host_s * 1e3, "ref_cpu_ms": None}
            if have_ref and spent < args.ref_budget_s:
                t, VLr, VRr = table_reference_row(prec, n, args.seed)
                spent += t
                diff = max(float((np.abs(V - R).max(0) / np.maximum(np.abs(R).max(0), 1e-300)).max())
                           for V, R in ((VLh, VLr), (VRh, VRr)))
                row.update({"ref_cpu_ms": t * 1e3, "host_speedup_vs_ref": t / host_s,
                            "max_col_rel_diff_vs_ref": diff})
            rows.append(row)
            print(f"[table] {prec} n={n}: device {dev_ms:.2f} ms, host {host_s * 1e3:.2f} ms, "
                  f"ref {row['ref_cpu_ms']} ms", file=sys.stderr, flush=True)
    print(json.dumps({"mode": "reference_table", "side": "B", "howmny": "A", "sizes": sizes,
                      "precisions": args.table_prec, "ref_kind": "reference" if have_ref else None,
                      "ref_threads": thr, "steps": args.steps, "warmup": args.warmup,
                      "data": "triangular pencils with the upstream benchmark generators' distributions "
                              "(U(-1,1) entries, P diagonal p + sign(p)), seeded",
                      "rows": rows}))
    return 0


def main():
    args = parse()
    if args.profile_case:
        return profile_case(args)
    if args.reference_table:
        return reference_table(args)
    if args.gemm_only:
        return gemm_only(args)
    if args.impl == "reference":
        return reference_arm(args)
    import torch
    import xtgevc3_b200 as X

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    n = args.n
    # inputs: one pencil per rank
    seeds = rank_seeds(args.seed, args.batch_seed, rank)
    S_h, P_h, ar, ai, be = host_pencil(n, seeds["pencil"])
    S = colmajor_cuda(S_h, torch)
    P = colmajor_cuda(P_h, torch)
    Q = orthogonal(n, seeds["q"], torch)
    Z = orthogonal(n, seeds["z"], torch)
    VL = torch.empty_like(Q)
    VR = torch.empty_like(Z)
    data = (S, P, ar, ai, be, Q, Z, VL, VR)
    peak_fp64 = dgemm_peak(torch)
    peak_int8 = int8_peak(torch)
    peaks = {}
    pk = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(pk):
        peaks = json.load(open(pk))
    peak_bf16 = peaks.get("bf16_tflops", 1590.0)
    peak_hbm = peaks.get("hbm_gbs", 6650.0)

    s = max(1, min(6, args.slices))
    s8 = max(1, min(7, args.slices_i8))
    nm_crt = max(2, min(16, args.moduli))
    forms = {"plain": 0, "split": X.SPLIT | X.slices(s), "split_i8": X.SPLIT | X.SPLIT_INT8 | X.slices(s8),
             "split_crt": X.SPLIT | X.SPLIT_CRT | X.slices(nm_crt)}
    names = ["plain", "split", "split_i8", "split_crt"] if args.form == "all" else [args.form]
    # the upstream library on the same inputs, once (rank 0 at N = 1): the CPU baseline, and
    # the reference result every form is compared with elementwise
    cpu, ref = None, None
    if rank == 0 and world == 1 and not args.no_cpu:
        thr = host_threads()
        Qh, Zh = Q.cpu().numpy(), Z.cpu().numpy()  # column-major tensors -> Fortran arrays
        RL, RR, t_cpu, kind = cpu_full(S_h, P_h, ar, ai, be, Qh, Zh, thr)
        cpu = {"value": 2 * n / t_cpu, "unit": UNIT, "cores": thr, "kind": kind, "seconds": t_cpu,
               "sample": f"one full upstream dtgevc3 SIDE=B HOWMNY=B call on the same n={n} pencil, Q, Z "
                         f"({thr} threads)"}
        ref = (colmajor_cuda(RL, torch), colmajor_cuda(RR, torch))
        del RL, RR, Qh, Zh
    res = {nm: measure_form(nm, forms[nm], args, X, torch, data, dist, local, world, ref) for nm in names}
    ref = None
    ok = [nm for nm in names if res[nm]["resid"] <= 1e-12]
    head = min(ok or names, key=lambda nm: res[nm]["ms"])
    h = res[head]
    kernels = h["kernels"]

    # roofline of the dominant kernel class of the headline form
    dom = max(kernels, key=lambda k: kernels[k]["ms"])
    kd = kernels[dom]
    if kd["flops"] > 0 and head == "split" and dom.startswith("gemm"):
        # BF16 slice products actually executed: pairs x the FP64-equivalent flops
        pairs = s * (s + 1) // 2
        achieved = pairs * kd["flops"] / (kd["ms"] * 1e-3) / 1e12
        roof = {"bound": "tensor", "achieved": achieved, "peak": peak_bf16, "unit": "TFLOP/s",
                "frac": achieved / peak_bf16, "kernel": dom,
                "fp64_equivalent_tflops": kd["flops"] / (kd["ms"] * 1e-3) / 1e12,
                "peak_source": "MEASURED_PEAKS.json bf16_tflops (burst), BF16 slice products counted"}
    elif kd["flops"] > 0 and head == "split_i8" and dom.startswith("gemm"):
        # INT8 slice products executed; the dense INT8 rate is twice the BF16 one on B200
        pairs = s8 * (s8 + 1) // 2
        achieved = pairs * kd["flops"] / (kd["ms"] * 1e-3) / 1e12
        peak_i8 = 2.0 * peak_bf16
        roof = {"bound": "tensor", "achieved": achieved, "peak": peak_i8, "unit": "TOP/s",
                "frac": achieved / peak_i8, "kernel": dom,
                "fp64_equivalent_tflops": kd["flops"] / (kd["ms"] * 1e-3) / 1e12,
                "peak_source": "2 x MEASURED_PEAKS.json bf16_tflops (burst): INT8 dense rate, not measured; "
                               "INT8 slice products counted"}
    elif kd["flops"] > 0 and head == "split_crt" and dom == "split_gemm":
        # the residue GEMM kernel: one INT8 product per modulus
        achieved = nm_crt * kd["flops"] / (kd["ms"] * 1e-3) / 1e12
        peak_i8 = peak_int8 if peak_int8 else 2.0 * peak_bf16
        roof = {"bound": "tensor", "achieved": achieved, "peak": peak_i8, "unit": "TOP/s",
                "frac": achieved / peak_i8, "kernel": "gemm_crt_kernel (split_gemm class)",
                "fp64_equivalent_tflops": kd["flops"] / (kd["ms"] * 1e-3) / 1e12,
                "peak_source": ("cuBLASLt INT8 GEMM 8192^3 (torch._int_mm) burst measured in this run"
                                if peak_int8 else "2 x MEASURED_PEAKS.json bf16_tflops (INT8 not measured)") +
                               "; one INT8 product per modulus counted"}
    elif kd["flops"] > 0:
        achieved = kd["flops"] / (kd["ms"] * 1e-3) / 1e12
        roof = {"bound": "tensor", "achieved": achieved, "peak": peak_fp64, "unit": "TFLOP/s",
                "frac": achieved / peak_fp64, "kernel": dom,
                "peak_source": "cuBLAS DGEMM 8192^3 burst measured in this run (FP64; MEASURED_PEAKS.json "
                               "has no FP64 figure)"}
    else:
        achieved = kd["bytes"] / (kd["ms"] * 1e-3) / 1e9
        roof = {"bound": "hbm", "achieved": achieved, "peak": peak_hbm, "unit": "GB/s",
                "frac": achieved / peak_hbm, "kernel": dom, "peak_source": "MEASURED_PEAKS.json hbm_gbs"}
    tinfo = load_traffic()
    traffic = None
    key = f"{head}:{dom}"
    if tinfo and key in tinfo.get("bytes_per_flop", {}) and kd["flops"] > 0:
        traffic = tinfo["bytes_per_flop"][key] * kd["flops"] / kd["launches"]
        roof["traffic_note"] = tinfo.get("note", "")
    elif tinfo and key in tinfo.get("bytes_per_algorithmic_byte", {}) and kd["bytes"] > 0:
        traffic = tinfo["bytes_per_algorithmic_byte"][key] * kd["bytes"] / kd["launches"]
        roof["traffic_note"] = tinfo.get("note_bytes", "")
    roof["traffic"] = traffic
    roof["algorithmic_per_launch"] = (kd["flops"] if kd["flops"] > 0 else kd["bytes"]) / kd["launches"]
    for k in kernels.values():
        if k["flops"] > 0:
            k["tflops_fp64_equivalent"] = k["flops"] / (k["ms"] * 1e-3) / 1e12
        k["gbs"] = k["bytes"] / (k["ms"] * 1e-3) / 1e9 if k["ms"] > 0 else None

    # end-to-end through the host-pointer C ABI (pinned host buffers, copies timed)
    def pinned(shape):
        t = torch.empty((shape[1], shape[0]), dtype=torch.float64, pin_memory=True)
        return t.numpy().T  # Fortran-ordered view

    hS, hP, hQ, hZ, hVL, hVR = (pinned((n, n)) for _ in range(6))
    hS[...] = S_h
    hP[...] = P_h
    hQ[...] = Q.t().cpu().numpy().T
    hZ[...] = Z.t().cpu().numpy().T
    X.set_flags(h["flags"])
    e2e_t = []
    try:
        for it in range(args.warmup + args.steps):
            np.copyto(hVL, hQ)
            np.copyto(hVR, hZ)
            if dist:
                dist.barrier()
            t0 = time.perf_counter()
            _, _, m_, info_ = X.tgevc3("B", "B", hS, hP, ar, be, alphai=ai, VL=hVL, VR=hVR)
            t1 = time.perf_counter()
            assert info_ == 0
            if it >= args.warmup:
                e2e_t.append(t1 - t0)
    finally:
        X.set_flags(0)
    e2e_s = max_over_ranks(float(np.mean(e2e_t)), dist, torch)
    # bytes the host path moves: S and P as their upper trapezoid (rows <= col + 1) in the
    # library's pieces (512-column panels from the right alternating with 512-row strips from
    # the top, each the rest of the trapezoid), Q and Z whole in; VL and VR whole out
    def trapezoid_pieces(w=512):
        tot, cf, rt = 0, n, 0
        while cf >= 1 and rt <= cf:
            c0 = max(cf - w, 0)
            tot += (min(n, cf + 1) - rt) * (cf - c0)
            cf = c0
            if not (cf >= 1 and rt <= cf):
                break
            r1 = min(rt + w, n)
            tot += (r1 - rt) * (cf - max(rt - 1, 0))
            rt = r1
        return tot
    trap = trapezoid_pieces()
    e2e = {"value": world * 2 * n / e2e_s, "unit": UNIT, "h2d_bytes_per_step": (2 * trap + 2 * n * n) * 8,
           "d2h_bytes_per_step": 2 * n * n * 8, "ms_per_step": 1e3 * e2e_s,
           "path": f"xtgevc3_dtgevc3 (host pointers, pinned), {head} form, H2D/D2H inside the call (S, P "
                   f"in pieces while the solve runs, norms from host threads; Q, Z in row panels, each "
                   f"side's back-transform and download following them panel by panel)"}

    norm = measure_normalize(args, X, torch, data, peak_hbm) if rank == 0 else None
    batched = measure_batched(args, X, torch, dist, world) if args.batch_count > 0 else None
    adjoint = measure_adjoint(args, X, torch) if args.adjoint_n > 0 and rank == 0 else None
    zleg = measure_ztgevc3(args, X, torch) if args.z_n > 0 and rank == 0 else None
    trleg = measure_trevc3(args, X, torch) if args.trevc3_n > 0 and rank == 0 else None
    txleg = measure_tgexc(args, X, torch) if args.tgexc_n > 0 and rank == 0 else None
    dxleg = measure_tgexc(args, X, torch, real=True) if args.tgexc_n > 0 and rank == 0 else None
    bxleg = measure_tgexc_blocks(args, X, torch) if args.tgexc_n > 0 and rank == 0 else None
    qzleg = measure_gges(args, X, torch) if args.gges_n > 0 and rank == 0 else None
    difleg = measure_tgsna_dif(args, X, torch) if args.tgsna_n > 0 and rank == 0 else None
    senleg = measure_tgsen(args, X, torch) if args.tgsen_n > 0 and rank == 0 else None

    if rank == 0:
        form_desc = {"plain": "plain FP64 (DMMA)", "split": f"split precision, {s} BF16 slices (tcgen05)",
                     "split_i8": f"split precision, {s8} INT8 slices (tcgen05 kind::i8)",
                     "split_crt": f"split precision, {nm_crt} INT8 residues (CRT, tcgen05 kind::i8)"}
        forms_out = {nm: {"value": r["value"], "ms_per_step": r["ms"], "resid_max": r["resid"],
                          "meets_resid_bound": r["resid"] <= 1e-12, "max_rel_diff_vs_reference": r["err_vs_ref"],
                          "refined_columns_per_call": r["refined_columns"],
                          "kernels_ms_per_step": {k: v["ms_per_step"] for k, v in r["kernels"].items()}}
                     for nm, r in res.items()}
        if "plain" in res:
            for nm in forms_out:
                forms_out[nm]["speedup_vs_plain"] = res["plain"]["ms"] / res[nm]["ms"]
        # one compact line per form inside `config` (kept by record parsers that drop extra keys)
        forms_brief = {nm: {"ms": round(f["ms_per_step"], 3), "resid": f["resid_max"],
                            "err_vs_ref": f["max_rel_diff_vs_reference"], "refined": f["refined_columns_per_call"],
                            "x_plain": round(f.get("speedup_vs_plain", 0.0), 3)} for nm, f in forms_out.items()}
        line = {"metric": METRIC, "value": h["value"], "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": h["ms"], "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f64", "data": DATA,
                "config": {"workload": f"dtgevc3 SIDE=B HOWMNY=B n={n}", "n": n, "side": "B", "howmny": "B",
                           "form": form_desc[head], "pencils_per_gpu": 1,
                           "l2": "inputs larger than L2 (S,P,Q,Z = 2 GiB); no flush",
                           "parallelism": f"independent pencil per GPU x{world}",
                           "resid_max": h["resid"], "resid_bound": 1e-12,
                           "max_rel_diff_vs_reference": h["err_vs_ref"],
                           "reference_for_diff": "upstream dtgevc3 (oracle/_ref) on the same S, P, Q, Z; columns "
                                                 "compared after normalisation" if h["err_vs_ref"] is not None else None,
                           "forms": forms_brief,
                           "peaks_measured_here": {"fp64_dgemm_tflops": peak_fp64, "int8_imma_tops": peak_int8},
                           "normalize": None if norm is None else {
                               "ms": norm["ms_per_call"], "gbs": norm["gbs"], "frac_of_hbm": norm["frac_of_hbm"]},
                           "neighbours": neighbours_brief({"ztgexc": txleg, "dtgexc": dxleg, "dtgexc_blocks": bxleg,
                                                           "dtrevc3": trleg, "adjoint": adjoint, "dgges": qzleg,
                                                           "dtgsna_dif": difleg, "dtgsen": senleg}),
                           "batched": None if batched is None else {
                               "pencils_per_s": batched["value"], "speedup_vs_loop": batched["speedup_vs_loop"],
                               "d_ms": batched["d"]["ms"], "s_ms": batched["s"]["ms"],
                               "d_max_rel_diff_vs_loop": batched["d"]["max_rel_diff_vs_loop"]}},
                "forms": forms_out, "clocks": h["clocks"], "e2e": e2e, "gpu_launches": h["launches"],
                "roofline": roof, "kernels": kernels, "cpu_baseline": cpu, "normalize": norm, "batched": batched,
                "adjoint": adjoint, "ztgevc3": zleg, "dtrevc3": trleg, "ztgexc": txleg, "dtgexc": dxleg,
                "dtgexc_blocks": bxleg, "dgges": qzleg, "dtgsna_dif": difleg, "dtgsen": senleg}
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
