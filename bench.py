#!/usr/bin/env python
"""Zolo-PD time-to-solution benchmark on B200 (one JSON line on rank 0).

Workload (the reference's mixed-vs-FP64 headline case): Zolo-PD of an
n = 8192 square FP64 matrix A = U diag(s) V^T with Haar U, V and s log-uniform
in [1e-12, 1] (endpoints pinned, kappa = 1e12), Zolotarev degree r = 8.  One
step = the full solve a user runs: bounds (alpha = ||A||_F, beta from a QR
condition estimate) + PZOLOPD1 + H = sym(Q^T A), on a matrix resident in HBM.
Inputs are 512 MiB per matrix, far above the 126 MB L2, so no flush is needed.
The headline is the fast FP64 form; the reference's own steps on the GPU are
timed beside it (both must reach backward error and orthogonality <= 1e-13).

  python bench.py [--gpus N --steps K --warmup W] [--impl reference]

Multi-GPU: one process per GPU (torchrun), each rank solves its own matrix
(replicas; the path has no data exchange), timed on the device as the max over
ranks.  ``--impl reference`` times the CPU restatement of the reference
(``oracle/``, NumPy + OpenBLAS on all host cores) on a bounded sample.
"""
from __future__ import annotations

import argparse
import importlib.util
import json
import math
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))


def load_pkg():
    if "zolo_svd_b200" in sys.modules:
        return sys.modules["zolo_svd_b200"]
    pkg_dir = os.path.join(ROOT, "zolo-svd_b200")
    spec = importlib.util.spec_from_file_location("zolo_svd_b200", os.path.join(pkg_dir, "__init__.py"),
                                                  submodule_search_locations=[pkg_dir])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["zolo_svd_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


METRIC = "Zolo-PD/SVD n=8192 time-to-solution: mixed vs FP64 GPU at bwd err<=1e-13"
UNIT = "s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="zolo", choices=["zolo", "reference"])
    ap.add_argument("--n", type=int, default=8192)
    ap.add_argument("--rk", type=int, default=8)
    ap.add_argument("--kappa", type=float, default=1e12)
    ap.add_argument("--cpu-sample-n", type=int, default=1536)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    return ap.parse_args()


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.dev = device_index
        self.samples = []
        self.proc = None
        self.th = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.dev}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
            return
        self.th = threading.Thread(target=self._read, daemon=True)
        self.th.start()

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                self.samples.append(parts)

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        if self.th:
            self.th.join(timeout=2)
        sm = [float(p[1]) for p in self.samples if p[1].replace(".", "").isdigit()]
        mx = [float(p[2]) for p in self.samples if p[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for p in self.samples:
            for i, nm in enumerate(names):
                if p[5 + i].lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(self.samples)}


# ---------------------------------------------------------------------------
# synthetic input (seeded): A = U diag(s) V^T
# ---------------------------------------------------------------------------
def make_input_gpu(torch, n: int, kappa: float, seed: int):
    g = torch.Generator(device="cuda")
    g.manual_seed(seed)
    def haar():
        z = torch.randn(n, n, dtype=torch.float64, device="cuda", generator=g)
        q, r = torch.linalg.qr(z)
        return q * torch.sign(torch.diagonal(r))[None, :]
    u = haar()
    v = haar()
    e = torch.rand(n, dtype=torch.float64, device="cuda", generator=g) * (-math.log10(kappa))
    e[0] = 0.0
    e[-1] = -math.log10(kappa)
    s = torch.sort(10.0 ** e, descending=True).values
    a_rowmajor = (u * s[None, :]) @ v.T          # A (row-major view)
    del u, v
    # column-major storage: tensor T with T[j, i] = A[i, j]
    return a_rowmajor.T.contiguous(), s


def fp64_peak_tflops(torch) -> float:
    """cuBLAS DGEMM 8192^3 throughput measured in this run (the FP64 tensor roofline)."""
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device="cuda")
    b = torch.randn(n, n, dtype=torch.float64, device="cuda")
    c = torch.empty_like(a)
    for _ in range(2):
        torch.matmul(a, b, out=c)
    torch.cuda.synchronize()
    best = 0.0
    for _ in range(5):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b, out=c)
        e1.record()
        torch.cuda.synchronize()
        best = max(best, 2.0 * n ** 3 / (e0.elapsed_time(e1) * 1e-3) / 1e12)
    del a, b, c
    torch.cuda.empty_cache()
    return best


# ---------------------------------------------------------------------------
# CPU baseline: the oracle restatement on a bounded sample
# ---------------------------------------------------------------------------
def cpu_baseline(n_full: int, n_s: int, rk: int, kappa: float) -> dict:
    sys.path.insert(0, ROOT)
    from oracle import zolo_oracle as zo  # the CPU restatement, used only as the baseline
    rng = np.random.default_rng(1003)
    e = rng.uniform(-math.log10(kappa), 0.0, n_s)
    e[0], e[-1] = 0.0, -math.log10(kappa)
    s = np.sort(10.0 ** e)[::-1]
    a, _, _ = zo.make_matrix(n_s, s, 1003)
    t0 = time.perf_counter()
    al, be, _ = zo.bounds_zolodrv(a)
    q, st = zo.pzolopd1("N", rk, a, al, be)
    h = zo.polar_h(q, a)
    t = time.perf_counter() - t0
    scale = (n_full / n_s) ** 3
    return {"value": t * scale, "unit": UNIT, "cores": os.cpu_count(), "kind": "port",
            "sample": f"oracle pzolopd1 (NumPy/OpenBLAS, {os.cpu_count()} threads, 1x1 grid, no MPI) on "
                      f"n={n_s}, kappa={kappa:g}, r={rk}: {t:.2f} s, scaled by (n/{n_s})^3 = {scale:.0f}",
            "sample_seconds": t, "iterations": st.iterations}


def max_over_ranks(dist, value: float, device: str) -> float:
    """The slowest rank's time: every rank contributes its own device time (the bench's
    N-GPU numbers are the max over ranks, never a wall clock)."""
    if dist is None:
        return value
    import torch
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    times = []
    for i in range(args.warmup + args.steps):
        cb = cpu_baseline(args.n, args.cpu_sample_n, args.rk, args.kappa)
        if i >= args.warmup:
            times.append(cb["value"])
    v = float(np.mean(times))
    line = {"metric": METRIC, "value": v, "unit": UNIT, "impl": "reference", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": v * 1e3, "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"Zolo-PD r={args.rk}, n={args.n}, kappa={args.kappa:g}, FP64",
                       "n": args.n, "rk": args.rk, "kappa": args.kappa},
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": cb["cores"], "kind": "port",
                             "sample": cb["sample"]},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------
# GPU arm
# ---------------------------------------------------------------------------
# The two FP64 forms measured.  "fast" is the headline: bounds, Zolo-PD and H in
# one call (zolo_polar_dev, the QR of A/alpha reused by the first iteration), one
# QR of X shared by the r Zolotarev terms in the QR iterations, Cholesky iterations
# through S = sum_j w_j (X^T X + c_j I)^{-1} (explicit triangular inverses) and one
# Z = X S, beta = 1/||R^{-1}||_F (a lower bound on sigma_min up to sqrt(n) tighter than
# the reference driver's, which keeps CON = 1/beta where the Zolotarev coefficients are
# accurate), FP64 Newton-Schulz steps once ||X^T X - I||_F/sqrt(n) <= 0.1, and per
# iteration the Zolotarev term count (<= r) of the cheapest plan to convergence on one GPU.
# "reference_steps" runs the reference's own steps on the GPU as two calls (bounds, then PZOLOPD1): one
# structured QR of [X; sqrt(c_j) I] per term and the reference's stopping rule
# (pzolopd1.f90:381-397).
FORMS = {
    "fast": {"shared_qr": 1, "ns_finish": 1, "chol_inverse": 1, "beta_frob": 1, "term_plan": 1, "one_call": True},
    "reference_steps": {"shared_qr": 0, "ns_finish": 0, "chol_inverse": 0, "beta_frob": 0, "term_plan": 0,
                        "one_call": False},
}

# DRAM bytes (read + write) of one launch of the dominant kernel (DMMA GEMM, 64x128 tiles)
# from an ncu capture of a C = A B launch with M = N = K = 4096: 1408.2 MB + 124.7 MB.
DGEMM_TRAFFIC_BYTES = 1.5329e9
DGEMM_TRAFFIC_LAUNCH = "one 4096^3 C = A B launch (ncu capture; algorithmic A+B+C = 0.40 GB, L2 hit 84 %)"


def accuracy(torch, dA, dQ, dH, s_true=None) -> dict:
    n = dA.shape[0]
    A, Q, H = dA.T, dQ.T, dH.T  # row-major views of the column-major arrays
    nA = torch.linalg.norm(A)
    out = {"backward_error": float(torch.linalg.norm(A - Q @ H) / nA)}
    eye = torch.eye(n, dtype=torch.float64, device="cuda")
    out["orthogonality"] = float(torch.linalg.norm(Q.T @ Q - eye) / math.sqrt(n))
    del eye
    if s_true is not None:
        ev = torch.linalg.eigvalsh(0.5 * (H + H.T))
        out["sv_err_rel_smax"] = float(torch.max(torch.abs(torch.sort(ev, descending=True).values - s_true))
                                       / s_true[0])
    return out


def run_gpu(args):
    import torch
    zb = load_pkg()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    n, rk = args.n, args.rk
    stream = torch.cuda.current_stream()
    h = zb.Handle(local)
    h.set_stream(stream.cuda_stream)

    peak = fp64_peak_tflops(torch)
    dA, s_true = make_input_gpu(torch, n, args.kappa, 1003 + rank)
    dQ = torch.empty_like(dA)
    dH = torch.empty((n, n), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()

    form = {"name": "fast"}

    def set_form(name):
        form["name"] = name
        h.set_option(zb.OPT_SHARED_QR, FORMS[name]["shared_qr"])
        h.set_option(zb.OPT_NS_FINISH, FORMS[name]["ns_finish"])
        h.set_option(zb.OPT_CHOL_INVERSE, FORMS[name]["chol_inverse"])
        h.set_option(zb.OPT_BETA_FROB, FORMS[name]["beta_frob"])
        h.set_option(zb.OPT_TERM_PLAN, FORMS[name]["term_plan"])

    def step(src):
        if FORMS[form["name"]]["one_call"]:
            # bounds + Zolo-PD + H in one call: the QR of A/alpha is reused by the first iteration
            zb.polar_dev(h, rk, n, n, src.data_ptr(), n, dQ.data_ptr(), n, dH.data_ptr(), n)
            return h.stats()
        al, be, info = zb.bounds_dev(h, n, n, src.data_ptr(), n, mode=1)
        st_b = h.stats()
        zb.pzolopd1_dev(h, "N", rk, n, n, al, be, src.data_ptr(), n, dQ.data_ptr(), n, dH.data_ptr(), n)
        st = h.stats()
        st["launches"] += st_b["launches"]
        st["flops"] += st_b["flops"]
        st["flops_executed"] += st_b["flops_executed"]
        return st

    def timed(steps):
        """steps solves between a barrier + synchronize on both sides; device ms per step (max over ranks)."""
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        launches, last = 0, None
        e0.record(stream)
        for _ in range(steps):
            last = step(dA)
            launches += last["launches"]
        e1.record(stream)
        torch.cuda.synchronize()
        t = max_over_ranks(dist, e0.elapsed_time(e1) / steps, "cuda")
        return t, launches, last

    # ---- headline: the fast form ----
    set_form("fast")
    for _ in range(args.warmup):
        step(dA)
    clocks = ClockSampler(local)
    clocks.start()
    t_ms, launches, st_fast = timed(args.steps)
    ck = clocks.stop()
    acc_fast = accuracy(torch, dA, dQ, dH, s_true)

    # per-kernel-class device time of one more solve (CUDA events around every launch, outside the timed region)
    h.profile(True)
    h.profile_read(reset=True)
    step(dA)
    torch.cuda.synchronize()
    prof = h.profile_read(reset=True)
    h.profile(False)

    # ---- the reference's steps on the GPU (the plain FP64 form) ----
    set_form("reference_steps")
    step(dA)  # warm-up: its per-term stacks need their own workspace
    ref_steps = max(1, min(args.steps, 2))
    t_ref_ms, _, st_ref = timed(ref_steps)
    acc_ref = accuracy(torch, dA, dQ, dH)
    set_form("fast")

    # ---- e2e through the public API with host buffers: pinned A -> device, solve, Q and H back ----
    hA = torch.empty((n, n), dtype=torch.float64, pin_memory=True)
    hA.copy_(dA)
    hQ = torch.empty_like(hA, pin_memory=True)
    hH = torch.empty_like(hA, pin_memory=True)
    dA2 = torch.empty_like(dA)

    def e2e_step():
        dA2.copy_(hA, non_blocking=True)
        step(dA2)
        hQ.copy_(dQ, non_blocking=True)
        hH.copy_(dH, non_blocking=True)

    e2e_step()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    f0 = torch.cuda.Event(enable_timing=True)
    f1 = torch.cuda.Event(enable_timing=True)
    e2e_steps = max(1, min(args.steps, 2))
    f0.record(stream)
    for _ in range(e2e_steps):
        e2e_step()
    f1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = max_over_ranks(dist, f0.elapsed_time(f1) / e2e_steps, "cuda")

    gk = [k for k in prof if k.startswith("dgemm")]
    g = {"ms": sum(prof[k]["ms"] for k in gk), "flops": sum(prof[k]["flops"] for k in gk),
         "launches": sum(prof[k]["launches"] for k in gk)}
    prof_ms = sum(v["ms"] for v in prof.values())
    achieved = g["flops"] / (g["ms"] * 1e-3) / 1e12 if g["ms"] > 0 else 0.0
    per_class = {k: {"launches": v["launches"], "ms": round(v["ms"], 3),
                     "tflops": round(v["flops"] / (v["ms"] * 1e-3) / 1e12, 3) if v["ms"] > 0 else None}
                 for k, v in prof.items()}
    out = None
    if rank == 0:
        out = {
            "metric": METRIC, "value": t_ms / 1e3, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t_ms, "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"Zolo-PD r={rk} (bounds + PZOLOPD1 + H), n={n}, kappa={args.kappa:g}, "
                                   f"FP64 on DMMA, fast form (one call, shared QR of X, explicit-inverse Cholesky "
                                   f"iterations, Frobenius beta bound, Newton-Schulz finish, planned term counts)",
                       "n": n, "rk": rk, "kappa": args.kappa, "form": "fast", "precision": "fp64",
                       "parallelism": f"replicas x{world}",
                       "l2": "inputs 512 MiB per matrix > 126 MB L2 (no flush needed)"},
            "accuracy": dict(acc_fast, iterations=st_fast["iterations"], ns_steps=st_fast["ns_steps"],
                             branches=st_fast["branches"], terms=st_fast["terms"]),
            "phases_ms": {"bounds": st_fast["ms_bounds"], "iterations": st_fast["ms_step"],
                          "finish": st_fast["ms_finish"], "h_and_q": st_fast["ms_h"]},
            "forms": {
                "fast": {"s": t_ms / 1e3, "backward_error": acc_fast["backward_error"],
                         "orthogonality": acc_fast["orthogonality"], "branches": st_fast["branches"]},
                "reference_steps": {"s": t_ref_ms / 1e3, "steps": ref_steps,
                                    "backward_error": acc_ref["backward_error"],
                                    "orthogonality": acc_ref["orthogonality"], "branches": st_ref["branches"]},
                "speedup_fast_vs_reference_steps": t_ref_ms / t_ms,
                "mixed_precision": "not built: a low-precision iteration moves the polar factor by "
                                   "eps_low * spread of the singular values, above 1e-13",
            },
            "tflops_canonical": st_fast["flops"] / (t_ms * 1e-3) / 1e12,
            "tflops_executed": st_fast["flops_executed"] / (t_ms * 1e-3) / 1e12,
            "roofline": {"bound": "tensor", "kernel": "dgemm_kernel (FP64 DMMA mma.sync m16n8k8, all shapes)",
                         "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                         "frac": achieved / peak if peak else None,
                         "peak_source": "cuBLAS DGEMM 8192^3 measured in this run (FP64 tensor pipe)",
                         "traffic": DGEMM_TRAFFIC_BYTES, "traffic_launch": DGEMM_TRAFFIC_LAUNCH,
                         "share_of_step": g["ms"] / prof_ms if prof_ms else None,
                         "launches_per_step": g["launches"]},
            "kernel_classes": per_class,
            "e2e": {"value": e2e_ms / 1e3, "unit": UNIT, "h2d_bytes_per_step": 8 * n * n,
                    "d2h_bytes_per_step": 16 * n * n},
            "gpu_launches": int(launches),
            "clocks": ck,
        }
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    h.close()
    if rank == 0:
        if not args.no_cpu_baseline and world == 1:
            try:
                out["cpu_baseline"] = {k: v for k, v in cpu_baseline(n, args.cpu_sample_n, rk, args.kappa).items()
                                       if k in ("value", "unit", "cores", "kind", "sample")}
            except Exception as exc:  # the baseline must not hide the GPU line
                out["cpu_baseline"] = {"value": None, "error": str(exc)[:200]}
        print(json.dumps(out), flush=True)
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    return run_gpu(args)


if __name__ == "__main__":
    sys.exit(main())
