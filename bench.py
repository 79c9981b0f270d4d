#!/usr/bin/env python
"""Zolo-PD time-to-solution benchmark on B200 (one JSON line on rank 0).

Workload (the reference's mixed-vs-FP64 headline case): Zolo-PD of an
n = 8192 square FP64 matrix A = U diag(s) V^T with Haar U, V and s log-uniform
in [1e-12, 1] (endpoints pinned, kappa = 1e12), Zolotarev degree r = 8,
generated by NumPy's PCG64 (seed 1003) so that the CPU arm solves the same
matrix.  One step = the full solve a user runs: bounds (alpha = ||A||_F, beta
from a QR condition estimate) + PZOLOPD1 + H = sym(Q^T A), on a matrix resident
in HBM.  Inputs are 512 MiB per matrix, far above the 126 MB L2, so no flush is
needed.  The headline is the mixed form (the Cholesky iterations, Newton-Schulz
finish and Q/H products on the INT8 tensor cores with FP64 emulated from 8 digit
planes); the plain FP64 form and the reference's own steps on the GPU are timed
beside it (each must reach backward error and orthogonality <= 1e-13).

  python bench.py [--gpus N --steps K --warmup W] [--impl reference]

Multi-GPU: one process per GPU (torchrun), each rank solves its own matrix
(replicas; the path has no data exchange), timed on the device as the max over
ranks.  ``--impl reference`` times the CPU restatement of the reference
(``oracle/``, NumPy + OpenBLAS on all host cores) on one full solve of the same
matrix.
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
    ap.add_argument("--n", "--matrix-n", dest="n", type=int, default=8192)
    ap.add_argument("--rk", type=int, default=8)
    ap.add_argument("--kappa", type=float, default=1e12)
    ap.add_argument("--no-extras", action="store_true", help="skip the batch and Zolo-SVD configurations")
    ap.add_argument("--ref-timeout", type=float, default=1650.0,
                    help="seconds allowed for the reference arm's one full CPU solve")
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
def make_input(n: int, kappa: float, seed: int):
    """A = (U s) V^T in FP64 (column-major), Haar U and V from the QR of N(0,1) matrices with
    diag(R) > 0, s = 10^U[-log10 kappa, 0] with s_1 = 1, s_n = 1/kappa, sorted descending.
    All draws from one NumPy PCG64 stream: s first, then U, then V."""
    rng = np.random.default_rng(seed)
    e = rng.uniform(-math.log10(kappa), 0.0, n)
    e[0], e[-1] = 0.0, -math.log10(kappa)
    s = np.sort(10.0 ** e)[::-1].copy()

    def haar():
        q, r = np.linalg.qr(rng.standard_normal((n, n)))
        return q * np.sign(np.diag(r))[None, :]
    u = haar()
    v = haar()
    a = np.asfortranarray((u * s[None, :]) @ v.T)
    return a, s


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


def int8_library_tops(torch) -> float:
    """cuBLASLt INT8 GEMM (torch._int_mm, int32 out) 8192^3 throughput measured in this run: a
    library INT8 rate beside the tensor peak the INT8-emulated GEMM is compared with."""
    n = 8192
    a = torch.randint(-127, 128, (n, n), dtype=torch.int8, device="cuda")
    b = torch.randint(-127, 128, (n, n), dtype=torch.int8, device="cuda").t().contiguous().t()
    for _ in range(2):
        torch._int_mm(a, b)
    torch.cuda.synchronize()
    best = 0.0
    for _ in range(5):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        torch._int_mm(a, b)
        e1.record()
        torch.cuda.synchronize()
        best = max(best, 2.0 * n ** 3 / (e0.elapsed_time(e1) * 1e-3) / 1e12)
    del a, b
    torch.cuda.empty_cache()
    return best


# ---------------------------------------------------------------------------
# CPU reference arm: the oracle restatement, one full solve of the same matrix
# ---------------------------------------------------------------------------
def _oracle_solve(n: int, rk: int, kappa: float, seed: int, groups: int, conn) -> None:
    """Child process: generate the matrix, run bounds + PZOLOPD1 + H of the oracle, send the
    timings (the generation is outside the timed region).  With groups > 1 the r terms of each
    iteration run on `groups` worker processes of cores/groups BLAS threads each, as the
    reference runs them on r MPI process groups (pzolopd1.f90:298-374)."""
    sys.path.insert(0, ROOT)
    from oracle import zolo_oracle as zo  # the CPU restatement, used only as the baseline
    a, _ = make_input(n, kappa, seed)
    pool = None
    term_map = None
    if groups > 1:
        import multiprocessing as mp
        threads = max(1, (os.cpu_count() or 1) // groups)
        saved = {k: os.environ.get(k) for k in ("OPENBLAS_NUM_THREADS", "OMP_NUM_THREADS")}
        os.environ["OPENBLAS_NUM_THREADS"] = os.environ["OMP_NUM_THREADS"] = str(threads)
        pool = mp.get_context("spawn").Pool(groups)
        for k, v in saved.items():
            if v is None:
                os.environ.pop(k, None)
            else:
                os.environ[k] = v
        pool.starmap(zo.hfunc, [(0.5,)] * groups)  # workers started and the oracle imported
        term_map = lambda fn, args: pool.starmap(fn, args)
    t0 = time.perf_counter()
    al, be, _ = zo.bounds_zolodrv(a)
    q, st = zo.pzolopd1("N", rk, a, al, be, term_map=term_map)
    h = zo.polar_h(q, a)
    t = time.perf_counter() - t0
    if pool:
        pool.close()
        pool.join()
    conn.send({"seconds": t, "iterations": st.iterations, "branches": st.branches,
               "backward_error": zo.backward_error(a, q, h), "orthogonality": zo.orthogonality(q)})
    conn.close()


def oracle_full_solve(n: int, rk: int, kappa: float, seed: int, timeout: float, groups: int = 1) -> dict:
    """One timed oracle solve in a spawned process (killed after `timeout` s)."""
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    parent, child = ctx.Pipe(duplex=False)
    p = ctx.Process(target=_oracle_solve, args=(n, rk, kappa, seed, groups, child))
    p.start()
    child.close()
    out = None
    if parent.poll(timeout):
        out = parent.recv()
    p.join(timeout=5)
    if p.is_alive():
        p.kill()
        p.join()
    return out


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    cores = os.cpu_count() or 1
    groups = max(1, min(args.rk, cores // 2))
    res = oracle_full_solve(args.n, args.rk, args.kappa, 1003, args.ref_timeout, groups)
    sample = (f"oracle bounds + pzolopd1 + H (NumPy/OpenBLAS) on the bench's own n={args.n}, "
              f"kappa={args.kappa:g} matrix (PCG64 seed 1003): one full solve, no scaling; the r terms of each "
              f"iteration on {groups} worker processes x {max(1, cores // groups)} BLAS threads (the reference's "
              f"r process groups), bounds and H on {cores} threads; {cores} host cores")
    v = res["seconds"] if res else None
    line = {"metric": METRIC, "value": v, "unit": UNIT, "impl": "reference", "n_gpus": args.gpus,
            "steps": 1 if res else 0, "steps_requested": args.steps, "warmup": 0,
            "ms_per_step": v * 1e3 if v else None, "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"Zolo-PD r={args.rk} (bounds + PZOLOPD1 + H), n={args.n}, "
                                   f"kappa={args.kappa:g}, FP64, the reference's steps on the CPU",
                       "n": args.n, "rk": args.rk, "kappa": args.kappa, "seed": 1003},
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": cores, "kind": "port", "sample": sample},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    if res:
        line["accuracy"] = {k: res[k] for k in ("backward_error", "orthogonality", "iterations", "branches")}
    else:
        line["unavailable"] = f"the oracle's full solve did not finish within {args.ref_timeout:.0f} s"
    print(json.dumps(line), flush=True)
    return 0


def max_over_ranks(dist, value: float, device: str) -> float:
    """The slowest rank's time: every rank contributes its own device time (the bench's
    N-GPU numbers are the max over ranks, never a wall clock)."""
    if dist is None:
        return value
    import torch
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


# ---------------------------------------------------------------------------
# GPU arm
# ---------------------------------------------------------------------------
# The forms measured.  "fp64" is the plain FP64 GPU form: bounds, Zolo-PD and H in one call
# (zolo_polar_dev, the QR of A/alpha reused by the first iteration), one QR of X shared by
# the r Zolotarev terms in the QR iterations, Cholesky iterations through
# S = sum_j w_j (X^T X + c_j I)^{-1} (explicit triangular inverses) and one Z = X S,
# beta = 1/||R^{-1}||_F, FP64 Newton-Schulz steps once ||X^T X - I||_F/sqrt(n) <= 0.1, and per
# iteration the Zolotarev term count (<= r) of the cheapest plan to convergence on one GPU.
# "mixed" (the headline) is the same with the large products of the Cholesky iterations, the
# Newton-Schulz finish and Q, H on the INT8 tensor cores (FP64 emulated from 8 digit planes,
# ozaki.cu); the bounds and the QR iterations stay on the FP64 tensor path.
# "reference_steps" runs the reference's own steps on the GPU as two calls (bounds, then
# PZOLOPD1): one structured QR of [X; sqrt(c_j) I] per term and the reference's stopping rule
# (pzolopd1.f90:381-397).
FORMS = {
    "mixed": {"shared_qr": 1, "ns_finish": 1, "chol_inverse": 1, "beta_frob": 1, "term_plan": 1, "mixed": 1,
              "one_call": True},
    "fp64": {"shared_qr": 1, "ns_finish": 1, "chol_inverse": 1, "beta_frob": 1, "term_plan": 1, "mixed": 0,
             "one_call": True},
    "reference_steps": {"shared_qr": 0, "ns_finish": 0, "chol_inverse": 0, "beta_frob": 0, "term_plan": 0,
                        "mixed": 0, "one_call": False},
}
ACCURACY_TARGET = 1e-13

# DRAM bytes (read + write) of one launch of the dominant kernel (DMMA GEMM, 64x128 tiles)
# from an ncu capture of a C = A B launch with M = N = K = 4096: 1408.2 MB + 124.7 MB.
DGEMM_TRAFFIC_BYTES = 1.5329e9
DGEMM_TRAFFIC_LAUNCH = "one 4096^3 C = A B launch (ncu capture; algorithmic A+B+C = 0.40 GB, L2 hit 84 %)"
OZ_SLICES = 8
OZ_PRODUCTS = OZ_SLICES * (OZ_SLICES + 1) // 2  # INT8 digit products per emulated FP64 product


def measured_peaks() -> dict:
    """MEASURED_PEAKS.json (driver-written) if present: HBM GB/s and dense bf16 TFLOP/s."""
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f)
    except Exception:
        return {}


def int8_peak_tops() -> tuple[float, str]:
    """Dense INT8 tensor peak: the INT8 rate of tcgen05 is twice its BF16 rate, so twice the
    measured dense bf16 throughput (burst); the recipe's fallback 1.59 PFLOP/s bf16 otherwise."""
    pk = measured_peaks()
    for key in ("bf16_tflops", "bf16_dense_tflops"):
        if isinstance(pk.get(key), (int, float)) and pk[key] > 0:
            return 2.0 * pk[key], f"2 x measured dense bf16 ({pk[key]:.0f} TFLOP/s, MEASURED_PEAKS.json)"
    return 2.0 * 1590.0, "2 x fallback dense bf16 (1590 TFLOP/s)"


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


def haar_np(rng, m: int, n: int):
    q, r = np.linalg.qr(rng.standard_normal((m, n)))
    return q * np.sign(np.diag(r))[None, :]


def bench_batch_c4(torch, zb, h, reps: int = 3) -> dict:
    """Configuration 4: 512 matrices, n log-uniform in [64, 1024], m = n (1 + U[0,1]), kappa
    log-uniform in [1e2, 1e14], s geometric; PCG64 seed 1004 (sizes, kappa) and 1004 + i
    (member i's Haar factors).  One zolo_qdwh_batch_dev call per timed repetition (cached bucket
    graphs replayed; the synchronized loop, the first eager call and the capturing call timed
    beside it); the worst member's backward error and orthogonality over 10 n eps."""
    rng = np.random.default_rng(1004)
    mats = []
    for i in range(512):
        n = int(round(math.exp(rng.uniform(math.log(64), math.log(1024)))))
        m = int(round(n * (1 + rng.uniform(0, 1))))
        kappa = 10 ** rng.uniform(2, 14)
        s = np.geomspace(1.0, 1.0 / kappa, n)
        r2 = np.random.default_rng(1004 + i)
        a = np.asfortranarray((haar_np(r2, m, n) * s[None, :]) @ haar_np(r2, n, n).T)
        mats.append((a, s))
    da = [torch.from_numpy(a.T.copy()).to("cuda") for a, _ in mats]
    dq = [torch.empty_like(x) for x in da]
    dh = [torch.empty((a.shape[1], a.shape[1]), dtype=torch.float64, device="cuda") for a, _ in mats]
    members = [(a.shape[0], a.shape[1], x.data_ptr(), a.shape[0], q.data_ptr(), a.shape[0], hh.data_ptr(),
                a.shape[1]) for (a, _), x, q, hh in zip(mats, da, dq, dh)]
    stream = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def timed(calls):
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(calls):
            r = zb.qdwh_batch_dev(h, members)
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / calls, r
    # the host-synchronized loop (ZOLO_OPT_BATCH_GRAPH = 0), after a call that sizes the workspace
    h.set_option(zb.OPT_BATCH_GRAPH, 0)
    zb.qdwh_batch_dev(h, members)
    ms_sync, _ = timed(1)
    # the scheduled form: the first call of each bucket shape issues its launches eagerly, the
    # second captures them as one graph per bucket, later calls replay the graphs (timed)
    h.set_option(zb.OPT_BATCH_GRAPH, 1)
    ms_first, _ = timed(1)
    ms_capture, _ = timed(1)
    ms, (info, its) = timed(reps)
    gst = zb.batch_stats(h)
    st = h.stats()
    worst_b = worst_o = worst_s = 0.0
    for (a, s), x, q, hh in zip(mats, da, dq, dh):
        n = a.shape[1]
        A, Q, H = x.T, q.T, hh.T
        be = float(torch.linalg.norm(A - Q @ H) / torch.linalg.norm(A))
        orth = float(torch.linalg.norm(Q.T @ Q - torch.eye(n, dtype=torch.float64, device="cuda")) / math.sqrt(n))
        ev = torch.sort(torch.linalg.eigvalsh(0.5 * (H + H.T)), descending=True).values
        sv = float(torch.max(torch.abs(ev - torch.from_numpy(s).to("cuda"))))
        tol = 10 * n * 2.220446049250313e-16
        worst_b, worst_o, worst_s = max(worst_b, be / tol), max(worst_o, orth / tol), max(worst_s, sv)
    out = {"workload": "512 matrices, n in [64, 1024] log-uniform, m in [n, 2n], kappa in [1e2, 1e14], QDWH-PD "
                       "batched (zolo_qdwh_batch_dev)", "ms": ms, "matrices_per_s": 512 / (ms * 1e-3), "reps": reps,
           "info_nonzero": int(sum(1 for v in info if v)), "max_iterations": int(max(its)),
           "tflops_useful": st["flops"] / (ms * 1e-3) / 1e12,
           "tflops_executed": st["flops_executed"] / (ms * 1e-3) / 1e12,
           "worst_backward_error_over_10neps": worst_b, "worst_orthogonality_over_10neps": worst_o,
           "worst_sv_err_rel_smax": worst_s,
           "launch": "one CUDA graph per bucket (iterations, H, unpacking) replayed on eight worker streams; "
                     "bounds eager", "buckets": gst["buckets"], "graph_replays": gst["graph_replays"],
           "ms_first_call_eager": ms_first, "ms_capture_call": ms_capture, "ms_synchronized_loop": ms_sync}
    del da, dq, dh
    torch.cuda.empty_cache()
    return out


def bench_svd_c5(torch, zb, h) -> dict:
    """Configuration 5: Zolo-SVD of a 16384 x 8192 matrix, kappa = 1e10: 70 % of s geometric in
    [1e-10, 1], 20 % exactly 1, 10 % in clusters of relative gap 1e-9; Gaussians from PCG64 seed
    1005, their QR (Haar factors) on the GPU.  After one untimed call (the workspace), one timed
    zolo_svd_dev call per form on the same matrix
    (Zolo-PD r = 8, then the spectral divide-and-conquer eigensolver on H): the FP64 fast form,
    and the mixed form beside it (the Cholesky iterations, finish and Q/H products of both the
    Zolo-PD and the eigensolver's QDWH solves on the INT8-emulated GEMM)."""
    m, n = 16384, 8192
    rng = np.random.default_rng(1005)
    n70, n20 = int(0.7 * n), int(0.2 * n)
    n10 = n - n70 - n20
    base = np.geomspace(1e-1, 1e-9, n10 // 8 + 1)
    clus = (base[:, None] * (1 + 1e-9 * np.arange(8))[None, :]).reshape(-1)[:n10]
    s = np.sort(np.concatenate([np.geomspace(1.0, 1e-10, n70), np.ones(n20), clus]))[::-1].copy()

    def haar_gpu(r, c):
        g = torch.from_numpy(rng.standard_normal((c, r)).T.copy()).to("cuda")
        q, rr = torch.linalg.qr(g)
        return q * torch.sign(torch.diagonal(rr))[None, :]
    u = haar_gpu(m, n)
    v = haar_gpu(n, n)
    st = torch.from_numpy(s).to("cuda")
    a = (u * st[None, :]) @ v.T
    del u, v
    da = a.T.contiguous()
    du = torch.empty_like(da)
    ds = torch.empty(n, dtype=torch.float64, device="cuda")
    dv = torch.empty((n, n), dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream()
    eye = torch.eye(n, dtype=torch.float64, device="cuda")
    out = {"workload": "Zolo-SVD 16384 x 8192, kappa 1e10, 20 % sigma = 1, clusters of gap 1e-9 (zolo_svd_dev, "
                       "Zolo-PD r = 8 + spectral divide-and-conquer), FP64 fast form and mixed form"}
    saved = h.get_option(zb.OPT_MIXED)
    # an untimed call first: the first solve of these shapes allocates the workspace
    h.set_option(zb.OPT_MIXED, 0)
    zb.svd_dev(h, m, n, da.data_ptr(), m, du.data_ptr(), m, ds.data_ptr(), dv.data_ptr(), n, algo=1, rk=8)
    for form, mixed in (("fp64", 0), ("mixed", 1)):
        h.set_option(zb.OPT_MIXED, mixed)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        zb.svd_dev(h, m, n, da.data_ptr(), m, du.data_ptr(), m, ds.data_ptr(), dv.data_ptr(), n, algo=1, rk=8)
        e1.record(stream)
        torch.cuda.synchronize()
        U, V = du.T, dv.T
        out[form] = {"s": e0.elapsed_time(e1) / 1e3,
                     "residual": float(torch.linalg.norm(a - (U * ds[None, :]) @ V.T) / torch.linalg.norm(a)),
                     "sv_err_rel_smax": float(torch.max(torch.abs(torch.sort(ds, descending=True).values - st))
                                              / st[0]),
                     "orth_u": float(torch.linalg.norm(U.T @ U - eye) / math.sqrt(n)),
                     "orth_v": float(torch.linalg.norm(V.T @ V - eye) / math.sqrt(n))}
    h.set_option(zb.OPT_MIXED, saved)
    out["speedup_mixed_vs_fp64"] = out["fp64"]["s"] / out["mixed"]["s"]
    del a, da, du, dv, eye
    torch.cuda.empty_cache()
    return out


def run_gpu(args):
    import torch
    # options of the library's default handle (the one the reference-named host-array entry
    # points use) come from the environment: the e2e leg calls pzolopd1_ like an unchanged
    # Fortran driver with the fast and mixed options selected this way
    os.environ["ZOLO_FAST"] = "1"
    os.environ["ZOLO_OPT_MIXED"] = "1"
    zb = load_pkg()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    os.environ["ZOLO_DEVICE"] = str(local)
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
    try:
        i8_lib = int8_library_tops(torch)
    except Exception:  # torch._int_mm unavailable: the line carries null
        i8_lib = None
    a_host, s_host = make_input(n, args.kappa, 1003 + rank)
    dA = torch.from_numpy(a_host.T.copy()).to("cuda")  # column-major storage: dA[j, i] = A[i, j]
    s_true = torch.from_numpy(s_host).to("cuda")
    del a_host
    dQ = torch.empty_like(dA)
    dH = torch.empty((n, n), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()

    def set_form(name):
        f = FORMS[name]
        h.set_option(zb.OPT_SHARED_QR, f["shared_qr"])
        h.set_option(zb.OPT_NS_FINISH, f["ns_finish"])
        h.set_option(zb.OPT_CHOL_INVERSE, f["chol_inverse"])
        h.set_option(zb.OPT_BETA_FROB, f["beta_frob"])
        h.set_option(zb.OPT_TERM_PLAN, f["term_plan"])
        h.set_option(zb.OPT_MIXED, f["mixed"])
        return f

    def step(form, src):
        if form["one_call"]:
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

    def timed(form, steps):
        """steps solves between a barrier + synchronize on both sides; device ms per step (max over ranks)."""
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        launches, last = 0, None
        e0.record(stream)
        for _ in range(steps):
            last = step(form, dA)
            launches += last["launches"]
        e1.record(stream)
        torch.cuda.synchronize()
        t = max_over_ranks(dist, e0.elapsed_time(e1) / steps, "cuda")
        return t, launches, last

    def profiled(form):
        """per-kernel-class device time of one more solve: CUDA events around every launch,
        each launch timed alone (the device synchronized around it), the way a profiler's
        serialized launch list times it, so that the look-ahead panels running beside the
        trailing updates are not counted in the updates' time"""
        h.profile(True, serialize=True)
        h.profile_read(reset=True)
        step(form, dA)
        torch.cuda.synchronize()
        prof = h.profile_read(reset=True)
        h.profile(False)
        return prof

    results = {}
    # ---- headline: the mixed form (its W warm-up solves, K timed, clocks sampled) ----
    f = set_form("mixed")
    for _ in range(args.warmup):
        step(f, dA)
    clocks = ClockSampler(local)
    clocks.start()
    t_mixed, launches, st_mixed = timed(f, args.steps)
    ck = clocks.stop()
    results["mixed"] = (t_mixed, st_mixed, accuracy(torch, dA, dQ, dH, s_true), args.steps)
    prof_mixed = profiled(f)

    # ---- the plain FP64 form (same number of timed solves) ----
    f = set_form("fp64")
    for _ in range(max(1, min(args.warmup, 2))):
        step(f, dA)
    t_fp64, launches_fp64, st_fp64 = timed(f, args.steps)
    results["fp64"] = (t_fp64, st_fp64, accuracy(torch, dA, dQ, dH, s_true), args.steps)
    prof_fp64 = profiled(f)

    # ---- the reference's steps on the GPU ----
    f = set_form("reference_steps")
    step(f, dA)  # warm-up: its per-term stacks need their own workspace
    ref_steps = max(1, min(args.steps, 2))
    t_ref, _, st_ref = timed(f, ref_steps)
    results["reference_steps"] = (t_ref, st_ref, accuracy(torch, dA, dQ, dH), ref_steps)
    set_form("mixed")

    ok_mixed = (results["mixed"][2]["backward_error"] <= ACCURACY_TARGET
                and results["mixed"][2]["orthogonality"] <= ACCURACY_TARGET)
    head = "mixed" if ok_mixed else "fp64"
    t_ms, st_head, acc_head, _ = results[head]
    prof = prof_mixed if head == "mixed" else prof_fp64
    total_launches = launches if head == "mixed" else launches_fp64
    h.release()  # the default handle below gets the device memory

    # ---- e2e through the reference-facing C-ABI: pzolopd1_ on host arrays, as an unchanged
    # Fortran driver calls it (test_zolodrv1.f90:198), default handle with the options from
    # the environment; A in from pinned host memory and Q back, inside the timed region ----
    hA = torch.empty((n, n), dtype=torch.float64, pin_memory=True)
    hA.copy_(dA)
    hQ = torch.empty_like(hA, pin_memory=True)
    al_drv, be_drv, _ = zb.bounds_dev(h, n, n, dA.data_ptr(), n, mode=1)  # the driver's own bounds
    h.release()
    del dQ, dH
    torch.cuda.synchronize()
    torch.cuda.empty_cache()

    def e2e_call():
        info = zb.pzolopd_f77("N", rk, n, n, al_drv, be_drv, hA.data_ptr(), n, hQ.data_ptr(), n, "pzolopd1_")
        if info != 0:
            raise RuntimeError(f"pzolopd1_ INFO = {info}")

    e2e_call()  # creates the default handle and its workspace
    e2e_steps = max(1, min(args.steps, 3))
    if dist:
        dist.barrier()
    w0 = time.perf_counter()
    for _ in range(e2e_steps):
        e2e_call()
    e2e_s = max_over_ranks(dist, (time.perf_counter() - w0) / e2e_steps, "cuda")
    st_e2e = zb.DefaultHandle().stats()
    zb.lib().zolo_release_workspace(zb.DefaultHandle().ptr)
    # the other configurations, on one GPU: the 512-matrix batch and the full Zolo-SVD
    extras = {}
    if world == 1 and not args.no_extras:
        set_form("fp64")
        for name, fn in (("batch_c4", bench_batch_c4), ("svd_c5", bench_svd_c5)):
            try:
                extras[name] = fn(torch, zb, h)
            except Exception as exc:  # an extra must not hide the headline line
                extras[name] = {"error": str(exc)[:300]}
            h.release()
    q_e2e = torch.from_numpy(hQ.numpy()).to("cuda")
    eye = torch.eye(n, dtype=torch.float64, device="cuda")
    e2e_orth = float(torch.linalg.norm(q_e2e.T @ q_e2e - eye) / math.sqrt(n))  # Q^T Q (transposes cancel)
    del q_e2e, eye

    gk = [k for k in prof if k.startswith("dgemm")]
    g = {"ms": sum(prof[k]["ms"] for k in gk), "flops": sum(prof[k]["flops"] for k in gk),
         "launches": sum(prof[k]["launches"] for k in gk)}
    oz = prof.get("ozgemm", {"ms": 0.0, "flops": 0.0, "launches": 0})
    # the same DMMA roofline in the plain FP64 form, where DMMA carries every product
    gk64 = [k for k in prof_fp64 if k.startswith("dgemm")]
    g64 = {"ms": sum(prof_fp64[k]["ms"] for k in gk64), "flops": sum(prof_fp64[k]["flops"] for k in gk64),
           "launches": sum(prof_fp64[k]["launches"] for k in gk64)}
    ach64 = g64["flops"] / (g64["ms"] * 1e-3) / 1e12 if g64["ms"] > 0 else 0.0
    # shares of the timed step (the profiled solve times each launch alone, like the
    # serialized ncu launch list whose shares are relative to the solve's kernel time)
    prof_ms = t_ms
    achieved = g["flops"] / (g["ms"] * 1e-3) / 1e12 if g["ms"] > 0 else 0.0
    per_class = {k: {"launches": v["launches"], "ms": round(v["ms"], 3),
                     "tflops": round(v["flops"] / (v["ms"] * 1e-3) / 1e12, 3) if v["ms"] > 0 else None}
                 for k, v in prof.items()}
    i8_peak, i8_src = int8_peak_tops()
    oz_tops = OZ_PRODUCTS * oz["flops"] / (oz["ms"] * 1e-3) / 1e12 if oz["ms"] > 0 else 0.0

    def form_entry(name):
        t, st, acc, k = results[name]
        return {"s": t / 1e3, "steps": k, "backward_error": acc["backward_error"],
                "orthogonality": acc["orthogonality"], "sv_err_rel_smax": acc.get("sv_err_rel_smax"),
                "branches": st["branches"], "terms": st["terms"],
                "phases_ms": {"bounds": st["ms_bounds"], "iterations": st["ms_step"], "finish": st["ms_finish"],
                              "h_and_q": st["ms_h"]}}

    out = None
    if rank == 0:
        out = {
            "metric": METRIC, "value": t_ms / 1e3, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t_ms, "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"Zolo-PD r={rk} (bounds + PZOLOPD1 + H), n={n}, kappa={args.kappa:g}, "
                                   f"{head} form" + (" (FP64 emulated on INT8 tcgen05 for the Cholesky "
                                                     "iterations, finish and Q/H; bounds and QR iterations on "
                                                     "FP64 DMMA)" if head == "mixed" else " (FP64 on DMMA)"),
                       "n": n, "rk": rk, "kappa": args.kappa, "form": head, "seed": 1003 + rank,
                       "generator": "NumPy PCG64: s, then Haar U, V (QR of N(0,1), diag(R) > 0)",
                       "parallelism": f"replicas x{world}",
                       "l2": "inputs 512 MiB per matrix > 126 MB L2 (no flush needed)"},
            "accuracy": dict(acc_head, iterations=st_head["iterations"], ns_steps=st_head["ns_steps"],
                             branches=st_head["branches"], terms=st_head["terms"], target=ACCURACY_TARGET),
            "phases_ms": {"bounds": st_head["ms_bounds"], "iterations": st_head["ms_step"],
                          "finish": st_head["ms_finish"], "h_and_q": st_head["ms_h"]},
            "forms": {
                "mixed": form_entry("mixed"),
                "fp64": form_entry("fp64"),
                "reference_steps": form_entry("reference_steps"),
                "speedup_mixed_vs_fp64": t_fp64 / t_mixed,
                "mixed_meets_target": ok_mixed,
                "speedup_fp64_vs_reference_steps": t_ref / t_fp64,
            },
            "tflops_canonical": st_head["flops"] / (t_ms * 1e-3) / 1e12,
            "tflops_executed": st_head["flops_executed"] / (t_ms * 1e-3) / 1e12,
            "roofline": {"bound": "tensor", "kernel": "dgemm_kernel (FP64 DMMA mma.sync m16n8k8, all shapes)",
                         "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                         "frac": achieved / peak if peak else None,
                         "peak_source": "cuBLAS DGEMM 8192^3 measured in this run (FP64 tensor pipe)",
                         "traffic": DGEMM_TRAFFIC_BYTES, "traffic_launch": DGEMM_TRAFFIC_LAUNCH,
                         "share_of_step": g["ms"] / prof_ms if prof_ms else None,
                         "launches_per_step": g["launches"]},
            "roofline_fp64_form": {"bound": "tensor", "kernel": "dgemm_kernel (all shapes) in the plain FP64 form",
                                   "achieved": ach64, "peak": peak, "unit": "TFLOP/s",
                                   "frac": ach64 / peak if peak else None,
                                   "share_of_step": g64["ms"] / t_fp64 if t_fp64 else None,
                                   "launches_per_step": g64["launches"]},
            "roofline_ozgemm": {"bound": "tensor", "kernel": "ozgemm_kernel<8> (INT8 tcgen05.mma kind::i8, TMA, "
                                                             "TMEM accumulators)",
                                "achieved": oz_tops, "peak": i8_peak, "unit": "TOP/s (int8)",
                                "frac": oz_tops / i8_peak if i8_peak else None, "peak_source": i8_src,
                                "fp64_equivalent_tflops": oz["flops"] / (oz["ms"] * 1e-3) / 1e12 if oz["ms"] else None,
                                "share_of_step": oz["ms"] / prof_ms if prof_ms else None,
                                "launches_per_step": oz["launches"],
                                "int8_products_per_fp64_product": OZ_PRODUCTS,
                                "library_int8_tops": i8_lib,
                                "library_int8_source": "cuBLASLt INT8 GEMM 8192^3 (torch._int_mm) measured in "
                                                       "this run"},
            "kernel_classes": per_class,
            "e2e": {"value": e2e_s, "unit": UNIT, "h2d_bytes_per_step": 8 * n * n, "d2h_bytes_per_step": 8 * n * n,
                    "call": "pzolopd1_ (gfortran symbol) on pinned host arrays, default handle with ZOLO_FAST=1 "
                            "ZOLO_OPT_MIXED=1 from the environment; returns Q (PZOLOPD1 forms no H)",
                    "steps": e2e_steps, "branches": st_e2e["branches"], "orthogonality": e2e_orth},
            "configs": extras,
            "gpu_launches": int(total_launches),
            "clocks": ck,
            "cpu_baseline": {"value": None, "unit": UNIT, "cores": os.cpu_count(), "kind": "port",
                             "sample": "none here: one full oracle solve of this matrix takes minutes; it is "
                                       "timed, unscaled, by bench.py --impl reference"},
        }
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    h.close()
    if rank == 0:
        print(json.dumps(out), flush=True)
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    return run_gpu(args)


if __name__ == "__main__":
    sys.exit(main())
