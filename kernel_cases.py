#!/usr/bin/env python
"""Single-kernel cases of the polar-decomposition path, run through the C-ABI.

Each case builds its operands on the GPU, runs the named operation `--reps`
times and prints the device time per repetition (CUDA events on the handle's
stream).  The cases are the shapes that dominate a Zolo-PD / QDWH solve, so a
profiler pointed at one case sees the same kernel configuration as the full
solve (e.g. ``ncu -k regex:dgemm_kernel ... python kernel_cases.py --case gemm_nn``):

  gemm_nn      C = A B, M = N = K = n          (general DMMA GEMM, 128 x 128 tiles)
  gemm_rank32  C -= A B, M = N = n, K = 32     (streaming rank-32 update kernel)
  gemm_k128    C -= A B, M = N = n, K = 128    (block-reflector update, 64 x 64 tiles, C preloaded)
  gemm_m32     P = V^T W, M = 32, N = K = n    (panel projection, 32 x 64 tiles)
  syrk         lower(C) = A^T A, n x n          (Gram of the Cholesky form)
  geqrf        Householder QR of an n x n matrix (panel kernel + trailing GEMMs)
  potrf        Cholesky of an SPD n x n matrix  (leaf kernel + GEMMs)
  oz_nn        C = A B, M = N = K = n, FP64 emulated on the INT8 tensor cores (--slices planes)
  oz_syrk      lower(C) = A^T A, n x n, emulated (one splitting for both sides)
  oz_k128      C -= A B, M = N = n, K = 128, emulated (the block-reflector update shape)
  oz_m512      P = V^T W, M = 512, N = K = n, emulated (four batched 128-row projections)
  gemm_m512    the same on the DMMA GEMM
  polar        one Zolo-PD solve (bounds + PZOLOPD1 + H, zolo_polar_dev, FP64 fast form), kappa 1e12
  polar_mixed  the same in the mixed form (ZOLO_OPT_MIXED = 1)
  batch        the 512-matrix batched QDWH (zolo_qdwh_batch_dev), bucket graphs replayed

  python kernel_cases.py --case gemm_nn --n 4096 --reps 3
"""
from __future__ import annotations

import argparse
import importlib.util
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(HERE, "zolo-svd_b200")


def load_pkg():
    if "zolo_svd_b200" in sys.modules:
        return sys.modules["zolo_svd_b200"]
    spec = importlib.util.spec_from_file_location("zolo_svd_b200", os.path.join(PKG, "__init__.py"),
                                                  submodule_search_locations=[PKG])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["zolo_svd_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


CASES = ("gemm_nn", "gemm_rank32", "gemm_k128", "gemm_m32", "syrk", "geqrf", "potrf", "oz_nn", "oz_syrk", "oz_k128",
         "oz_m512", "gemm_m512", "polar", "polar_mixed", "batch")


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--case", choices=CASES, required=True)
    ap.add_argument("--n", type=int, default=4096)
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--slices", type=int, default=8)
    args = ap.parse_args()
    import torch
    zb = load_pkg()
    n = args.n
    h = zb.Handle(0)
    stream = torch.cuda.current_stream()
    h.set_stream(stream.cuda_stream)
    g = torch.Generator(device="cuda")
    g.manual_seed(7)
    f64 = dict(dtype=torch.float64, device="cuda")

    def randn(r, c):
        return torch.randn(c, r, generator=g, **f64)  # column-major r x c (torch row-major c x r)

    lib = zb.lib()
    flops = 0.0
    if args.case in ("gemm_nn", "gemm_rank32", "gemm_k128", "gemm_m32", "syrk"):
        if args.case == "gemm_nn":
            M, N, K, ta, tri = n, n, n, b"N", 0
        elif args.case == "gemm_rank32":
            M, N, K, ta, tri = n, n, 32, b"N", 0
        elif args.case == "gemm_k128":
            M, N, K, ta, tri = n, n, 128, b"N", 0
        elif args.case == "gemm_m32":
            M, N, K, ta, tri = 32, n, n, b"T", 0
        else:
            M, N, K, ta, tri = n, n, n, b"T", 1
        a = randn(K, M) if ta == b"T" else randn(M, K)
        b = randn(K, N)
        c = randn(M, N)
        lda = a.shape[1]
        beta = 1.0 if args.case in ("gemm_rank32", "gemm_k128") else 0.0
        alpha = -1.0 if args.case in ("gemm_rank32", "gemm_k128") else 1.0
        flops = (1.0 if tri else 2.0) * M * N * K

        def run():
            rc = lib.zolo_dgemm_dev(h.ptr, ta, b"N", M, N, K, alpha, a.data_ptr(), lda, b.data_ptr(), K, beta,
                                    c.data_ptr(), M, tri, 0)
            if rc:
                raise zb.ZoloError("zolo_dgemm_dev", rc)
    elif args.case in ("polar", "polar_mixed"):
        # A = U diag(s) V^T, s log-uniform in [1e-12, 1] (endpoints pinned), Haar U, V
        def haar():
            q, r = torch.linalg.qr(randn(n, n))
            return q * torch.sign(torch.diagonal(r))[None, :]
        e = torch.rand(n, generator=g, **f64) * -12.0
        e[0], e[-1] = 0.0, -12.0
        sv = torch.sort(10.0 ** e, descending=True).values
        u, v = haar(), haar()
        a = ((u * sv[None, :]) @ v.T).T.contiguous()  # column-major storage of A
        del u, v
        q = torch.empty_like(a)
        hh = torch.empty_like(a)
        for opt in (zb.OPT_SHARED_QR, zb.OPT_NS_FINISH, zb.OPT_CHOL_INVERSE, zb.OPT_BETA_FROB, zb.OPT_TERM_PLAN):
            h.set_option(opt, 1)
        h.set_option(zb.OPT_MIXED, 1 if args.case == "polar_mixed" else 0)
        flops = 0.0

        def run():
            zb.polar_dev(h, 8, n, n, a.data_ptr(), n, q.data_ptr(), n, hh.data_ptr(), n)
    elif args.case in ("oz_k128", "oz_m512", "gemm_m512"):
        if args.case == "oz_k128":
            M, N, K, ta, alpha, beta = n, n, 128, b"N", -1.0, 1.0
        else:
            M, N, K, ta, alpha, beta = 512, n, n, b"T", 1.0, 0.0
        a = randn(K, M) if ta == b"T" else randn(M, K)
        b = randn(K, N)
        c = randn(M, N)
        lda = a.shape[1]
        flops = 2.0 * M * N * K
        oz = args.case.startswith("oz")

        def run():
            if oz:
                rc = lib.zolo_ozgemm_dev(h.ptr, ta, b"N", M, N, K, alpha, a.data_ptr(), lda, b.data_ptr(), K, beta,
                                         c.data_ptr(), M, 0, 0, args.slices)
            else:
                rc = lib.zolo_dgemm_dev(h.ptr, ta, b"N", M, N, K, alpha, a.data_ptr(), lda, b.data_ptr(), K, beta,
                                        c.data_ptr(), M, 0, 0)
            if rc:
                raise zb.ZoloError("gemm", rc)
    elif args.case in ("oz_nn", "oz_syrk"):
        tri = 1 if args.case == "oz_syrk" else 0
        ta = b"T" if tri else b"N"
        a = randn(n, n)
        b = a if tri else randn(n, n)
        c = randn(n, n)
        flops = (1.0 if tri else 2.0) * n ** 3

        def run():
            rc = lib.zolo_ozgemm_dev(h.ptr, ta, b"N", n, n, n, 1.0, a.data_ptr(), n, b.data_ptr(), n, 0.0,
                                     c.data_ptr(), n, tri, 0, args.slices)
            if rc:
                raise zb.ZoloError("zolo_ozgemm_dev", rc)
    elif args.case == "batch":
        # the 512-member configuration's sizes (PCG64 seed 1004: n log-uniform in [64, 1024],
        # m = n (1 + U[0,1]), kappa log-uniform in [1e2, 1e14], s geometric), the members built
        # on the GPU from Haar factors; two calls first (eager, then captured), so that the
        # timed calls replay the bucket graphs
        import math
        import numpy as np
        rng = np.random.default_rng(1004)
        mats = []
        for _ in range(512):
            nn = int(round(math.exp(rng.uniform(math.log(64), math.log(1024)))))
            mm = int(round(nn * (1 + rng.uniform(0, 1))))
            kap = 10 ** rng.uniform(2, 14)
            su = torch.from_numpy(np.geomspace(1.0, 1.0 / kap, nn)).to("cuda")
            qu, ru = torch.linalg.qr(randn(mm, nn).T)
            qv, rv = torch.linalg.qr(randn(nn, nn))
            am = (qu * su[None, :]) @ qv.T  # m x n, row-major
            mats.append((mm, nn, am.T.contiguous()))
        outs = [(torch.empty_like(x), torch.empty((nn, nn), **f64)) for mm, nn, x in mats]
        members = [(mm, nn, x.data_ptr(), mm, q.data_ptr(), mm, hq.data_ptr(), nn)
                   for (mm, nn, x), (q, hq) in zip(mats, outs)]
        zb.qdwh_batch_dev(h, members)

        def run():
            zb.qdwh_batch_dev(h, members)
    elif args.case == "geqrf":
        w0 = randn(n, n)
        w = torch.empty_like(w0)
        tau = torch.empty(n, **f64)
        t = torch.empty(((n + 31) // 32) * 1024, **f64)
        flops = 4.0 / 3.0 * n ** 3

        def run():
            w.copy_(w0)
            rc = lib.zolo_dgeqrf_dev(h.ptr, n, n, -1, w.data_ptr(), n, tau.data_ptr(), t.data_ptr())
            if rc:
                raise zb.ZoloError("zolo_dgeqrf_dev", rc)
    else:
        x = randn(n, n)
        spd = (x.T @ x) / n + torch.eye(n, **f64)
        w = torch.empty_like(spd)
        flops = n ** 3 / 3.0

        def run():
            w.copy_(spd)
            rc = lib.zolo_dpotrf_dev(h.ptr, n, w.data_ptr(), n)
            if rc:
                raise zb.ZoloError("zolo_dpotrf_dev", rc)

    run()
    torch.cuda.synchronize()
    for i in range(args.reps):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        run()
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        rate = f", {flops / (ms * 1e-3) / 1e12:.2f} TFLOP/s" if flops else ""
        print(f"{args.case} n={n} rep {i}: {ms:.3f} ms{rate}", flush=True)
    if args.case == "batch":
        st = zb.batch_stats(h)
        print(f"batch: {h.stats()['launches']} kernel launches per call, {st['buckets']} buckets, "
              f"{st['graph_replays']} graph replays", flush=True)
    h.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())
