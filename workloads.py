#!/usr/bin/env python
"""The reference's other benchmark workloads on one GPU, through the device entry
points, with time and accuracy (one JSON line per workload).  The n = 8192 Zolo-PD
headline is bench.py; these are the remaining configurations, on seeded synthetic
matrices A = U diag(s) V^T with Haar U, V and the stated spectra:

  c1  QDWH-PD (PQDWHFACS), n = 1024, s geometric in [1e-8, 1]
  c2  Zolo-PD r = 8, n = 4096, s geometric in [1e-16, 1] with 5 % duplicated values,
      reference stopping rule, Newton-Schulz finish, and the fast form (zolo_polar_dev
      with every cost option)
  c4  512 matrices, n log-uniform in [64, 1024], m = n (1 + U[0, 1]), kappa
      log-uniform in [1e2, 1e14], s geometric: batched QDWH-PD (zolo_qdwh_batch_dev)
      against one zolo_qdwh_dev call per matrix
  c5  Zolo-SVD (Zolo-PD r = 8 + eigensolver of H), 16384 x 8192: 70 % of s geometric
      in [1e-10, 1], 20 % exactly 1, 10 % in clusters of relative gap 1e-9; with the
      fast options, with the reference's steps, and with QDWH as the polar step

Device times are CUDA events around the calls on the handle's stream (inputs
resident in HBM, a warm-up call first).

  python workloads.py c1 c2 c4 c5
"""
from __future__ import annotations

import importlib.util
import json
import math
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


def main(argv) -> int:
    import torch
    zb = load_pkg()
    h = zb.Handle(0)
    st = torch.cuda.current_stream()
    h.set_stream(st.cuda_stream)
    eye = lambda n: torch.eye(n, dtype=torch.float64, device="cuda")  # noqa: E731

    def haar(m, n, g):
        q, r = torch.linalg.qr(torch.randn(m, n, dtype=torch.float64, device="cuda", generator=g))
        return q * torch.sign(torch.diagonal(r))[None, :]

    def timed(fn, reps=1):
        fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        for _ in range(reps):
            fn()
        e1.record(st)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    def set_fast(on):
        # the cost options of the fast form (each changes the cost, not the result beyond rounding)
        for opt in (zb.OPT_NS_FINISH, zb.OPT_CHOL_INVERSE, zb.OPT_BETA_FROB, zb.OPT_TERM_PLAN):
            h.set_option(opt, 1 if on else 0)

    def pd_errors(a, q, hh, s=None):
        n = q.shape[1]
        out = {"backward_error": float(torch.linalg.norm(a - q @ hh) / torch.linalg.norm(a)),
               "orthogonality": float(torch.linalg.norm(q.T @ q - eye(n)) / math.sqrt(n))}
        if s is not None:
            ev = torch.sort(torch.linalg.eigvalsh(0.5 * (hh + hh.T)), descending=True).values
            out["sv_err_rel_smax"] = float(torch.max(torch.abs(ev - s)) / s[0])
        return out

    for w in argv:
        if w == "c1":
            n = 1024
            g = torch.Generator(device="cuda")
            g.manual_seed(1001)
            s = torch.logspace(0, -8, n, dtype=torch.float64, device="cuda")
            u, v = haar(n, n, g), haar(n, n, g)
            a = (u * s[None, :]) @ v.T
            da = a.T.contiguous()
            dq, dh = torch.empty_like(da), torch.empty_like(da)
            ms = timed(lambda: zb.qdwh_dev(h, "N", n, n, 0.0, da.data_ptr(), n, dq.data_ptr(), n, dh.data_ptr(), n,
                                           0, 12, 0), reps=5)
            stt = h.stats()
            line = {"workload": "c1 QDWH-PD n=1024 kappa=1e8", "ms": ms, "iterations": stt["iterations"],
                    "branches": stt["branches"], "tflops_canonical": stt["flops"] / (ms * 1e-3) / 1e12}
            line.update(pd_errors(a, dq.T, dh.T, s))
            print(json.dumps(line), flush=True)
        elif w == "c2":
            n = 4096
            g = torch.Generator(device="cuda")
            g.manual_seed(1002)
            s = torch.logspace(0, -16, n, dtype=torch.float64, device="cuda")
            idx = torch.randperm(n - 1, generator=g, device="cuda")[: n // 20] + 1
            s[idx] = s[idx - 1]
            s = torch.sort(s, descending=True).values
            u, v = haar(n, n, g), haar(n, n, g)
            a = (u * s[None, :]) @ v.T
            da = a.T.contiguous()
            dq, dh = torch.empty_like(da), torch.empty_like(da)
            for form in ("reference_rule", "ns_finish", "fast"):
                set_fast(form == "fast")
                h.set_option(zb.OPT_NS_FINISH, 0 if form == "reference_rule" else 1)

                def run():
                    if form == "fast":
                        zb.polar_dev(h, 8, n, n, da.data_ptr(), n, dq.data_ptr(), n, dh.data_ptr(), n)
                        return
                    al, be, _ = zb.bounds_dev(h, n, n, da.data_ptr(), n, mode=1)
                    zb.pzolopd1_dev(h, "N", 8, n, n, al, be, da.data_ptr(), n, dq.data_ptr(), n, dh.data_ptr(), n)
                ms = timed(run, reps=3)
                stt = h.stats()
                line = {"workload": "c2 Zolo-PD r=8 n=4096 kappa=1e16 clustered", "form": form, "ms": ms,
                        "branches": stt["branches"], "terms": stt["terms"]}
                line.update(pd_errors(a, dq.T, dh.T, s))
                print(json.dumps(line), flush=True)
            set_fast(False)
        elif w == "c4":
            import numpy as np
            rng = np.random.default_rng(1004)
            g = torch.Generator(device="cuda")
            g.manual_seed(1004)
            mats = []
            for i in range(512):
                n = int(round(math.exp(rng.uniform(math.log(64), math.log(1024)))))
                m = int(round(n * (1 + rng.uniform(0, 1))))
                kappa = 10 ** rng.uniform(2, 14)
                s = torch.logspace(0, -math.log10(kappa), n, dtype=torch.float64, device="cuda")
                u, v = haar(m, n, g), haar(n, n, g)
                a = (u * s[None, :]) @ v.T
                mats.append((m, n, a, a.T.contiguous(), s))
            dq = [torch.empty_like(x[3]) for x in mats]
            dh = [torch.empty((x[1], x[1]), dtype=torch.float64, device="cuda") for x in mats]
            members = [(m, n, da.data_ptr(), m, q.data_ptr(), m, hh.data_ptr(), n)
                       for (m, n, _, da, _), q, hh in zip(mats, dq, dh)]
            res = {}
            ms_b = timed(lambda: res.update(r=zb.qdwh_batch_dev(h, members)), reps=3)
            stt = h.stats()
            info, its = res["r"]
            worst = {"backward_error": 0.0, "orthogonality": 0.0, "sv_err_rel_smax": 0.0}
            for (m, n, a, da, s), q, hh in zip(mats, dq, dh):
                e = pd_errors(a, q.T, hh.T, s)
                for k in worst:
                    worst[k] = max(worst[k], e[k] / (10 * n * 2.220446049250313e-16) if k != "sv_err_rel_smax"
                                   else e[k])
            # one solve per matrix, the same inputs
            def loop():
                for (m, n, _, da, _), q, hh in zip(mats, dq, dh):
                    zb.qdwh_dev(h, "N", m, n, 0.0, da.data_ptr(), m, q.data_ptr(), m, hh.data_ptr(), n, 0, 12, 0)
            ms_l = timed(loop, reps=1)
            line = {"workload": "c4 512 matrices n in [64,1024] m in [n,2n] kappa in [1e2,1e14], QDWH-PD",
                    "ms_batched": ms_b, "matrices_per_s_batched": 512 / (ms_b * 1e-3),
                    "ms_per_matrix_loop": ms_l, "matrices_per_s_loop": 512 / (ms_l * 1e-3),
                    "speedup": ms_l / ms_b, "info_nonzero": int(sum(1 for x in info if x)),
                    "max_iterations": int(max(its)),
                    "tflops_useful": stt["flops"] / (ms_b * 1e-3) / 1e12,
                    "tflops_executed": stt["flops_executed"] / (ms_b * 1e-3) / 1e12,
                    "worst_backward_error_over_10neps": worst["backward_error"],
                    "worst_orthogonality_over_10neps": worst["orthogonality"],
                    "worst_sv_err_rel_smax": worst["sv_err_rel_smax"]}
            print(json.dumps(line), flush=True)
            del mats, dq, dh
            torch.cuda.empty_cache()
            h.release()
        elif w == "c5":
            m, n = 16384, 8192
            g = torch.Generator(device="cuda")
            g.manual_seed(1005)
            n70, n20 = int(0.7 * n), int(0.2 * n)
            n10 = n - n70 - n20
            geo = torch.logspace(0, -10, n70, dtype=torch.float64, device="cuda")
            one = torch.ones(n20, dtype=torch.float64, device="cuda")
            base = torch.logspace(-1, -9, n10 // 8 + 1, dtype=torch.float64, device="cuda")
            rel = 1 + 1e-9 * torch.arange(8, dtype=torch.float64, device="cuda")
            s = torch.sort(torch.cat([geo, one, (base[:, None] * rel[None, :]).reshape(-1)[:n10]]),
                           descending=True).values
            u, v = haar(m, n, g), haar(n, n, g)
            a = (u * s[None, :]) @ v.T
            del u, v
            da = a.T.contiguous()
            du = torch.empty_like(da)
            ds = torch.empty(n, dtype=torch.float64, device="cuda")
            dv = torch.empty((n, n), dtype=torch.float64, device="cuda")
            for algo, fast in ((1, True), (1, False), (0, False)):
                set_fast(fast)
                ms = timed(lambda: zb.svd_dev(h, m, n, da.data_ptr(), m, du.data_ptr(), m, ds.data_ptr(),
                                              dv.data_ptr(), n, algo=algo, rk=8))
                U, V = du.T, dv.T
                line = {"workload": "c5 Zolo-SVD 16384x8192 kappa=1e10 clustered",
                        "polar": ("zolo-pd r=8" + (" fast options" if fast else "")) if algo else "qdwh", "ms": ms,
                        "residual": float(torch.linalg.norm(a - (U * ds[None, :]) @ V.T) / torch.linalg.norm(a)),
                        "sv_err_rel_smax": float(torch.max(torch.abs(torch.sort(ds, descending=True).values - s))
                                                 / s[0]),
                        "orth_u": float(torch.linalg.norm(U.T @ U - eye(n)) / math.sqrt(n)),
                        "orth_v": float(torch.linalg.norm(V.T @ V - eye(n)) / math.sqrt(n))}
                print(json.dumps(line), flush=True)
            set_fast(False)
            del a, da, du, dv
            torch.cuda.empty_cache()
            h.release()
        else:
            print(json.dumps({"workload": w, "error": "unknown workload"}), flush=True)
    h.close()
    return 0


if __name__ == "__main__":
    sys.exit(main(sys.argv[1:] or ["c1", "c2", "c4", "c5"]))
