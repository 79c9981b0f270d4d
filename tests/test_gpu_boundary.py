"""The reference-facing boundary on the GPU: the gfortran-mangled pzolopd1_ / pzolopd2_
called as an unchanged Fortran driver calls them (test_zolodrv1.f90:198: host arrays,
arguments by reference, hidden CHARACTER lengths), with the default handle's options
taken from the environment (ZOLO_FAST, ZOLO_OPT_<NAME>).  Each case runs in a child
process so that the default handle is created with that environment.  Tolerances:
backward error and orthogonality <= 10 n eps, the polar factor within 100 n eps kappa
of the one built into the matrix, PZOLOPD2 bitwise equal to PZOLOPD1."""
import json
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CHILD = r"""
import json, math, sys
import numpy as np
sys.path.insert(0, ROOT)
import importlib.util
spec = importlib.util.spec_from_file_location("zolo_svd_b200", ROOT + "/zolo-svd_b200/__init__.py",
                                              submodule_search_locations=[ROOT + "/zolo-svd_b200"])
zb = importlib.util.module_from_spec(spec); sys.modules["zolo_svd_b200"] = zb; spec.loader.exec_module(zb)
from oracle import zolo_oracle as zo
n, kappa = N, KAPPA
s = np.geomspace(1.0, 1.0 / kappa, n)
a, u, v = zo.make_matrix(n, s, 4242)
al, be, _ = zo.bounds_zolodrv(a)           # the driver's own bounds (LU 1-norm estimate)
q1 = np.zeros((n, n), order="F"); q2 = np.zeros((n, n), order="F")
i1 = zb.pzolopd_f77("N", 8, n, n, al, be, a.ctypes.data, n, q1.ctypes.data, n, "pzolopd1_")
st = zb.DefaultHandle().stats()
i2 = zb.pzolopd_f77("N", 8, n, n, al, be, a.ctypes.data, n, q2.ctypes.data, n, "pzolopd2_")
h = zb.DefaultHandle()
opts = {k: h.get_option(getattr(zb, "OPT_" + k)) for k in
        ("SHARED_QR", "NS_FINISH", "CHOL_INVERSE", "BETA_FROB", "TERM_PLAN", "MIXED", "MIXED_SLICES", "OWN_BOUNDS")}
hh = zo.polar_h(q1, a)
print(json.dumps({"info": [i1, i2], "opts": opts, "same": bool(np.array_equal(q1, q2)),
                  "bwd": zo.backward_error(a, q1, hh), "orth": zo.orthogonality(q1),
                  "dq": float(np.linalg.norm(q1 - u @ v.T) / math.sqrt(n)),
                  "branches": st["branches"], "terms": st["terms"], "alpha": st["alpha"], "beta": st["beta"],
                  "al": al, "be": be}))
"""


def run_child(env_extra, n=1024, kappa=1e8):
    env = dict(os.environ)
    for k in list(env):
        if k.startswith("ZOLO_OPT_") or k == "ZOLO_FAST":
            del env[k]
    env.update(env_extra)
    code = CHILD.replace("ROOT", repr(ROOT)).replace("N, KAPPA", f"{n}, {kappa!r}")
    r = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    return json.loads(r.stdout.strip().splitlines()[-1])


def check(out, n, kappa):
    eps = 2.220446049250313e-16
    assert out["info"] == [0, 0]
    assert out["same"]  # PZOLOPD2 is PZOLOPD1's contract (pzolopd2.f90 cannot link)
    assert out["bwd"] <= 10 * n * eps and out["orth"] <= 10 * n * eps
    assert out["dq"] <= 100 * n * eps * kappa


def test_unchanged_driver_reference_steps():
    out = run_child({})
    assert out["opts"] == {"SHARED_QR": 1, "NS_FINISH": 0, "CHOL_INVERSE": 0, "BETA_FROB": 0, "TERM_PLAN": 0,
                           "MIXED": 0, "MIXED_SLICES": 8, "OWN_BOUNDS": 0}
    assert out["alpha"] == out["al"] and out["beta"] == out["be"]  # the caller's bounds are used
    check(out, 1024, 1e8)


def test_unchanged_driver_fast_and_mixed_from_environment():
    out = run_child({"ZOLO_FAST": "1", "ZOLO_OPT_MIXED": "1", "ZOLO_OPT_TERM_PLAN": "1", "ZOLO_OPT_MIXED_SLICES": "x"},
                    n=2048, kappa=1e12)
    assert out["opts"] == {"SHARED_QR": 1, "NS_FINISH": 1, "CHOL_INVERSE": 1, "BETA_FROB": 1, "TERM_PLAN": 1,
                           "MIXED": 1, "MIXED_SLICES": 8, "OWN_BOUNDS": 1}
    assert out["beta"] != out["be"]  # the library's own (Frobenius) bound replaced the driver's
    assert out["branches"][0] == "QR" and max(out["terms"]) <= 8
    check(out, 2048, 1e12)


def test_environment_override_of_fast():
    out = run_child({"ZOLO_FAST": "1", "ZOLO_OPT_OWN_BOUNDS": "0", "ZOLO_OPT_SHARED_QR": "0"})
    assert out["opts"]["OWN_BOUNDS"] == 0 and out["opts"]["SHARED_QR"] == 0 and out["opts"]["NS_FINISH"] == 1
    assert out["beta"] == out["be"]
    check(out, 1024, 1e8)
