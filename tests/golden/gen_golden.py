"""Generate the golden fixtures used by the tests (run from the repository root).

    python tests/golden/gen_golden.py

1. ``zolo_scalars.json``: Zolotarev shifts c_i, weights a_i, FONE and the next
   CON for (CON, r) pairs, and the QDWH weight h(l), all evaluated with mpmath
   at 50 digits -- independently of the double-precision AGM / Landen code the
   reference uses (Auxil_Zolo.f90:36-200, hfunc.f90:2-42).  The modulus is
   taken from the double value alpha = acos(1/CON) exactly as the reference
   forms it (Auxil_Zolo.f90:176-177), so the fixture pins the elliptic-function
   evaluation, not the rounding of alpha.
2. ``known_polar.npz``: small matrices A = U diag(s) V^T with their exact
   polar factor U V^T, H = V diag(s) V^T and singular values, plus the oracle's
   QDWH / Zolo-PD outputs (iteration count and branch sequence) for regression.
"""
from __future__ import annotations

import json
import math
import os
import sys

import mpmath as mp
import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.abspath(os.path.join(HERE, "..", "..")))

from oracle import zolo_oracle as zo  # noqa: E402

mp.mp.dps = 50


def mp_coeff(con: float, rk: int):
    alpha = mp.mpf(math.acos(1.0 / con))  # the double the reference computes
    m = mp.sin(alpha) ** 2
    kk = mp.ellipk(m)
    c = []
    for i in range(1, 2 * rk + 1):
        u = i * kk / (2 * rk + 1)
        sn = mp.ellipfun("sn", u, m=m)
        cn = mp.ellipfun("cn", u, m=m)
        c.append(sn ** 2 / cn ** 2)
    a = []
    for i in range(1, rk + 1):
        v = mp.mpf(1)
        for j in range(1, rk + 1):
            v *= c[2 * i - 2] - c[2 * j - 1]
            if i != j:
                v /= c[2 * i - 2] - c[2 * j - 2]
        a.append(-v)
    fone = mp.mpf(1)
    for i in range(1, rk + 1):
        fone *= (1 + c[2 * i - 1]) / (1 + c[2 * i - 2])
    cn_ = mp.mpf(con)
    fcon = cn_
    for i in range(1, rk + 1):
        fcon *= (cn_ ** 2 + c[2 * i - 1]) / (cn_ ** 2 + c[2 * i - 2])
    nxt = max(fcon / fone, mp.mpf(1))
    return [float(x) for x in c], [float(x) for x in a], float(fone), float(nxt)


def mp_hfunc(x: float) -> float:
    x = mp.mpf(x)
    x2 = x * x
    if abs(x - 1) <= 30 * zo.EPS:
        ww = mp.mpf(0)
    else:
        ww = mp.cbrt(4 * (1 - x2) / (x2 * x2))
    s1 = mp.sqrt(1 + ww)
    return float(s1 + mp.sqrt(8 - 4 * ww + 8 * (2 - x2) / (x2 * s1)) / 2)


def main() -> None:
    cons = [1.5, 10.0, 1.0e2, 1.0e4, 1.0e8, 1.0e12, 1.0e16]
    rows = []
    for con in cons:
        for rk in range(1, 9):
            c, a, fone, nxt = mp_coeff(con, rk)
            rows.append(dict(con=con, rk=rk, c=c, a=a, fone=fone, next_con=nxt))
    hx = [1.0e-16, 1.0e-12, 1.0e-8, 1.0e-4, 1.0e-2, 0.1, 0.5, 0.9, 0.999]
    hv = [dict(x=x, h=mp_hfunc(x)) for x in hx]
    with open(os.path.join(HERE, "zolo_scalars.json"), "w") as f:
        json.dump(dict(coeff=rows, hfunc=hv), f, indent=1)

    cases = {}
    for tag, (m, n, kappa, seed) in dict(k7=(7, 7, 1e4, 11), k33=(33, 33, 1e8, 12),
                                         k64=(64, 64, 1e12, 13), r96x64=(96, 64, 1e6, 14)).items():
        s = np.geomspace(1.0, 1.0 / kappa, n)
        a, u, v = zo.make_matrix(n, s, seed, m=m)
        cases[f"{tag}_a"] = a
        cases[f"{tag}_up"] = u @ v.T
        cases[f"{tag}_h"] = (v * s[None, :]) @ v.T
        cases[f"{tag}_s"] = s
        if m == n:
            q, h, st = zo.pqdwhfacs("N", a)
            cases[f"{tag}_qdwh_q"] = q
            cases[f"{tag}_qdwh_its"] = np.array([st.iterations, st.branches.count("QR")])
            al, be, _ = zo.bounds_zolodrv(a)
            qz, stz = zo.pzolopd1("N", 4, a, al, be)
            cases[f"{tag}_zolo4_q"] = qz
            cases[f"{tag}_zolo4_its"] = np.array([stz.iterations, stz.branches.count("QR")])
            cases[f"{tag}_zolo4_ab"] = np.array([al, be])
    np.savez_compressed(os.path.join(HERE, "known_polar.npz"), **cases)


if __name__ == "__main__":
    main()
