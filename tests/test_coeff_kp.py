"""Zolotarev coefficients from the complementary modulus (zolo_compute_coeff_kp, the
term plan's coefficients) against 60-digit mpmath elliptic functions, over CON from 2 to
1e22 (no GPU).  Compute_Coeff's own formula (alpha = acos(1/CON)) agrees with them where
it is exact, i.e. to ~1e-16 CON relative."""
import mpmath as mp
import numpy as np
import pytest

import zolo_svd_b200 as zb
from oracle import zolo_oracle as zo


def _mp_coeff(con, r):
    with mp.workdps(60):
        kp = mp.mpf(1) / mp.mpf(con)
        m = 1 - kp ** 2
        k = mp.ellipk(m)
        c = []
        for i in range(1, 2 * r + 1):
            u = i * k / (2 * r + 1)
            c.append((mp.ellipfun("sn", u, m=m) / mp.ellipfun("cn", u, m=m)) ** 2)
        a = []
        for i in range(1, r + 1):
            v = mp.mpf(1)
            for j in range(1, r + 1):
                v *= c[2 * i - 2] - c[2 * j - 1]
                if i != j:
                    v /= c[2 * i - 2] - c[2 * j - 2]
            a.append(v)
        return [float(x) for x in c + a]


@pytest.mark.parametrize("con", [2.0, 30.0, 1e4, 1e7, 1e9, 1e13, 1e16, 1e19, 1e22])
def test_coeff_kp_against_mpmath(con):
    for r in (1, 3, 8):
        got = zb.compute_coeff_kp(con, zo.EPS, r)
        ref = np.array(_mp_coeff(con, r))
        assert np.max(np.abs(got - ref) / np.abs(ref)) <= 1e-9, (con, r)
        if con <= 1e4:
            assert np.max(np.abs(zb.compute_coeff(con, zo.EPS, r) - got) / np.abs(ref)) <= max(1e-13, 50 * zo.EPS * con)


def test_coeff_kp_rejects_bad_input():
    with pytest.raises(zb.ZoloError):
        zb.compute_coeff_kp(1.0, zo.EPS, 3)
    with pytest.raises(zb.ZoloError):
        zb.compute_coeff_kp(10.0, zo.EPS, 9)
