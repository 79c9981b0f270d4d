"""The CPU oracle against the golden fixtures and known-answer matrices (no GPU)."""
import json
import math
import os

import numpy as np
import pytest

from oracle import zolo_oracle as zo

GOLD = os.path.join(os.path.dirname(__file__), "golden")


@pytest.fixture(scope="module")
def scalars():
    with open(os.path.join(GOLD, "zolo_scalars.json")) as f:
        return json.load(f)


def _rel(a, b):
    a = np.asarray(a, dtype=float)
    b = np.asarray(b, dtype=float)
    return float(np.max(np.abs(a - b) / np.abs(b)))


def test_coeff_against_mpmath(scalars):
    """c_i, a_i, FONE, next CON vs 50-digit mpmath.

    The reference's double AGM / Landen evaluation (Auxil_Zolo.f90:36-128) loses
    accuracy as the modulus approaches 1: its relative error grows like eps*CON
    (cn(u) -> 0 near u = K is found by cancellation).  Agreement is
    required up to rounding; the bound used is max(1e-13, 20*eps*CON).
    """
    for row in scalars["coeff"]:
        con, rk = row["con"], row["rk"]
        c = zo.compute_coeff(con, zo.EPS, rk)
        fone = zo.zolo_fone(c, rk)
        nxt = zo.zolo_next_con(con, c, rk, fone)
        tol = max(1e-13, 20 * zo.EPS * con)
        assert _rel(c[: 2 * rk], row["c"]) <= tol, (con, rk)
        assert _rel(-c[2 * rk:], row["a"]) <= tol, (con, rk)
        assert _rel(fone, row["fone"]) <= tol, (con, rk)
        assert _rel(nxt, row["next_con"]) <= max(tol, 1e-12), (con, rk)


def test_hfunc_against_mpmath(scalars):
    for row in scalars["hfunc"]:
        assert abs(zo.hfunc(row["x"]) - row["h"]) <= 4 * zo.EPS * row["h"]


def test_qdwh_weights_monotone():
    l = 1e-12
    for _ in range(8):
        a, b, c, ln = zo.qdwh_weights(l)
        assert ln >= l - 4 * zo.EPS and ln <= 1.0 + 1e-12
        assert abs(b - (a - 1) ** 2 / 4) < 1e-12 * max(1, b)
        l = ln
    assert abs(l - 1.0) < 1e-12


def test_choosem_table():
    assert zo.choosem(1.0005) == 2 and zo.choosem(1.5) == 6 and zo.choosem(2.0) == 8
    assert zo.choosem(1e2) == 3 and zo.choosem(1e8) == 6 and zo.choosem(1e12) == 7 and zo.choosem(1e16) == 8


@pytest.fixture(scope="module")
def known():
    return dict(np.load(os.path.join(GOLD, "known_polar.npz")))


@pytest.mark.parametrize("tag,kappa", [("k7", 1e4), ("k33", 1e8), ("k64", 1e12)])
def test_oracle_qdwh_known_answer(known, tag, kappa):
    a = known[f"{tag}_a"]
    n = a.shape[1]
    q, h, st = zo.pqdwhfacs("N", a)
    assert st.info == 0
    assert zo.backward_error(a, q, h) <= 10 * n * zo.EPS
    assert zo.orthogonality(q) <= 10 * n * zo.EPS
    # polar factor vs the exact U V^T: conditioning ~ 1/sigma_min
    err = np.linalg.norm(q - known[f"{tag}_up"]) / math.sqrt(n)
    assert err <= 100 * zo.EPS * kappa * n
    # singular values = eig(H), relative to sigma_max
    ev = np.sort(np.linalg.eigvalsh(h))[::-1]
    assert np.max(np.abs(ev - known[f"{tag}_s"])) <= 1e-12 * known[f"{tag}_s"][0]
    # regression: same iteration count and branch split as when the fixture was made
    its = known[f"{tag}_qdwh_its"]
    assert st.iterations == its[0] and st.branches.count("QR") == its[1]


@pytest.mark.parametrize("tag", ["k7", "k33", "k64"])
def test_oracle_zolo_known_answer(known, tag):
    a = known[f"{tag}_a"]
    n = a.shape[1]
    al, be = known[f"{tag}_zolo4_ab"]
    q, st = zo.pzolopd1("N", 4, a, al, be)
    h = zo.polar_h(q, a)
    assert zo.backward_error(a, q, h) <= 10 * n * zo.EPS
    assert zo.orthogonality(q) <= 10 * n * zo.EPS
    its = known[f"{tag}_zolo4_its"]
    assert st.iterations == its[0] and st.branches.count("QR") == its[1]
    assert np.allclose(q, known[f"{tag}_zolo4_q"], atol=1e-13)


def test_zolo_terms_sum_equals_rational():
    """sum_j a_j x/(x^2 + c_2j-1) + x equals x prod (x^2+c_2j)/(x^2+c_2j-1) (partial fractions)."""
    con, rk = 1e6, 5
    c = zo.compute_coeff(con, zo.EPS, rk)
    for x in (1.0, 10.0, 1e3, con):
        lhs = x * (1.0 + sum(-c[2 * rk + j] / (x * x + c[2 * j]) for j in range(rk)))
        rhs = x
        for j in range(rk):
            rhs *= (x * x + c[2 * j + 1]) / (x * x + c[2 * j])
        assert abs(lhs - rhs) <= 1e-9 * abs(rhs)


def test_zoloqr_equals_zolochol_term():
    rng = np.random.default_rng(3)
    x = rng.standard_normal((40, 30)) / 10
    c = zo.compute_coeff(50.0, zo.EPS, 3)
    for ip in (1, 2, 3):
        zq = zo.zoloqr(x, c, 3, ip)
        zc, info = zo.zolochol("N", x, c, 3, ip)
        assert info == 0
        assert np.allclose(zq, zc, rtol=1e-10, atol=1e-12)


def test_structured_qr_q2_upper_triangular():
    rng = np.random.default_rng(4)
    x = rng.standard_normal((50, 20))
    w = np.vstack([x, 3.0 * np.eye(20)])
    q = zo.house_qr_q(w)
    assert np.all(np.tril(q[50:], -1) == 0.0)


def test_rectangular_oracle():
    rng = np.random.default_rng(5)
    s = np.geomspace(1, 1e-6, 30)
    a, u, v = zo.make_matrix(30, s, 21, m=45)
    q, h, st = zo.pqdwhfacs("N", a, bounds="qr")
    assert zo.backward_error(a, q, h) <= 10 * 30 * zo.EPS
    assert zo.orthogonality(q) <= 10 * 30 * zo.EPS


def test_spectral_split_oracle():
    rng = np.random.default_rng(6)
    n = 40
    v = zo.haar(n, rng)
    lam = np.concatenate([np.linspace(-3, -1, 15), np.linspace(0.5, 2, 25)])
    a = (v * lam) @ v.T
    a = 0.5 * (a + a.T)
    q, h, st = zo.pqdwhfacs("S", a, sigma=0.0)
    ev, vecs, rk = zo.zoloeig(a, q, np.random.default_rng(7))
    assert rk == 15
    assert np.allclose(np.sort(ev), np.sort(lam[:15]), atol=1e-12)
