"""End-to-end parity of the polar decompositions on the GPU, through the
reference-named C-ABI entry points, against the oracle on the same seeded
matrices.  Acceptance (per the target of 10*n*eps): backward error
||A - QH||_F/||A||_F and orthogonality ||Q^T Q - I||_F/sqrt(n) each <= 10*n*eps
(floored at 1e-14 for tiny n), singular values eig(H) within 1e-12 of the
oracle relative to sigma_max, the same iteration count / branch sequence as the
oracle when both start from the same bounds, and Q within
max(1e-12, 100*n*eps*kappa) of the oracle's Q."""
import math
import os

import numpy as np
import pytest

import zolo_svd_b200 as zb
from oracle import zolo_oracle as zo

pytestmark = pytest.mark.gpu
EPS = zo.EPS
GOLD = os.path.join(os.path.dirname(__file__), "golden")


def tol_n(n):
    return max(10 * n * EPS, 1e-14)


def check_pd(a, q, h, n):
    assert zo.backward_error(a, q, h) <= tol_n(n)
    assert zo.orthogonality(q) <= tol_n(n)


@pytest.mark.parametrize("n,kappa", [(1, 1.0), (2, 10.0), (7, 1e4), (33, 1e8), (64, 1e12), (65, 1e8), (100, 1e12),
                                     (130, 1e16)])
def test_pqdwhfacs_vs_oracle(n, kappa):
    s = np.geomspace(1.0, 1.0 / kappa, n) if n > 1 else np.array([0.5])
    a, u, v = zo.make_matrix(n, s, 100 + n)
    q, h, info = zb.pqdwhfacs("N", a)
    assert info == 0
    q_o, h_o, st_o = zo.pqdwhfacs("N", a, bounds="qr")
    check_pd(a, q, h, n)
    ev = np.sort(np.linalg.eigvalsh(h))
    ev_o = np.sort(np.linalg.eigvalsh(h_o))
    assert np.max(np.abs(ev - ev_o)) <= 1e-12 * max(ev_o.max(), 1e-300)
    assert np.linalg.norm(q - q_o) / math.sqrt(n) <= max(1e-12, 100 * n * EPS * kappa)


def test_pqdwhfacs_iteration_sequence_matches_oracle():
    n = 96
    s = np.geomspace(1.0, 1e-10, n)
    a, _, _ = zo.make_matrix(n, s, 7)
    h = zb.Handle(0)
    import torch
    da = zb.colmajor_to_device(a)
    dq = torch.zeros_like(da)
    zb.qdwh_dev(h, "N", n, n, 0.0, da.data_ptr(), n, dq.data_ptr(), n, 0, 1, 0, 12, 0)
    st = h.stats()
    _, _, st_o = zo.pqdwhfacs("N", a, bounds="qr")
    assert st["iterations"] == st_o.iterations
    assert st["branches"] == st_o.branches
    assert abs(st["beta"] - st_o.beta) <= 1e-4 * st_o.beta  # kappa = 1e10: ~kappa*eps
    h.close()


@pytest.mark.parametrize("rk", [1, 2, 4, 8])
@pytest.mark.parametrize("n,kappa", [(40, 1e6), (100, 1e12)])
def test_pzolopd1_vs_oracle(rk, n, kappa):
    s = np.geomspace(1.0, 1.0 / kappa, n)
    a, _, _ = zo.make_matrix(n, s, 200 + n + rk)
    al, be, _ = zo.bounds_zolodrv(a)
    q, info = zb.pzolopd1("N", rk, a, al, be)
    assert info == 0
    q_o, st_o = zo.pzolopd1("N", rk, a, al, be)
    h = zo.polar_h(q, a)
    check_pd(a, q, h, n)
    assert np.linalg.norm(q - q_o) / math.sqrt(n) <= max(1e-12, 100 * n * EPS * kappa)


def test_pzolopd1_branch_sequence_matches_oracle():
    import torch
    n, rk = 80, 4
    s = np.geomspace(1.0, 1e-12, n)
    a, _, _ = zo.make_matrix(n, s, 31)
    al, be, _ = zo.bounds_zolodrv(a)
    h = zb.Handle(0)
    da = zb.colmajor_to_device(a)
    dq = torch.zeros_like(da)
    zb.pzolopd1_dev(h, "N", rk, n, n, al, be, da.data_ptr(), n, dq.data_ptr(), n)
    st = h.stats()
    _, st_o = zo.pzolopd1("N", rk, a, al, be)
    assert st["iterations"] == st_o.iterations
    assert st["branches"] == st_o.branches
    np.testing.assert_array_equal(np.array(st["con"]), np.array(st_o.con))  # host scalar recursion is bitwise
    h.close()


@pytest.mark.parametrize("m,n,rk", [(64, 64, 8), (97, 97, 3), (200, 130, 5), (301, 300, 8), (700, 257, 2), (600, 600, 4)])
def test_pzolopd1_shared_qr_matches_per_term_qr(m, n, rk):
    """The QR iterations with one QR of X shared by the r terms (interleaved
    2n x n stacks) against one QR per (m+n) x n stack (zoloqr.f90:99-111) and
    against the oracle: same branch sequence, same iterate to rounding."""
    import torch
    kappa = 1e6  # the first step takes the QR form; Q is determined to ~kappa*eps
    s = np.geomspace(1.0, 1.0 / kappa, n)
    a, u, v = zo.make_matrix(n, s, 900 + m + n, m=m)
    h = zb.Handle(0)
    da = zb.colmajor_to_device(a)
    al, be, _ = zb.bounds_dev(h, m, n, da.data_ptr(), m, mode=1)
    out = {}
    for shared in (1, 0):
        h.set_option(zb.OPT_SHARED_QR, shared)
        dq = torch.zeros_like(da)
        dh = torch.zeros((n, n), dtype=torch.float64, device="cuda")
        zb.pzolopd1_dev(h, "N", rk, m, n, al, be, da.data_ptr(), m, dq.data_ptr(), m, dh.data_ptr(), n)
        out[shared] = (zb.device_to_colmajor(dq), zb.device_to_colmajor(dh), h.stats())
    h.close()
    (q1, h1, st1), (q0, h0, st0) = out[1], out[0]
    assert st1["branches"] == st0["branches"] and st1["branches"][0] == "QR"  # first step takes the QR form
    assert st1["iterations"] == st0["iterations"]
    check_pd(a, q1, h1, n)
    # both forms are backward stable; Q itself is determined to ~kappa * eps
    assert np.linalg.norm(q1 - q0) / math.sqrt(n) <= max(1e-12, 10 * n * EPS * kappa)
    assert np.linalg.norm(q1 - u @ v.T) / math.sqrt(n) <= max(1e-12, 100 * n * EPS * kappa)
    if m == n:
        q_o, st_o = zo.pzolopd1("N", rk, a, al, be)
        assert st1["branches"] == st_o.branches
        assert np.linalg.norm(q1 - q_o) / math.sqrt(n) <= max(1e-12, 100 * n * EPS * kappa)


def _pzolopd1_dev_run(h, a, rk, al, be, ns_finish):
    import torch
    m, n = a.shape
    h.set_option(zb.OPT_NS_FINISH, ns_finish)
    da = zb.colmajor_to_device(a)
    dq = torch.zeros_like(da)
    dh = torch.zeros((n, n), dtype=torch.float64, device="cuda")
    zb.pzolopd1_dev(h, "N", rk, m, n, al, be, da.data_ptr(), m, dq.data_ptr(), m, dh.data_ptr(), n)
    h.set_option(zb.OPT_NS_FINISH, 0)
    return zb.device_to_colmajor(dq), zb.device_to_colmajor(dh), h.stats()


@pytest.mark.parametrize("m,n,kappa,rk", [(300, 300, 1e12, 8), (256, 256, 1e16, 8), (200, 200, 1e8, 2),
                                          (330, 200, 1e12, 4), (129, 129, 1e14, 8), (160, 160, 1e10, 1)])
def test_ns_finish_matches_reference_rule(m, n, kappa, rk):
    """Finishing with FP64 Newton-Schulz once ||X^T X - I||_F/sqrt(n) <= 0.1 gives the
    reference rule's accuracy (10*n*eps) with no more Zolo iterations; the iterations it
    does run are the reference rule's."""
    s = np.geomspace(1.0, 1.0 / kappa, n)
    a, _, _ = zo.make_matrix(n, s, 500 + m + n + rk, m=m)
    h = zb.Handle(0)
    da = zb.colmajor_to_device(a)
    al, be, _ = zb.bounds_dev(h, m, n, da.data_ptr(), m, mode=1)
    q0, h0, st0 = _pzolopd1_dev_run(h, a, rk, al, be, 0)
    q1, h1, st1 = _pzolopd1_dev_run(h, a, rk, al, be, 1)
    h.close()
    assert st0["ns_finish"] == 0 and st0["ns_steps"] == 0
    it1 = st1["iterations"]
    assert it1 <= st0["iterations"]
    assert st1["branches"][:it1] == st0["branches"][:it1]
    if st1["ns_finish"]:
        assert 0 <= st1["ns_steps"] <= 12
        assert st1["branches"][it1:] == ["NS"] * st1["ns_steps"]
    else:
        assert st1["ns_steps"] == 0 and it1 == st0["iterations"]
    if (n, kappa, rk) == (300, 1e12, 8):
        assert st1["ns_finish"] == 1 and it1 < st0["iterations"]
    check_pd(a, q1, h1, n)
    check_pd(a, q0, h0, n)
    assert np.linalg.norm(q1 - q0) / math.sqrt(n) <= max(1e-12, 10 * n * EPS * kappa)


@pytest.mark.parametrize("m,n,kappa,rk", [(300, 300, 1e12, 8), (420, 250, 1e10, 4), (129, 129, 1e16, 8),
                                          (700, 700, 1e14, 8), (65, 65, 1e8, 3)])
def test_chol_inverse_matches_solve_form(m, n, kappa, rk):
    """Cholesky iterations through S = sum_j w_j L_j^{-T} L_j^{-1} and one Z = X S against the
    two-triangular-solve form (zolochol.f90:87-113): same branch sequence, both backward
    stable (10*n*eps), the same iterate to within kappa*eps."""
    s = np.geomspace(1.0, 1.0 / kappa, n)
    a, u, v = zo.make_matrix(n, s, 800 + m + n + rk, m=m)
    h = zb.Handle(0)
    da = zb.colmajor_to_device(a)
    al, be, _ = zb.bounds_dev(h, m, n, da.data_ptr(), m, mode=1)
    q0, h0, st0 = _pzolopd1_dev_run(h, a, rk, al, be, 0)
    h.set_option(zb.OPT_CHOL_INVERSE, 1)
    q1, h1, st1 = _pzolopd1_dev_run(h, a, rk, al, be, 0)
    h.set_option(zb.OPT_CHOL_INVERSE, 0)
    h.close()
    assert st1["branches"] == st0["branches"] and "CH" in st1["branches"]
    check_pd(a, q1, h1, n)
    assert np.linalg.norm(q1 - q0) / math.sqrt(n) <= max(1e-12, 10 * n * EPS * kappa)
    assert np.linalg.norm(q1 - u @ v.T) / math.sqrt(n) <= max(1e-12, 100 * n * EPS * kappa)


def test_solves_are_bitwise_reproducible():
    """Fixed reduction orders everywhere (no floating-point atomics): the same
    solve twice gives the same bits, for both Zolo-PD forms and QDWH."""
    import torch
    n = 300
    s = np.geomspace(1.0, 1e-12, n)
    a, _, _ = zo.make_matrix(n, s, 4242)
    h = zb.Handle(0)
    da = zb.colmajor_to_device(a)
    outs = []
    for rep in range(2):
        dq = torch.zeros_like(da)
        al, be, _ = zb.bounds_dev(h, n, n, da.data_ptr(), n, mode=1)
        zb.pzolopd1_dev(h, "N", 8, n, n, al, be, da.data_ptr(), n, dq.data_ptr(), n)
        dq2 = torch.zeros_like(da)
        zb.qdwh_dev(h, "N", n, n, 0.0, da.data_ptr(), n, dq2.data_ptr(), n, 0, 1, 0, 12, 0)
        outs.append((al, be, dq.clone(), dq2.clone()))
    h.close()
    assert outs[0][0] == outs[1][0] and outs[0][1] == outs[1][1]
    assert torch.equal(outs[0][2], outs[1][2])
    assert torch.equal(outs[0][3], outs[1][3])


@pytest.mark.parametrize("m,n,kappa", [(300, 300, 1e12), (420, 250, 1e10), (129, 129, 1e16)])
def test_polar_dev_matches_bounds_then_pzolopd1(m, n, kappa):
    """zolo_polar_dev (bounds + Zolo-PD + H sharing the QR of A/alpha) against the two
    separate calls: same alpha, beta and branch sequence, the same iterate to rounding."""
    import torch
    s = np.geomspace(1.0, 1.0 / kappa, n)
    a, _, _ = zo.make_matrix(n, s, 600 + m + n, m=m)
    h = zb.Handle(0)
    da = zb.colmajor_to_device(a)
    dq0, dq1 = torch.zeros_like(da), torch.zeros_like(da)
    dh0 = torch.zeros((n, n), dtype=torch.float64, device="cuda")
    dh1 = torch.zeros_like(dh0)
    torch.cuda.synchronize()
    al, be, _ = zb.bounds_dev(h, m, n, da.data_ptr(), m, mode=1)
    zb.pzolopd1_dev(h, "N", 8, m, n, al, be, da.data_ptr(), m, dq0.data_ptr(), m, dh0.data_ptr(), n)
    st0 = h.stats()
    assert zb.polar_dev(h, 8, m, n, da.data_ptr(), m, dq1.data_ptr(), m, dh1.data_ptr(), n) == 0
    st1 = h.stats()
    h.close()
    assert st1["alpha"] == al and st1["beta"] == be
    assert st1["branches"] == st0["branches"] and st1["branches"][0] == "QR"
    q0, q1 = zb.device_to_colmajor(dq0), zb.device_to_colmajor(dq1)
    check_pd(a, q1, zb.device_to_colmajor(dh1), n)
    assert np.linalg.norm(q1 - q0) / math.sqrt(n) <= max(1e-12, 10 * n * EPS * kappa)


def test_set_option_rejects_unknown():
    h = zb.Handle(0)
    with pytest.raises(zb.ZoloError):
        h.set_option(99, 1)
    h.close()


def test_zolopd_symmetric_vs_oracle():
    rng = np.random.default_rng(9)
    n = 60
    v = zo.haar(n, rng)
    lam = np.concatenate([-np.geomspace(1, 1e-6, 25), np.geomspace(1e-5, 1, 35)])
    a = (v * lam) @ v.T
    a = 0.5 * (a + a.T)
    q, h, info = zb.zolopd(a)
    assert info == 0
    q_o, h_o, st_o = zo.zolopd(a)
    # ZOLOPD stops once ||X_k+1 - X_k||_F <= (5 eps)^(1/3); on this symmetric indefinite
    # matrix the oracle itself ends at orthogonality ~1e-12, so the GPU is held to the oracle's level
    assert zo.backward_error(a, q, h) <= tol_n(n)
    assert zo.orthogonality(q) <= max(tol_n(n), 4 * zo.orthogonality(q_o))
    assert np.linalg.norm(q - q_o) / math.sqrt(n) <= 1e-8
    # symmetric input: polar factor is the matrix sign
    assert np.allclose(q, q.T, atol=1e-12)


def test_pqdwhfacs_shift_sigma():
    rng = np.random.default_rng(10)
    n = 50
    v = zo.haar(n, rng)
    lam = np.linspace(-2, 3, n)
    a = (v * lam) @ v.T
    a = 0.5 * (a + a.T)
    sigma = 0.37
    q, h, info = zb.pqdwhfacs("S", a, sigma=sigma)
    assert info == 0
    q_o, _, _ = zo.pqdwhfacs("S", a, sigma=sigma, bounds="qr")
    assert np.linalg.norm(q - q_o) <= 1e-10
    # sign(A - sigma I): eigenvalues +-1 with the split at sigma
    ev = np.linalg.eigvalsh(0.5 * (q + q.T))
    assert (ev < 0).sum() == (lam < sigma).sum()


def test_known_answer_fixtures():
    d = dict(np.load(os.path.join(GOLD, "known_polar.npz")))
    for tag, kappa in [("k7", 1e4), ("k33", 1e8), ("k64", 1e12)]:
        a = d[f"{tag}_a"]
        n = a.shape[1]
        q, h, info = zb.pqdwhfacs("N", a)
        assert info == 0
        check_pd(a, q, h, n)
        assert np.linalg.norm(q - d[f"{tag}_up"]) / math.sqrt(n) <= 100 * EPS * kappa * n
        ev = np.sort(np.linalg.eigvalsh(h))[::-1]
        assert np.max(np.abs(ev - d[f"{tag}_s"])) <= 1e-12
        al, be = d[f"{tag}_zolo4_ab"]
        qz, info = zb.pzolopd1("N", 4, a, al, be)
        assert info == 0
        assert np.allclose(qz, d[f"{tag}_zolo4_q"], atol=max(1e-12, 100 * n * EPS * kappa))


@pytest.mark.parametrize("m,n", [(96, 64), (150, 33), (257, 130)])
def test_rectangular_dev(m, n):
    import torch
    s = np.geomspace(1.0, 1e-8, n)
    a, u, v = zo.make_matrix(n, s, m + n, m=m)
    h = zb.Handle(0)
    da = zb.colmajor_to_device(a)
    dq = torch.zeros_like(da)
    dh = torch.zeros((n, n), dtype=torch.float64, device="cuda")
    zb.qdwh_dev(h, "N", m, n, 0.0, da.data_ptr(), m, dq.data_ptr(), m, dh.data_ptr(), n, 0, 12, 0)
    q = zb.device_to_colmajor(dq)
    hh = zb.device_to_colmajor(dh)
    check_pd(a, q, hh, n)
    assert np.linalg.norm(q - u @ v.T) / math.sqrt(n) <= 100 * n * EPS * 1e8
    # Zolo-PD on the rectangular matrix
    al, be, _ = zb.bounds_dev(h, m, n, da.data_ptr(), m, mode=1)
    zb.pzolopd1_dev(h, "N", 3, m, n, al, be, da.data_ptr(), m, dq.data_ptr(), m, dh.data_ptr(), n)
    q = zb.device_to_colmajor(dq)
    check_pd(a, q, zb.device_to_colmajor(dh), n)
    h.close()


def test_quick_return_and_bad_input():
    q, h, info = zb.pqdwhfacs("N", np.zeros((0, 0)))
    assert info == 0
    a = np.ones((6, 6))
    a[2, 3] = np.nan
    q, h, info = zb.pqdwhfacs("N", a)
    assert info > 0  # non-finite input: the bound estimate fails, nothing aborts
    q, h, info = zb.pqdwhfacs("N", np.zeros((5, 5)))
    assert info > 0  # zero matrix: ALPHA = 0


def test_bounds_dev_matches_oracle():
    n = 120
    s = np.geomspace(1, 1e-9, n)
    a, _, _ = zo.make_matrix(n, s, 77)
    h = zb.Handle(0)
    da = zb.colmajor_to_device(a)
    al, be, info = zb.bounds_dev(h, n, n, da.data_ptr(), n, mode=1)
    assert info == 0
    assert abs(al - np.linalg.norm(a)) <= 1e-14 * al
    be_o, _ = zo.bounds_qr_condest(a / al)
    # ||R^{-1}||_1 of an R with condition 1e9 is determined to ~kappa*eps relative
    assert abs(be - be_o) <= 1e-5 * be_o
    assert be <= s[-1] / al * (1 + 1e-8)  # a true lower bound on sigma_min(A/alpha)
    h.close()


@pytest.mark.parametrize("m,n,kappa", [(120, 120, 1e9), (300, 200, 1e14), (257, 257, 1e3)])
def test_bounds_frobenius_mode(m, n, kappa):
    """Mode 2: beta = 1/||R^{-1}||_F, a lower bound on sigma_min(A/alpha) that is never below
    mode 1's 1/(sqrt(n) ||R^{-1}||_1); a bad mode is rejected."""
    s = np.geomspace(1, 1.0 / kappa, n)
    a, _, _ = zo.make_matrix(n, s, 78 + m, m=m)
    h = zb.Handle(0)
    da = zb.colmajor_to_device(a)
    al, be1, _ = zb.bounds_dev(h, m, n, da.data_ptr(), m, mode=1)
    al2, be2, info = zb.bounds_dev(h, m, n, da.data_ptr(), m, mode=2)
    assert info == 0 and al2 == al
    r = np.linalg.qr(a / al, mode="r")
    ref = 1.0 / np.linalg.norm(np.linalg.inv(r))
    assert abs(be2 - ref) <= max(1e-10, 100 * n * EPS * kappa) * ref
    assert be1 * (1 - 1e-8) <= be2 <= s[-1] / al * (1 + 1e-8)
    with pytest.raises(zb.ZoloError):
        zb.bounds_dev(h, m, n, da.data_ptr(), m, mode=4)
    h.close()


@pytest.mark.parametrize("m,n,kappa", [(300, 300, 1e12), (400, 260, 1e15), (129, 129, 1e6)])
def test_polar_dev_frobenius_beta(m, n, kappa):
    """zolo_polar_dev with ZOLO_OPT_BETA_FROB: beta from mode 2, no more iterations than with
    the reference driver's beta, and the same polar factor (10 n eps; Q within kappa eps)."""
    import torch
    s = np.geomspace(1.0, 1.0 / kappa, n)
    a, u, v = zo.make_matrix(n, s, 650 + m + n, m=m)
    h = zb.Handle(0)
    da = zb.colmajor_to_device(a)
    out = {}
    for frob in (0, 1):
        h.set_option(zb.OPT_BETA_FROB, frob)
        dq = torch.zeros_like(da)
        dh = torch.zeros((n, n), dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        assert zb.polar_dev(h, 8, m, n, da.data_ptr(), m, dq.data_ptr(), m, dh.data_ptr(), n) == 0
        out[frob] = (zb.device_to_colmajor(dq), zb.device_to_colmajor(dh), h.stats())
    _, be2, _ = zb.bounds_dev(h, m, n, da.data_ptr(), m, mode=2)
    h.set_option(zb.OPT_BETA_FROB, 0)
    h.close()
    (q0, h0, st0), (q1, h1, st1) = out[0], out[1]
    assert st1["beta"] == be2 and st1["beta"] >= st0["beta"]
    assert st1["iterations"] <= st0["iterations"]
    check_pd(a, q1, h1, n)
    assert np.linalg.norm(q1 - q0) / math.sqrt(n) <= max(1e-12, 10 * n * EPS * kappa)
    assert np.linalg.norm(q1 - u @ v.T) / math.sqrt(n) <= max(1e-12, 100 * n * EPS * kappa)


@pytest.mark.parametrize("m,n,kappa", [(300, 300, 1e12), (420, 250, 1e8), (129, 129, 1e16), (500, 500, 1e3),
                                        (256, 256, 1e14), (200, 200, 1.0)])
@pytest.mark.parametrize("plan", [0, 1])
def test_fast_form_all_options(m, n, kappa, plan):
    """All cost options together (shared QR, explicit-inverse Cholesky, Frobenius beta, Newton-Schulz
    finish, and with `plan` the per-iteration term counts of the cost plan): backward stable
    (10 n eps, and below 1e-13), the same polar factor as the reference steps (Q within kappa eps),
    1..rk terms in every iteration (rk in every iteration without the plan)."""
    import torch
    s = np.geomspace(1.0, 1.0 / kappa, n)
    a, u, v = zo.make_matrix(n, s, 660 + m + n, m=m)
    h = zb.Handle(0)
    da = zb.colmajor_to_device(a)
    dq = torch.zeros_like(da)
    dh = torch.zeros((n, n), dtype=torch.float64, device="cuda")
    for opt in (zb.OPT_SHARED_QR, zb.OPT_NS_FINISH, zb.OPT_CHOL_INVERSE, zb.OPT_BETA_FROB):
        h.set_option(opt, 1)
    h.set_option(zb.OPT_TERM_PLAN, plan)
    torch.cuda.synchronize()
    assert zb.polar_dev(h, 8, m, n, da.data_ptr(), m, dq.data_ptr(), m, dh.data_ptr(), n) == 0
    st = h.stats()
    h.close()
    q, hh = zb.device_to_colmajor(dq), zb.device_to_colmajor(dh)
    check_pd(a, q, hh, n)
    assert zo.backward_error(a, q, hh) <= 1e-13
    assert np.linalg.norm(q - u @ v.T) / math.sqrt(n) <= max(1e-12, 100 * n * EPS * kappa)
    its = st["iterations"]
    assert len(st["terms"]) == its and all(1 <= t <= 8 for t in st["terms"])
    if not plan:
        assert all(t == 8 for t in st["terms"])


@pytest.mark.parametrize("m,n,kappa", [(330, 200, 1e12), (300, 300, 1e16), (257, 257, 1e4)])
def test_term_plan_through_pzolopd1(m, n, kappa):
    """The term plan on the PZOLOPD1 entry point (separate bounds, iterate not factored):
    backward stable, the same polar factor as the reference steps, 1..rk terms."""
    import torch
    s = np.geomspace(1.0, 1.0 / kappa, n)
    a, u, v = zo.make_matrix(n, s, 670 + m + n, m=m)
    h = zb.Handle(0)
    da = zb.colmajor_to_device(a)
    al, be, _ = zb.bounds_dev(h, m, n, da.data_ptr(), m, mode=2)
    for opt in (zb.OPT_NS_FINISH, zb.OPT_CHOL_INVERSE, zb.OPT_TERM_PLAN):
        h.set_option(opt, 1)
    dq = torch.zeros_like(da)
    dh = torch.zeros((n, n), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    assert zb.pzolopd1_dev(h, "N", 8, m, n, al, be, da.data_ptr(), m, dq.data_ptr(), m, dh.data_ptr(), n) == 0
    st = h.stats()
    h.close()
    q, hh = zb.device_to_colmajor(dq), zb.device_to_colmajor(dh)
    check_pd(a, q, hh, n)
    assert zo.backward_error(a, q, hh) <= 1e-13
    assert np.linalg.norm(q - u @ v.T) / math.sqrt(n) <= max(1e-12, 100 * n * EPS * kappa)
    assert all(1 <= t <= 8 for t in st["terms"])


@pytest.mark.parametrize("m,n", [(7, 5), (40, 33), (64, 64), (65, 65), (130, 1), (3, 3)])
def test_fast_form_small_sizes(m, n):
    """The fast form (factored iterate, term plan and the other cost options) at sizes below one
    64-column leaf or one 128-column block, and with dH = NULL: backward stable, orthogonal Q."""
    import torch
    s = np.geomspace(1.0, 1e-6, n)
    a, u, v = zo.make_matrix(n, s, 680 + m + n, m=m)
    h = zb.Handle(0)
    for opt in (zb.OPT_SHARED_QR, zb.OPT_NS_FINISH, zb.OPT_CHOL_INVERSE, zb.OPT_BETA_FROB, zb.OPT_TERM_PLAN):
        h.set_option(opt, 1)
    da = zb.colmajor_to_device(a)
    dq = torch.zeros_like(da)
    dh = torch.zeros((n, n), dtype=torch.float64, device="cuda")
    dq2 = torch.zeros_like(da)
    torch.cuda.synchronize()
    assert zb.polar_dev(h, 8, m, n, da.data_ptr(), m, dq.data_ptr(), m, dh.data_ptr(), n) == 0
    assert zb.polar_dev(h, 8, m, n, da.data_ptr(), m, dq2.data_ptr(), m, 0, 1) == 0  # no H
    h.close()
    q, hh, q2 = zb.device_to_colmajor(dq), zb.device_to_colmajor(dh), zb.device_to_colmajor(dq2)
    check_pd(a, q, hh, n)
    np.testing.assert_array_equal(q, q2)
    assert np.linalg.norm(q - u @ v.T) / math.sqrt(n) <= max(1e-12, 100 * n * EPS * 1e6)


def _run_polar(h, a, m, n, fast, inject=0, qdwh=False):
    import torch
    da = zb.colmajor_to_device(a)
    dq = torch.zeros_like(da)
    dh = torch.zeros((n, n), dtype=torch.float64, device="cuda")
    for opt in (zb.OPT_SHARED_QR, zb.OPT_NS_FINISH, zb.OPT_CHOL_INVERSE, zb.OPT_BETA_FROB, zb.OPT_TERM_PLAN):
        h.set_option(opt, 1 if fast else (1 if opt == zb.OPT_SHARED_QR else 0))
    h.set_option(zb.OPT_INJECT_CHOL_FAIL, inject)
    torch.cuda.synchronize()
    if qdwh:
        info = zb.qdwh_dev(h, "N", m, n, 0.0, da.data_ptr(), m, dq.data_ptr(), m, dh.data_ptr(), n, 0, 12, 0)
    elif fast:
        info = zb.polar_dev(h, 8, m, n, da.data_ptr(), m, dq.data_ptr(), m, dh.data_ptr(), n)
    else:
        al, be, _ = zb.bounds_dev(h, m, n, da.data_ptr(), m, mode=1)  # the driver's estimate, QR form
        info = zb.pzolopd1_dev(h, "N", 8, m, n, al, be, da.data_ptr(), m, dq.data_ptr(), m, dh.data_ptr(), n)
    h.set_option(zb.OPT_INJECT_CHOL_FAIL, 0)
    return info, zb.device_to_colmajor(dq), zb.device_to_colmajor(dh), h.stats()


@pytest.mark.parametrize("path", ["zolo_fast", "zolo_reference_rule", "qdwh"])
def test_cholesky_failure_recovers_with_qr_form(path):
    """A Cholesky-form step whose shifted Gram is reported not positive definite (host-side
    injection, ZOLO_OPT_INJECT_CHOL_FAIL) is redone in the QR form: INFO recorded in the stats,
    that iteration's branch is QR, and the result keeps the 10 n eps accuracy."""
    m, n, kappa = 300, 260, 1e8
    a, u, v = zo.make_matrix(n, np.geomspace(1.0, 1.0 / kappa, n), 910, m=m)
    h = zb.Handle(0)
    fast, qdwh = path == "zolo_fast", path == "qdwh"
    info0, q0, h0, st0 = _run_polar(h, a, m, n, fast, 0, qdwh)
    assert info0 == 0 and st0["info"] == 0
    k = st0["branches"].index("CH")  # first Cholesky-form iteration
    info1, q1, h1, st1 = _run_polar(h, a, m, n, fast, k + 1, qdwh)
    h.close()
    assert info1 == 0  # the solve completes; the factorization failure is reported in the stats
    assert st1["info"] == 1000000
    assert st1["branches"][k] == "QR" and st1["branches"][:k] == st0["branches"][:k]
    check_pd(a, q1, h1, n)
    assert np.linalg.norm(q1 - q0) / math.sqrt(n) <= 100 * n * EPS * kappa


def test_matrixmarket_symmetric_through_pqdwhfacs(tmp_path):
    """The reference's MatrixMarket driver flow (prepare_real_GEM, then PQDWHFACS with SYM = 'S'
    and a shift, pqdwh_fall.f90:189-207): a symmetric coordinate file read by zolo_read_mm and
    factored through the host-array entry point, against the oracle on the same matrix."""
    import scipy.io
    import scipy.sparse
    n = 240
    rng = np.random.default_rng(12)
    a = scipy.sparse.random(n, n, density=0.05, random_state=5, format="coo")
    a.data = rng.standard_normal(a.nnz)
    a = (a + a.T + scipy.sparse.diags(rng.uniform(0.5, 2.0, n))).tocoo()
    p = os.path.join(str(tmp_path), "sym.mtx")
    scipy.io.mmwrite(p, a, symmetry="symmetric")
    dense, kind = zb.read_mm(p)
    assert kind == "symmetric" and np.array_equal(dense, dense.T)
    sigma = float(np.median(np.diag(dense)))
    q, h, info = zb.pqdwhfacs("S", dense, sigma=sigma, polar="T")
    assert info == 0
    shifted = dense - sigma * np.eye(n)
    # H = sym(Q^T A) of the unshifted A (pqdwhfacs.f90:460-464), so the polar factor of A - sigma I
    # is Q with H - sigma sym(Q)
    check_pd(shifted, q, h - sigma * 0.5 * (q + q.T), n)
    q_o, h_o, st_o = zo.pqdwhfacs("S", dense, sigma=sigma, polar="T")
    ev = np.abs(np.linalg.eigvalsh(shifted))
    kappa = ev.max() / ev.min()
    assert np.linalg.norm(q - q_o) / math.sqrt(n) <= max(1e-12, 100 * n * EPS * kappa)


def _config_spectra(n, rng):
    """The five configurations' singular-value shapes at order n (kappa as configured)."""
    c1 = np.geomspace(1.0, 1e-8, n)
    c2 = np.geomspace(1.0, 1e-16, n)
    idx = rng.choice(np.arange(1, n), n // 20, replace=False)
    c2[idx] = c2[idx - 1]
    e = rng.uniform(-12, 0, n)
    e[0], e[-1] = 0.0, -12.0
    c3 = np.sort(10.0 ** e)[::-1]
    c4 = np.geomspace(1.0, 1.0 / 10 ** rng.uniform(2, 14), n)
    n70, n20 = int(0.7 * n), int(0.2 * n)
    base = np.geomspace(1e-1, 1e-9, (n - n70 - n20) // 8 + 1)
    clus = (base[:, None] * (1 + 1e-9 * np.arange(8))[None, :]).reshape(-1)[: n - n70 - n20]
    c5 = np.sort(np.concatenate([np.geomspace(1.0, 1e-10, n70), np.ones(n20), clus]))[::-1]
    return {"c1": c1, "c2": np.sort(c2)[::-1], "c3": c3, "c4": c4, "c5": c5}


@pytest.mark.parametrize("cfg", ["c1", "c2", "c3", "c4", "c5"])
def test_norm2_upper_bound_on_config_spectra(cfg):
    """zolo_bounds_dev mode 3: alpha >= sigma_max(A) (a guaranteed bound, within a 16-th root
    of the spectrum's weight of it, and never above ||A||_F), beta * alpha <= sigma_min(A); the
    Zolo-PD solve with ZOLO_OPT_NORM2_BOUND takes the smaller CON and stays backward stable."""
    import torch
    n = 640
    rng = np.random.default_rng(hash(cfg) % 1000)
    s = _config_spectra(n, rng)[cfg] * 3.7  # not normalized: sigma_max = 3.7
    a, u, v = zo.make_matrix(n, s, 3100 + int(cfg[1]))
    h = zb.Handle(0)
    da = zb.colmajor_to_device(a)
    torch.cuda.synchronize()
    al3, be3, _ = zb.bounds_dev(h, n, n, da.data_ptr(), n, mode=3)
    al2, be2, _ = zb.bounds_dev(h, n, n, da.data_ptr(), n, mode=2)
    smax, smin = s.max(), s.min()
    assert al3 >= smax and al3 <= al2 * (1 + 1e-12)
    assert al3 <= smax * n ** (1.0 / 16.0) * 1.001
    assert be3 * al3 <= smin * (1 + 1e-9) and abs(be3 * al3 - be2 * al2) <= 1e-9 * be2 * al2
    dq = torch.zeros_like(da)
    dh = torch.zeros_like(da)
    for opt in (zb.OPT_SHARED_QR, zb.OPT_NS_FINISH, zb.OPT_CHOL_INVERSE, zb.OPT_BETA_FROB, zb.OPT_TERM_PLAN):
        h.set_option(opt, 1)
    cons = []
    for norm2 in (0, 1):
        h.set_option(zb.OPT_NORM2_BOUND, norm2)
        assert zb.polar_dev(h, 8, n, n, da.data_ptr(), n, dq.data_ptr(), n, dh.data_ptr(), n) == 0
        st = h.stats()
        cons.append(st["con"][0] if "con" in st else None)
        q, hh = zb.device_to_colmajor(dq), zb.device_to_colmajor(dh)
        check_pd(a, q, hh, n)
    h.close()
    if cons[0] is not None:
        assert cons[1] <= cons[0] * (1 + 1e-12)


def test_sharded_driver_device_backend_matches_pzolopd1():
    """The r-term sharded driver (sharded.py) on one GPU with the library's per-term kernels
    (one rank, so no all-reduce): the reference's iteration, the same branch sequence and
    polar factor as zolo_pzolopd1_dev with per-term stacked QRs."""
    import importlib
    import torch
    sh = importlib.import_module("zolo_svd_b200.sharded")
    m, n, kappa = 260, 200, 1e10
    a, u, v = zo.make_matrix(n, np.geomspace(1.0, 1.0 / kappa, n), 777, m=m)
    h = zb.Handle(0)
    h.set_option(zb.OPT_SHARED_QR, 0)
    da = zb.colmajor_to_device(a)
    torch.cuda.synchronize()
    al, be, _ = zb.bounds_dev(h, m, n, da.data_ptr(), m, mode=1)
    dq = torch.zeros_like(da)
    assert zb.pzolopd1_dev(h, "N", 8, m, n, al, be, da.data_ptr(), m, dq.data_ptr(), m) == 0
    st = h.stats()
    x = da.clone()
    it, branches, info = sh.pzolopd1_sharded("N", 8, m, n, al, be, x, sh.DeviceBackend(h))
    h.close()
    assert info == 0 and it == st["iterations"] and branches == st["branches"]
    q1, q2 = zb.device_to_colmajor(dq), zb.device_to_colmajor(x)
    assert np.linalg.norm(q1 - q2) / math.sqrt(n) <= 100 * n * EPS * kappa
    assert zo.orthogonality(q2) <= tol_n(n)
