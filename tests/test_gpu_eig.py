"""Eigen stage and Zolo-SVD on the GPU through the C-ABI: the spectral
divide-and-conquer eigensolver with Jacobi leaves (replacing ELPA,
elpa_pdsyevd2.F90:199-200), ZoloEig (ZoloEig.f90:78-102) and the SVD assembly of
ZoloCHK1.f90:80-91, against LAPACK dsyevd / the oracle on seeded inputs.
Tolerances: eigenvalues / singular values within 1e-12 of sigma_max (the
target's singular-value bound); residual ||HZ - Z diag(w)||_F / ||H||_F and
orthogonality ||Z^T Z - I||_F / sqrt(n) within 10*n*eps (floored at 1e-14)."""
import math

import numpy as np
import pytest
import scipy.linalg as sla

import zolo_svd_b200 as zb
from oracle import zolo_oracle as zo

pytestmark = pytest.mark.gpu
EPS = zo.EPS


def tol_n(n):
    return max(10 * n * EPS, 1e-14)


@pytest.fixture(scope="module")
def h():
    hd = zb.Handle(0)
    yield hd
    hd.close()


def _syev(h, a):
    import torch
    n = a.shape[0]
    da = zb.colmajor_to_device(a)
    dw = torch.zeros(max(n, 1), dtype=torch.float64, device="cuda")
    dz = torch.zeros_like(da)
    torch.cuda.synchronize()
    zb.syev_dev(h, n, da.data_ptr(), n, dw.data_ptr(), dz.data_ptr(), n)
    return dw.cpu().numpy()[:n], zb.device_to_colmajor(dz)


def _sym_with_spectrum(n, lam, seed):
    q = zo.haar(n, np.random.default_rng(seed))
    a = (q * lam[None, :]) @ q.T
    return 0.5 * (a + a.T)


@pytest.mark.parametrize("n", [1, 5, 33, 64, 65, 100, 200, 301])
def test_syev_vs_lapack(h, n):
    rng = np.random.default_rng(n)
    x = rng.standard_normal((n, n))
    a = 0.5 * (x + x.T)
    w, z = _syev(h, a)
    w_ref = sla.eigh(a, eigvals_only=True, driver="evd")
    nrm = np.linalg.norm(a, 2)
    assert np.max(np.abs(w - w_ref)) <= 1e-12 * nrm
    assert np.all(np.diff(w) >= 0)  # ascending, like dsyevd
    res = np.linalg.norm(a @ z - z * w[None, :]) / np.linalg.norm(a)
    assert res <= tol_n(n)
    assert np.linalg.norm(z.T @ z - np.eye(n)) / math.sqrt(n) <= tol_n(n)


@pytest.mark.parametrize("zolo_min", [0, 96])
@pytest.mark.parametrize("n", [150, 301])
def test_syev_split_polar_forms(n, zolo_min):
    """ZOLO_OPT_EIG_ZOLO_MIN: with 0 every node splits on QDWH polar factors (a level's nodes
    in one batched solve); with 96 the nodes of at least 96 rows split on Zolo-PD's (fast
    form) and the smaller ones on batched QDWH.  Both agree with LAPACK dsyevd; the split
    statistics show which solvers ran."""
    hd = zb.Handle(0)
    hd.set_option(zb.OPT_EIG_ZOLO_MIN, zolo_min)
    rng = np.random.default_rng(1000 + n)
    # a spectrum symmetric about 0, so that the median shifts split the nodes in halves
    lam = np.sort(np.concatenate([np.linspace(-1.0, 1.0, n - 8), rng.uniform(-1e-3, 1e-3, 8)]))
    a = _sym_with_spectrum(n, lam, 40 + n)
    w, z = _syev(hd, a)
    st = hd.stats()
    qdwh_calls, zolo_calls, batched = st["terms"][:3]
    if zolo_min == 0:
        assert zolo_calls == 0 and qdwh_calls >= st["iterations"]
    else:
        assert zolo_calls >= 1  # the root (n >= 96) at least
    assert batched >= 2
    assert np.max(np.abs(w - np.sort(lam))) <= 1e-12
    assert np.linalg.norm(a @ z - z * w[None, :]) / np.linalg.norm(a) <= tol_n(n)
    assert np.linalg.norm(z.T @ z - np.eye(n)) / math.sqrt(n) <= tol_n(n)
    hd.close()


def test_syev_clustered_spd_spectrum(h):
    """SPD H with 20% of the eigenvalues exactly 1 and tight clusters (relative gap 1e-9),
    the eigen-stage stress case of the full SVD workload, scaled down."""
    n = 240
    rng = np.random.default_rng(5)
    lam = np.geomspace(1.0, 1e-10, n)
    lam[: n // 5] = 1.0
    for c0 in range(n // 5, n // 5 + 24, 6):
        lam[c0:c0 + 6] = lam[c0] * (1 + 1e-9 * np.arange(6))
    a = _sym_with_spectrum(n, lam, 6)
    w, z = _syev(h, a)
    assert np.max(np.abs(w - np.sort(lam))) <= 1e-12
    assert np.linalg.norm(a @ z - z * w[None, :]) / np.linalg.norm(a) <= tol_n(n)
    assert np.linalg.norm(z.T @ z - np.eye(n)) / math.sqrt(n) <= tol_n(n)


@pytest.mark.parametrize("algo", [0, 1])
@pytest.mark.parametrize("m,n,kappa", [(96, 96, 1e8), (150, 100, 1e10), (260, 130, 1e12)])
def test_svd_known_singular_values(h, algo, m, n, kappa):
    import torch
    s = np.geomspace(1.0, 1.0 / kappa, n)
    a, u, v = zo.make_matrix(n, s, 300 + m + n, m=m)
    da = zb.colmajor_to_device(a)
    du = torch.zeros_like(da)
    ds = torch.zeros(n, dtype=torch.float64, device="cuda")
    dv = torch.zeros((n, n), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    zb.svd_dev(h, m, n, da.data_ptr(), m, du.data_ptr(), m, ds.data_ptr(), dv.data_ptr(), n, algo=algo, rk=4)
    U = zb.device_to_colmajor(du)
    S = ds.cpu().numpy()
    V = zb.device_to_colmajor(dv)
    assert np.max(np.abs(S - np.sort(s))) <= 1e-12 * s[0]
    assert np.linalg.norm(a - (U * S[None, :]) @ V.T) / np.linalg.norm(a) <= tol_n(n)
    assert np.linalg.norm(U.T @ U - np.eye(n)) / math.sqrt(n) <= tol_n(n)
    assert np.linalg.norm(V.T @ V - np.eye(n)) / math.sqrt(n) <= tol_n(n)
    # the checks ZoloCHK1 prints: ||A V - U S||_F / sigma_max
    assert np.linalg.norm(a @ V - U * S[None, :]) / S.max() <= tol_n(n)


def test_zoloeig_vs_oracle():
    rng = np.random.default_rng(8)
    n = 90
    lam = np.concatenate([np.linspace(-2.0, -0.5, 37), np.linspace(0.25, 3.0, n - 37)])
    a = _sym_with_spectrum(n, lam, 9)
    q, _, info = zb.pqdwhfacs("S", a, sigma=0.0)
    assert info == 0
    w, vecs, V, E, info = zb.zoloeig(q, a)
    assert info == 0
    assert len(w) == 37
    assert np.max(np.abs(w - lam[:37])) <= 1e-12 * 3.0
    assert np.linalg.norm(a @ vecs - vecs * w[None, :]) / np.linalg.norm(a) <= tol_n(n)
    w_o, _, rk_o = zo.zoloeig(a, q, np.random.default_rng(1))
    assert rk_o == 37
    assert np.max(np.abs(np.sort(w_o) - w)) <= 1e-12 * 3.0
    # outputs as the reference leaves them: Q = V (orthogonal), As = V^T A V
    assert np.linalg.norm(V.T @ V - np.eye(n)) / math.sqrt(n) <= tol_n(n)
    assert np.allclose(E, V.T @ a @ V, atol=1e-12)
