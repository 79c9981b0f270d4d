"""The mixed form (ZOLO_OPT_MIXED = 1): the large products of the Cholesky-form
iterations, of the Newton-Schulz finish and of Q and H run on the INT8 tensor
cores (FP64 emulated from 8 digit planes), the bounds and the QR-form iterations
on the FP64 tensor path.  Checked through the C-ABI against the FP64 form on the
same matrices and against the prescribed singular values:

  backward error ||A - QH||_F/||A||_F and orthogonality ||Q^T Q - I||_F/sqrt(n)
  <= min(10 n eps, 1e-13) (the mixed form's accuracy target), eigenvalues of H
  within 1e-12 sigma_max, the polar factor within 100 n eps kappa of the FP64
  form's, and the emulated GEMM actually launched (profiler class "ozgemm").
"""
import math

import numpy as np
import pytest

import zolo_svd_b200 as zb
from oracle import zolo_oracle as zo

pytestmark = pytest.mark.gpu
EPS = zo.EPS
FAST = ((zb.OPT_SHARED_QR, 1), (zb.OPT_NS_FINISH, 1), (zb.OPT_CHOL_INVERSE, 1), (zb.OPT_BETA_FROB, 1),
        (zb.OPT_TERM_PLAN, 1))


@pytest.fixture(scope="module")
def h():
    hd = zb.Handle(0)
    yield hd
    hd.close()


def _matrix(torch, m, n, kappa, seed):
    g = torch.Generator(device="cuda")
    g.manual_seed(seed)

    def haar(r, c):
        q, rr = torch.linalg.qr(torch.randn(r, c, dtype=torch.float64, device="cuda", generator=g))
        return q * torch.sign(torch.diagonal(rr))[None, :]
    u, v = haar(m, n), haar(n, n)
    e = torch.rand(n, dtype=torch.float64, device="cuda", generator=g) * -math.log10(kappa)
    e[0], e[-1] = 0.0, -math.log10(kappa)
    s = torch.sort(10.0 ** e, descending=True).values
    a = (u * s[None, :]) @ v.T
    return a, a.T.contiguous(), s


def _solve(h, torch, da, m, n, mixed, qdwh=False):
    for opt, val in FAST:
        h.set_option(opt, val)
    h.set_option(zb.OPT_MIXED, mixed)
    dq = torch.empty_like(da)
    dh = torch.empty((n, n), dtype=torch.float64, device="cuda")
    h.profile(True)
    h.profile_read(reset=True)
    if qdwh:
        zb.qdwh_dev(h, "N", m, n, 0.0, da.data_ptr(), m, dq.data_ptr(), m, dh.data_ptr(), n, 0, 12, 0)
    else:
        zb.polar_dev(h, 8, m, n, da.data_ptr(), m, dq.data_ptr(), m, dh.data_ptr(), n)
    torch.cuda.synchronize()
    prof = h.profile_read(reset=True)
    h.profile(False)
    h.set_option(zb.OPT_MIXED, 0)
    return dq.T, dh.T, prof, h.stats()


def _check(torch, a, q, hh, s, n):
    tol = min(10 * n * EPS, 1e-13)
    be = float(torch.linalg.norm(a - q @ hh) / torch.linalg.norm(a))
    orth = float(torch.linalg.norm(q.T @ q - torch.eye(n, dtype=torch.float64, device="cuda")) / math.sqrt(n))
    assert be <= tol, be
    assert orth <= tol, orth
    ev = torch.sort(torch.linalg.eigvalsh(0.5 * (hh + hh.T)), descending=True).values
    assert float(torch.max(torch.abs(ev - s))) <= 1e-12 * float(s[0])


@pytest.mark.parametrize("m,n,kappa", [(2048, 2048, 1e12), (3000, 2000, 1e8), (2560, 2560, 1e16)])
def test_mixed_zolo_polar(h, m, n, kappa):
    import torch
    a, da, s = _matrix(torch, m, n, kappa, 1700 + n)
    q1, h1, p1, st1 = _solve(h, torch, da, m, n, 1)
    assert p1["ozgemm"]["launches"] > 0  # the emulated products ran
    _check(torch, a, q1, h1, s, n)
    q0, h0, p0, st0 = _solve(h, torch, da, m, n, 0)
    assert p0["ozgemm"]["launches"] == 0
    _check(torch, a, q0, h0, s, n)
    assert st1["branches"][0] == st0["branches"][0] == "QR"  # the QR phase is the FP64 one in both
    dq = float(torch.linalg.norm(q1 - q0)) / math.sqrt(n)
    assert dq <= 100 * n * EPS * kappa or dq <= 1e-12


def test_mixed_qdwh(h):
    import torch
    n = 2048
    a, da, s = _matrix(torch, n, n, 1e8, 1901)
    q1, h1, p1, st1 = _solve(h, torch, da, n, n, 1, qdwh=True)
    assert p1["ozgemm"]["launches"] > 0
    _check(torch, a, q1, h1, s, n)
    q0, h0, _, st0 = _solve(h, torch, da, n, n, 0, qdwh=True)
    assert st1["branches"] == st0["branches"]
    assert float(torch.linalg.norm(q1 - q0)) / math.sqrt(n) <= 100 * n * EPS * 1e8


def test_mixed_option_values(h):
    with pytest.raises(zb.ZoloError):
        h.set_option(zb.OPT_MIXED, 2)
    with pytest.raises(zb.ZoloError):
        h.set_option(zb.OPT_MIXED_SLICES, 9)
    h.set_option(zb.OPT_MIXED_SLICES, 8)
