"""Batched QDWH-PD (zolo_qdwh_batch_dev) on the GPU: many matrices of different
sizes, shapes and conditioning in one call, each member checked against the
single-matrix PQDWHFACS path (zolo_qdwh_dev) on the same input and against its
known polar factor.  Tolerances per member: backward error and orthogonality
<= 10*n*eps (floored at 1e-14); eigenvalues of H within 1e-12 of sigma_max; Q
within max(1e-12, 100*n*eps*kappa) of U V^T."""
import math

import numpy as np
import pytest

import zolo_svd_b200 as zb
from oracle import zolo_oracle as zo

pytestmark = pytest.mark.gpu
EPS = zo.EPS


def tol_n(n):
    return max(10 * n * EPS, 1e-14)


def _members(seed, count, nmin, nmax):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        n = int(round(math.exp(rng.uniform(math.log(nmin), math.log(nmax)))))
        m = int(round(n * (1 + rng.uniform(0, 1)))) if i % 3 else n
        kappa = 10 ** rng.uniform(2, 12)
        s = np.geomspace(1.0, 1.0 / kappa, n) * 10 ** rng.uniform(-3, 3)  # members of very different scale
        a, u, v = zo.make_matrix(n, s, 7000 + seed + i, m=m)
        out.append((a, u @ v.T, s, kappa))
    return out


def _run_batch(h, mats):
    import torch
    dev = [zb.colmajor_to_device(a) for a, *_ in mats]
    dq = [torch.zeros_like(d) for d in dev]
    dh = [torch.zeros((a.shape[1], a.shape[1]), dtype=torch.float64, device="cuda") for a, *_ in mats]
    torch.cuda.synchronize()
    members = [(a.shape[0], a.shape[1], d.data_ptr(), a.shape[0], q.data_ptr(), a.shape[0], hh.data_ptr(),
                a.shape[1]) for (a, *_), d, q, hh in zip(mats, dev, dq, dh)]
    info, its = zb.qdwh_batch_dev(h, members)
    return info, its, [zb.device_to_colmajor(q) for q in dq], [zb.device_to_colmajor(x) for x in dh]


def test_batch_matches_single_and_known_polar():
    import torch
    h = zb.Handle(0)
    mats = _members(1, 24, 5, 300)
    info, its, qs, hs = _run_batch(h, mats)
    assert info == [0] * len(mats)
    for (a, uv, s, kappa), q, hh, it in zip(mats, qs, hs, its):
        m, n = a.shape
        assert 1 <= it <= 13
        assert zo.backward_error(a, q, hh) <= tol_n(n)
        assert zo.orthogonality(q) <= tol_n(n)
        ev = np.sort(np.linalg.eigvalsh(hh))[::-1]
        assert np.max(np.abs(ev - s)) <= 1e-12 * s[0]
        assert np.linalg.norm(q - uv) / math.sqrt(n) <= max(1e-12, 100 * n * EPS * kappa)
        # the single-matrix path on the same input
        da = zb.colmajor_to_device(a)
        dq1 = torch.zeros_like(da)
        torch.cuda.synchronize()
        zb.qdwh_dev(h, "N", m, n, 0.0, da.data_ptr(), m, dq1.data_ptr(), m, 0, 1, 0, 12, 0)
        q1 = zb.device_to_colmajor(dq1)
        assert np.linalg.norm(q - q1) / math.sqrt(n) <= max(1e-12, 100 * n * EPS * kappa)
    h.close()


def test_batch_bad_member_and_empty():
    """A zero matrix gets INFO > 0 (its bounds fail) and leaves the other members of
    its bucket exact; an empty batch is a no-op."""
    h = zb.Handle(0)
    mats = _members(2, 5, 40, 60)
    a0 = np.zeros((50, 50))
    mats.insert(2, (a0, np.eye(50), np.ones(50), 1.0))
    info, its, qs, hs = _run_batch(h, mats)
    assert info[2] > 0
    for k, ((a, uv, s, kappa), q, hh) in enumerate(zip(mats, qs, hs)):
        if k == 2:
            continue
        assert info[k] == 0
        assert zo.backward_error(a, q, hh) <= tol_n(a.shape[1])
        assert zo.orthogonality(q) <= tol_n(a.shape[1])
    assert zb.qdwh_batch_dev(h, []) == ([], [])
    h.close()
