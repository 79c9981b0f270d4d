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


def _close(xs, ys, rel):
    for x, y in zip(xs, ys):
        assert np.max(np.abs(x - y)) <= rel * max(1.0, np.max(np.abs(y)))


def test_batch_graph_matches_synchronized_loop():
    """ZOLO_OPT_BATCH_GRAPH: the scheduled run (issued eagerly on the first call of a bucket
    shape, captured as a graph on the second, the cached graph replayed on the third; or
    always eagerly with option value 2) takes the synchronized loop's steps: the same
    iteration counts and, to rounding, the same Q and H."""
    h = zb.Handle(0)
    mats = _members(3, 24, 5, 300)
    h.set_option(zb.OPT_BATCH_GRAPH, 0)
    info0, its0, q0, h0 = _run_batch(h, mats)
    st = zb.batch_stats(h)
    assert st["buckets"] > 1 and st["sync_loops"] == st["buckets"]
    h.set_option(zb.OPT_BATCH_GRAPH, 1)
    for call, key in enumerate(("eager_scheduled", "graph_captures", "graph_replays")):
        info, its, q, hh = _run_batch(h, mats)
        st = zb.batch_stats(h)
        assert st[key] == st["buckets"], (call, st)
        assert st["restarts"] == 0 and st["resumes"] == 0 and st["sync_loops"] == 0
        assert info == info0 and its == its0
        _close(q, q0, 1e-13)
        _close(hh, h0, 1e-13)
    h.set_option(zb.OPT_BATCH_GRAPH, 2)  # the schedule issued eagerly on every call
    info, its, q, hh = _run_batch(h, mats)
    st = zb.batch_stats(h)
    assert st["eager_scheduled"] == st["buckets"] and st["graph_replays"] == 0
    assert info == info0 and its == its0
    _close(q, q0, 1e-13)
    h.close()


@pytest.mark.parametrize("inject", ["cholesky", "error"])
def test_batch_graph_recovery_paths(inject):
    """The checks after a scheduled run, driven by host-side injection: a Cholesky step
    reported failed reruns its bucket through the synchronized loop (QR form at that step);
    a member whose last error is reported high continues there for one more step.  Both on
    the eager and on the captured run; every member stays accurate."""
    h = zb.Handle(0)
    mats = _members(4, 16, 20, 200)
    info0, its0, _, _ = _run_batch(h, mats)
    h.release()
    if inject == "cholesky":
        h.set_option(zb.OPT_INJECT_CHOL_FAIL, 4)  # the fourth step, a Cholesky-form one
    else:
        h.set_option(zb.OPT_INJECT_BATCH_ERR, 1)
    for call in range(2):
        info, its, qs, hs = _run_batch(h, mats)
        st = zb.batch_stats(h)
        assert st["eager_scheduled" if call == 0 else "graph_captures"] == st["buckets"]
        assert info == [0] * len(mats)
        if inject == "cholesky":
            assert st["restarts"] >= 1 and st["resumes"] == 0
        else:
            assert st["resumes"] == st["buckets"] and st["restarts"] == 0
            d = [b - a for a, b in zip(its0, its)]
            assert set(d) <= {0, 1} and sum(d) == st["buckets"], d
        for (a, uv, s, kappa), q, hh in zip(mats, qs, hs):
            n = a.shape[1]
            assert zo.backward_error(a, q, hh) <= tol_n(n)
            assert zo.orthogonality(q) <= tol_n(n)
            assert np.linalg.norm(q - uv) / math.sqrt(n) <= max(1e-12, 100 * n * EPS * kappa)
    h.set_option(zb.OPT_INJECT_CHOL_FAIL, 0)
    h.set_option(zb.OPT_INJECT_BATCH_ERR, 0)
    h.close()


def test_batch_autotune_model():
    """zolo_batch_autotune measures a cost model within the FP64 tensor path's range (latency
    terms >= 0, 0.5 < rate < 60 TF/s) whose plan solves a batch correctly and not much slower
    than the default model's plan."""
    import ctypes as C
    import time
    import torch
    h = zb.Handle(0)
    mats = _members(5, 48, 24, 400)
    tuned = (C.c_double * 5)()
    assert zb.lib().zolo_batch_autotune(h.ptr, tuned) == 0
    lat0, lat1, rate, nhalf, streams = list(tuned)
    assert lat0 >= 0 and lat1 >= 0 and 0.5 < rate < 60 and 0 <= nhalf < 8192 and streams >= 1
    times = {}
    for name, md in (("default", (4.0, 0.35, 25.0, 384.0, 8.0)), ("tuned", tuple(tuned))):
        assert zb.lib().zolo_batch_set_model(h.ptr, (C.c_double * 5)(*md)) == 0
        for _ in range(2):
            _run_batch(h, mats)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        info, its, qs, hs = _run_batch(h, mats)
        times[name] = time.perf_counter() - t0
        assert info == [0] * len(mats)
        for (a, uv, s, kappa), q, hh in zip(mats, qs, hs):
            n = a.shape[1]
            assert zo.backward_error(a, q, hh) <= tol_n(n) and zo.orthogonality(q) <= tol_n(n)
    assert times["tuned"] <= 1.6 * times["default"], times
    h.close()


def config4_members(seed=1004, count=512):
    """Configuration 4: n = round(exp U[ln 64, ln 1024]), m = round(n (1 + U[0, 1])),
    kappa = 10^U[2, 14], s geometric from 1 to 1/kappa; member i generated from PCG64 seed
    seed + i (Haar U m x n, V n x n)."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        n = int(round(math.exp(rng.uniform(math.log(64), math.log(1024)))))
        m = int(round(n * (1 + rng.uniform(0, 1))))
        kappa = 10 ** rng.uniform(2, 14)
        s = np.geomspace(1.0, 1.0 / kappa, n)
        a, u, v = zo.make_matrix(n, s, seed + i, m=m)
        out.append((a, u, v, s, kappa))
    return out


def test_batch_config4_full_size():
    """The 512-member configuration at full size in one call (run three times: eagerly, captured,
    replayed, with the same results): every member backward stable and
    orthogonal to 10 n eps, its singular values within 1e-12 sigma_max, its polar factor within
    100 n eps kappa of U V^T; a sample of members against the oracle's PQDWHFACS."""
    import torch
    h = zb.Handle(0)
    mats = config4_members()
    dev = [zb.colmajor_to_device(a) for a, *_ in mats]
    dq = [torch.zeros_like(d) for d in dev]
    dh = [torch.zeros((a.shape[1], a.shape[1]), dtype=torch.float64, device="cuda") for a, *_ in mats]
    torch.cuda.synchronize()
    members = [(a.shape[0], a.shape[1], d.data_ptr(), a.shape[0], q.data_ptr(), a.shape[0], hh.data_ptr(),
                a.shape[1]) for (a, *_), d, q, hh in zip(mats, dev, dq, dh)]
    # three calls: the schedule issued eagerly, captured as graphs, the graphs replayed
    first = None
    for key in ("eager_scheduled", "graph_captures", "graph_replays"):
        for q in dq:
            q.zero_()
        info, its = zb.qdwh_batch_dev(h, members)
        st = zb.batch_stats(h)
        assert st[key] == st["buckets"] and st["restarts"] == 0, st
        assert info == [0] * len(mats)
        if first is None:
            first = ([q.clone() for q in dq], its)
        else:
            assert its == first[1]
            assert max(float(torch.max(torch.abs(q - q1))) for q, q1 in zip(dq, first[0])) <= 1e-13
    worst = 0.0
    for k, ((a, u, v, s, kappa), q_d, h_d) in enumerate(zip(mats, dq, dh)):
        m, n = a.shape
        q, hh = zb.device_to_colmajor(q_d), zb.device_to_colmajor(h_d)
        be, orth = zo.backward_error(a, q, hh), zo.orthogonality(q)
        worst = max(worst, be / (10 * n * EPS), orth / (10 * n * EPS))
        assert be <= tol_n(n) and orth <= tol_n(n), (k, be, orth)
        ev = np.sort(np.linalg.eigvalsh(0.5 * (hh + hh.T)))[::-1]
        assert np.max(np.abs(ev - s)) <= 1e-12 * s[0], k
        assert np.linalg.norm(q - u @ v.T) / math.sqrt(n) <= max(1e-12, 100 * n * EPS * kappa), k
        if k % 64 == 0:  # a sample against the oracle on the same member
            q_o, h_o, st_o = zo.pqdwhfacs("N", a, bounds="qr")
            assert np.linalg.norm(q - q_o) / math.sqrt(n) <= max(1e-12, 100 * n * EPS * kappa), k
            assert abs(its[k] - st_o.iterations) <= 2, (k, its[k], st_o.iterations)  # padding shifts beta
    assert worst <= 1.0
    h.close()
