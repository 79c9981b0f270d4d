"""Kernel-level parity on the GPU through the C-ABI: DMMA GEMM (all transposes,
triangle-only output, triangular-operand skip, split-K), recursive Cholesky and
triangular solves, the structured Householder QR / explicit Q, the ZOLOQR and
ZOLOCHOL terms and FormX2, each against LAPACK / the oracle on the same inputs.
FP64 tolerances are stated per test (multiples of k*eps relative to |A||B|)."""
import ctypes as C

import numpy as np
import pytest
import scipy.linalg as sla
from scipy.linalg import lapack

import zolo_svd_b200 as zb
from oracle import zolo_oracle as zo

pytestmark = pytest.mark.gpu
EPS = zo.EPS


@pytest.fixture(scope="module")
def h():
    import torch
    torch.cuda.init()
    hd = zb.Handle(0)
    yield hd
    hd.close()


def dev(a):
    import torch
    t = zb.colmajor_to_device(np.asarray(a, dtype=np.float64))
    torch.cuda.synchronize()
    return t


def host(t):
    import torch
    torch.cuda.synchronize()
    return zb.device_to_colmajor(t)


def empty(m, n):
    import torch
    return torch.zeros((n, m), dtype=torch.float64, device="cuda")


def op(a, t):
    return a.T if t == "T" else a


SHAPES = [(1, 1, 1), (7, 5, 3), (16, 8, 8), (128, 128, 16), (130, 129, 67), (257, 300, 513), (64, 1000, 33)]


@pytest.mark.parametrize("ta", ["N", "T"])
@pytest.mark.parametrize("tb", ["N", "T"])
@pytest.mark.parametrize("mnk", SHAPES)
def test_dgemm_vs_numpy(h, ta, tb, mnk):
    m, n, k = mnk
    rng = np.random.default_rng(m * 1000 + n + k)
    a = rng.standard_normal((k, m) if ta == "T" else (m, k))
    b = rng.standard_normal((n, k) if tb == "T" else (k, n))
    c0 = rng.standard_normal((m, n))
    alpha, beta = 1.25, -0.5
    da, db, dc = dev(a), dev(b), dev(c0)
    r = zb.lib().zolo_dgemm_dev(h.ptr, ta.encode(), tb.encode(), m, n, k, alpha, da.data_ptr(), a.shape[0],
                                db.data_ptr(), b.shape[0], beta, dc.data_ptr(), m, 0, 0)
    assert r == 0
    ref = alpha * op(a, ta) @ op(b, tb) + beta * c0
    bound = 2 * (k + 2) * EPS * (abs(alpha) * np.abs(op(a, ta)) @ np.abs(op(b, tb)) + abs(beta) * np.abs(c0))
    assert np.all(np.abs(host(dc) - ref) <= bound + 1e-300)


# rank-k updates C = beta*C + alpha*A*B with K <= 32 and M*N >= 16 * 128 * 32 take the
# persistent streaming kernel (update.cu): partial tiles, K < 8, odd M and K with
# 16-byte copies (even leading dimensions), odd leading dimensions and 8-byte-aligned
# (not 16) pointers (8-byte copies), beta = 0 (C not read) and beta = 1
@pytest.mark.parametrize("m,n,k,alpha,beta,off,pad", [
    (512, 512, 32, -1.0, 1.0, 0, 0), (1000, 700, 7, 0.5, 1.0, 1, 1), (300, 1200, 1, -1.0, 1.0, 0, 0),
    (129, 2049, 31, 1.0, 0.0, 1, 2), (4100, 70, 32, -1.0, 1.0, 0, 0), (777, 333, 16, 2.0, -0.5, 1, 1),
    (1001, 300, 31, -1.0, 1.0, 0, 1), (255, 1031, 17, -1.0, 1.0, 0, 1), (1026, 1000, 16, 1.5, 0.0, 0, 0),
    (2050, 520, 2, -1.0, 1.0, 0, 2)])
def test_dgemm_streaming_rank_update(h, m, n, k, alpha, beta, off, pad):
    import torch
    rng = np.random.default_rng(m + n + k)
    a = rng.standard_normal((m, k))
    b = rng.standard_normal((k, n))
    c0 = rng.standard_normal((m, n))
    lda, ldb, ldc = m + pad, k + pad, m + pad
    def padded(x, ld):
        buf = torch.zeros(x.shape[1] * ld + off, dtype=torch.float64, device="cuda")
        view = buf[off:off + x.shape[1] * ld].view(x.shape[1], ld)
        view[:, : x.shape[0]] = torch.from_numpy(np.ascontiguousarray(x.T)).cuda()
        return buf, view
    ba, va = padded(a, lda)
    bb, vb = padded(b, ldb)
    bc, vc = padded(c0, ldc)
    torch.cuda.synchronize()
    r = zb.lib().zolo_dgemm_dev(h.ptr, b"N", b"N", m, n, k, alpha, va.data_ptr(), lda, vb.data_ptr(), ldb, beta,
                                vc.data_ptr(), ldc, 0, 0)
    assert r == 0
    torch.cuda.synchronize()
    got = vc[:, :m].T.cpu().numpy()
    ref = alpha * a @ b + beta * c0
    bound = 2 * (k + 2) * EPS * (abs(alpha) * np.abs(a) @ np.abs(b) + abs(beta) * np.abs(c0))
    assert np.all(np.abs(got - ref) <= bound + 1e-300)
    # the padding rows of C (ldc > m) are untouched
    if pad:
        assert torch.count_nonzero(vc[:, m:]).item() == 0


def test_dgemm_lower_triangle_only(h):
    rng = np.random.default_rng(1)
    m, k = 300, 77
    x = rng.standard_normal((k, m))
    c0 = rng.standard_normal((m, m))
    dx, dc = dev(x), dev(c0)
    r = zb.lib().zolo_dgemm_dev(h.ptr, b"T", b"N", m, m, k, 1.0, dx.data_ptr(), k, dx.data_ptr(), k, 0.0,
                                dc.data_ptr(), m, 1, 0)
    assert r == 0
    got = host(dc)
    ref = x.T @ x
    il = np.tril_indices(m)
    iu = np.triu_indices(m, 1)
    assert np.allclose(got[il], ref[il], rtol=0, atol=4 * k * EPS * np.abs(x).max() ** 2 * 2)
    np.testing.assert_array_equal(got[iu], c0[iu])  # upper triangle untouched


def test_dgemm_triangular_operand_skip(h):
    """op(B) = Q2^T with Q2 upper triangular: the k < n part is skipped (Q1 Q2^T of zoloqr.f90:111)."""
    rng = np.random.default_rng(2)
    m, n = 190, 260
    q1 = rng.standard_normal((m, n))
    q2 = np.triu(rng.standard_normal((n, n)))
    d1, d2, dc = dev(q1), dev(q2), dev(np.zeros((m, n)))
    r = zb.lib().zolo_dgemm_dev(h.ptr, b"N", b"T", m, n, n, 1.0, d1.data_ptr(), m, d2.data_ptr(), n, 0.0,
                                dc.data_ptr(), m, 0, 1)
    assert r == 0
    ref = q1 @ q2.T
    assert np.allclose(host(dc), ref, rtol=0, atol=4 * n * EPS * (np.abs(q1) @ np.abs(q2.T)).max())


def test_dgemm_row_triangular_skip(h):
    """kfrom_n = 2: op(A) = Y^T with Y lower triangular, so row i of op(A) is zero for
    k < i; with a lower-triangle output this is Y^T Y of the explicit-inverse Cholesky form."""
    rng = np.random.default_rng(4)
    n = 333
    y = np.tril(rng.standard_normal((n, n)))
    c0 = rng.standard_normal((n, n))
    dy, dc = dev(y), dev(c0)
    r = zb.lib().zolo_dgemm_dev(h.ptr, b"T", b"N", n, n, n, -0.5, dy.data_ptr(), n, dy.data_ptr(), n, 0.0,
                                dc.data_ptr(), n, 1, 2)
    assert r == 0
    got = host(dc)
    ref = -0.5 * y.T @ y
    il, iu = np.tril_indices(n), np.triu_indices(n, 1)
    assert np.allclose(got[il], ref[il], rtol=0, atol=4 * n * EPS * (np.abs(y.T) @ np.abs(y)).max())
    np.testing.assert_array_equal(got[iu], c0[iu])


def test_dgemm_both_triangular_skip(h):
    """kfrom_n = 3: op(A) upper and op(B) lower triangular, so entry (i, j) sums k >= max(i, j)
    only (Q1 Q2^T of the shared-QR Zolotarev terms, both factors upper triangular)."""
    rng = np.random.default_rng(5)
    n = 301
    q1 = np.triu(rng.standard_normal((n, n)))
    q2 = np.triu(rng.standard_normal((n, n)))
    d1, d2, dc = dev(q1), dev(q2), dev(rng.standard_normal((n, n)))
    r = zb.lib().zolo_dgemm_dev(h.ptr, b"N", b"T", n, n, n, 2.0, d1.data_ptr(), n, d2.data_ptr(), n, 0.0,
                                dc.data_ptr(), n, 0, 3)
    assert r == 0
    ref = 2.0 * q1 @ q2.T
    assert np.allclose(host(dc), ref, rtol=0, atol=8 * n * EPS * (np.abs(q1) @ np.abs(q2.T)).max())


@pytest.mark.parametrize("n", [1, 40, 64, 65, 130, 300, 700])
def test_trtri_vs_numpy(h, n):
    """Y = L^{-1} by the recursive blocked inverse (diagonal 64-blocks inverted in one kernel,
    off-diagonal blocks Y21 = -Y22 L21 Y11 with both triangular skips); the upper triangle of
    the input is ignored and that of Y is zero.  Tolerance: forward error of a triangular
    inverse, <= c * n * eps * cond(L) relative to |L^{-1}|."""
    rng = np.random.default_rng(n + 11)
    x = rng.standard_normal((n + 3, n))
    l_true = np.linalg.cholesky(x.T @ x + n * np.eye(n))
    l_in = l_true + np.triu(rng.standard_normal((n, n)), 1)  # garbage above the diagonal
    dl, dy = dev(l_in), dev(rng.standard_normal((n, n)))
    assert zb.lib().zolo_dtrtri_dev(h.ptr, n, dl.data_ptr(), n, dy.data_ptr(), n) == 0
    got = host(dy)
    ref = np.linalg.inv(l_true)
    cond = np.linalg.cond(l_true)
    assert np.count_nonzero(np.triu(got, 1)) == 0
    assert np.linalg.norm(got - ref) <= 10 * n * EPS * cond * np.linalg.norm(ref)
    assert np.linalg.norm(got @ l_true - np.eye(n)) <= 10 * n * EPS * cond
    assert zb.lib().zolo_dtrtri_dev(h.ptr, -1, dl.data_ptr(), n, dy.data_ptr(), n) == -2


def test_dgemm_split_k(h):
    """Small output with a long reduction takes the split-K path (deterministic partial sums)."""
    rng = np.random.default_rng(3)
    m, n, k = 32, 64, 20000
    a = rng.standard_normal((k, m))
    b = rng.standard_normal((k, n))
    da, db, dc = dev(a), dev(b), dev(np.zeros((m, n)))
    outs = []
    for _ in range(2):
        r = zb.lib().zolo_dgemm_dev(h.ptr, b"T", b"N", m, n, k, 1.0, da.data_ptr(), k, db.data_ptr(), k, 0.0,
                                    dc.data_ptr(), m, 0, 0)
        assert r == 0
        outs.append(host(dc))
    ref = a.T @ b
    assert np.all(np.abs(outs[0] - ref) <= 2 * k * EPS * (np.abs(a.T) @ np.abs(b)))
    np.testing.assert_array_equal(outs[0], outs[1])  # run-to-run identical


@pytest.mark.parametrize("n", [1, 7, 64, 65, 100, 200, 513])
def test_potrf_vs_lapack(h, n):
    rng = np.random.default_rng(n)
    x = rng.standard_normal((n + 5, n))
    a = x.T @ x + n * np.eye(n)
    da = dev(a)
    info = zb.lib().zolo_dpotrf_dev(h.ptr, n, da.data_ptr(), n)
    assert info == 0
    l_ref = np.linalg.cholesky(a)
    got = np.tril(host(da))
    assert np.allclose(got, l_ref, rtol=0, atol=20 * n * EPS * np.sqrt(np.abs(np.diag(a)).max()))


def test_potrf_not_spd_reports_info(h):
    n = 150
    a = np.eye(n)
    a[100, 100] = -1.0
    da = dev(a)
    info = zb.lib().zolo_dpotrf_dev(h.ptr, n, da.data_ptr(), n)
    _, linfo = lapack.dpotrf(a, lower=1)
    assert info == linfo == 101


@pytest.mark.parametrize("trans", ["T", "N"])
@pytest.mark.parametrize("mn", [(5, 3), (70, 64), (129, 130), (300, 257)])
def test_trsm_vs_numpy(h, trans, mn):
    m, n = mn
    rng = np.random.default_rng(m + n)
    l = np.tril(rng.standard_normal((n, n))) + 4 * np.eye(n)
    x = rng.standard_normal((m, n))
    dl, dx, dy = dev(l), dev(x), dev(np.zeros((m, n)))
    r = zb.lib().zolo_dtrsm_dev(h.ptr, trans.encode(), m, n, dl.data_ptr(), n, dx.data_ptr(), m, dy.data_ptr(), m)
    assert r == 0
    ref = x @ np.linalg.inv(l.T if trans == "T" else l)
    got = host(dy)
    assert np.allclose(got, ref, rtol=1e-12, atol=1e-12 * np.abs(ref).max())


def _qr_gpu(h, w, m_top):
    mtot, n = w.shape
    dw = dev(w)
    import torch
    dtau = torch.zeros(n, dtype=torch.float64, device="cuda")
    dT = torch.zeros(((n + 31) // 32) * 1024, dtype=torch.float64, device="cuda")
    assert zb.lib().zolo_dgeqrf_dev(h.ptr, mtot, n, m_top, dw.data_ptr(), mtot, dtau.data_ptr(), dT.data_ptr()) == 0
    dq = dev(np.zeros((mtot, n)))
    assert zb.lib().zolo_dorgqr_dev(h.ptr, mtot, n, m_top, dw.data_ptr(), mtot, dT.data_ptr(), dq.data_ptr(),
                                    mtot) == 0
    return host(dw), dtau.cpu().numpy(), host(dq)


@pytest.mark.parametrize("mn", [(1, 1), (5, 3), (40, 32), (100, 33), (300, 200), (1000, 96), (700, 300), (513, 513),
                                (1031, 260)])
def test_geqrf_orgqr_unstructured_vs_lapack(h, mn):
    m, n = mn
    rng = np.random.default_rng(m * 7 + n)
    a = rng.standard_normal((m, n))
    w, tau, q = _qr_gpu(h, a, -1)
    qr, tau_ref, _, _ = lapack.dgeqrf(np.asfortranarray(a))
    q_ref, _, _ = lapack.dorgqr(qr, tau_ref)
    tol = 50 * max(m, 1) * EPS
    assert np.allclose(tau, tau_ref, rtol=0, atol=tol)
    assert np.allclose(np.triu(w[:n]), np.triu(qr[:n]), rtol=0, atol=tol * np.abs(a).max() * 4)
    assert np.allclose(q, q_ref, rtol=0, atol=tol)


@pytest.mark.parametrize("mn", [(64, 64), (100, 70), (257, 129), (600, 300), (301, 257), (390, 390)])
def test_structured_stack_qr(h, mn):
    """[X; sqrt(c) I]: the row-windowed factorisation gives LAPACK's Q and an exactly upper triangular Q2."""
    m, n = mn
    rng = np.random.default_rng(m + 3 * n)
    x = rng.standard_normal((m, n)) / 5
    w0 = np.vstack([x, 0.7 * np.eye(n)])
    w, tau, q = _qr_gpu(h, w0, m)
    q_ref = zo.house_qr_q(w0)
    assert np.allclose(q, q_ref, rtol=0, atol=100 * (m + n) * EPS)
    assert np.all(np.tril(q[m:], -1) == 0.0)


@pytest.mark.parametrize("which", ["qr", "chol"])
def test_zolo_term_kernels_vs_oracle(h, which):
    rng = np.random.default_rng(11)
    m, n, rk = 90, 70, 3
    x = rng.standard_normal((m, n)) / 8
    coeff = zo.compute_coeff(40.0, EPS, rk)
    dx = dev(x)
    for ip in range(1, rk + 1):
        c = coeff[2 * ip - 2]
        a = -coeff[2 * rk + ip - 1]
        dz = dev(np.zeros((m, n)))
        f = zb.lib().zolo_zoloqr_dev if which == "qr" else zb.lib().zolo_zolochol_dev
        assert f(h.ptr, m, n, dx.data_ptr(), m, c, a, dz.data_ptr(), m) == 0
        if which == "qr":
            ref = zo.zoloqr(x, coeff, rk, ip)
        else:
            ref, info = zo.zolochol("N", x, coeff, rk, ip)
        assert np.allclose(host(dz), ref, rtol=1e-11, atol=1e-12 * np.abs(ref).max())


def test_formx2_vs_oracle(h):
    rng = np.random.default_rng(12)
    m, n = 123, 77
    x = rng.standard_normal((m, n))
    z = rng.standard_normal((m, n))
    dx, dz = dev(x), dev(z)
    err = C.c_double()
    assert zb.lib().zolo_formx2_dev(h.ptr, m, n, 1.7, dx.data_ptr(), m, dz.data_ptr(), m, C.byref(err)) == 0
    x2, e_ref = zo.formx2(x, z, 1.7)
    assert np.allclose(host(dx), x2, rtol=4 * EPS, atol=4 * EPS)
    assert abs(err.value - e_ref) <= 1e-13 * e_ref
