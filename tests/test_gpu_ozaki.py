"""FP64 products emulated on the INT8 tensor cores (zolo_ozgemm_dev, ozaki.cu)
against NumPy and against the DMMA GEMM (zolo_dgemm_dev) on the same inputs.

Tolerance (stated per element, rigorous for the splitting): with S digit planes
each row r of op(A) and column c of op(B) is represented to 2^(e - 7S), e the
exponent with max < 2^e <= 2 max, and the dropped digit products t + u >= S add
at most S * 2^(e_r + f_c - 7S) per k, so

    |C - C_ref|(r, c) <= 4 (S + 2) K 2^(-7S) max_k|op(A)(r,k)| max_k|op(B)(k,c)|
                        + 2 (K + 2) eps (|alpha| |op(A)| |op(B)| + |beta| |C0|)(r, c)

(the second term is the FP64 rounding of the reference and of the recombination).
"""
import numpy as np
import pytest

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


def op(a, t):
    return a.T if t == "T" else a


def bound(oa, ob, c0, alpha, beta, s):
    k = oa.shape[1]
    ra = np.max(np.abs(oa), axis=1, initial=0.0)[:, None]
    cb = np.max(np.abs(ob), axis=0, initial=0.0)[None, :]
    split = 4 * (s + 2) * k * 2.0 ** (-7 * s) * abs(alpha) * ra * cb
    fp = 2 * (k + 2) * EPS * (abs(alpha) * np.abs(oa) @ np.abs(ob) + abs(beta) * np.abs(c0))
    return split + fp + 1e-300


def run(h, ta, tb, a, b, c0, alpha, beta, s, tri=0, kfrom=0):
    m = op(a, ta).shape[0]
    n = op(b, tb).shape[1]
    k = op(a, ta).shape[1]
    da, db, dc = dev(a), dev(b), dev(c0)
    r = zb.lib().zolo_ozgemm_dev(h.ptr, ta.encode(), tb.encode(), m, n, k, alpha, da.data_ptr(), a.shape[0],
                                 db.data_ptr(), b.shape[0], beta, dc.data_ptr(), m, tri, kfrom, s)
    assert r == 0, r
    return host(dc)


SHAPES = [(1, 1, 1), (7, 5, 3), (65, 65, 65), (130, 129, 67), (257, 300, 513), (513, 64, 1000), (64, 1000, 33)]


@pytest.mark.parametrize("ta", ["N", "T"])
@pytest.mark.parametrize("tb", ["N", "T"])
@pytest.mark.parametrize("mnk", SHAPES)
def test_ozgemm_vs_numpy(h, ta, tb, mnk):
    m, n, k = mnk
    rng = np.random.default_rng(m * 1000 + n + k)
    a = rng.standard_normal((k, m) if ta == "T" else (m, k))
    b = rng.standard_normal((n, k) if tb == "T" else (k, n))
    c0 = rng.standard_normal((m, n))
    alpha, beta = 1.25, -0.5
    got = run(h, ta, tb, a, b, c0, alpha, beta, 8)
    ref = alpha * op(a, ta) @ op(b, tb) + beta * c0
    assert np.all(np.abs(got - ref) <= bound(op(a, ta), op(b, tb), c0, alpha, beta, 8))


@pytest.mark.parametrize("s", [6, 7, 8])
def test_ozgemm_slices_accuracy(h, s):
    """Normwise error falls by ~2^-7 per digit plane; 8 planes reach FP64 level."""
    rng = np.random.default_rng(11 + s)
    m, n, k = 384, 320, 1000
    a = rng.standard_normal((m, k)) * np.exp(rng.uniform(-8, 8, (m, 1)))  # rows of very different scale
    b = rng.standard_normal((k, n))
    got = run(h, "N", "N", a, b, np.zeros((m, n)), 1.0, 0.0, s)
    ref = a @ b
    assert np.all(np.abs(got - ref) <= bound(a, b, np.zeros((m, n)), 1.0, 0.0, s))
    rel = np.linalg.norm((got - ref) / np.max(np.abs(a), axis=1, keepdims=True)) / (np.sqrt(k) * np.linalg.norm(b))
    assert rel <= {6: 1e-12, 7: 1e-14, 8: 1e-15}[s], rel


def test_ozgemm_vs_dmma(h):
    """Same product through the DMMA GEMM and the INT8 emulation: agreement at FP64 level."""
    import torch
    rng = np.random.default_rng(5)
    n = 2048
    a = rng.standard_normal((n, n)) / np.sqrt(n)
    b = rng.standard_normal((n, n)) / np.sqrt(n)
    da, db = dev(a), dev(b)
    c1 = torch.zeros_like(da)
    c2 = torch.zeros_like(da)
    assert zb.lib().zolo_dgemm_dev(h.ptr, b"N", b"T", n, n, n, 1.0, da.data_ptr(), n, db.data_ptr(), n, 0.0,
                                   c1.data_ptr(), n, 0, 0) == 0
    for _ in range(2):  # two calls in a row: the workspace is reused
        assert zb.lib().zolo_ozgemm_dev(h.ptr, b"N", b"T", n, n, n, 1.0, da.data_ptr(), n, db.data_ptr(), n, 0.0,
                                        c2.data_ptr(), n, 0, 0, 8) == 0
    x1, x2 = host(c1), host(c2)
    ref = a @ b.T
    e1 = np.linalg.norm(x1 - ref) / np.linalg.norm(ref)
    e2 = np.linalg.norm(x2 - ref) / np.linalg.norm(ref)
    assert e2 <= 1e-15 and e2 <= 20 * max(e1, EPS), (e1, e2)


def test_ozgemm_gram_lower(h):
    """Gram X^T X (one splitting for both sides) into the lower triangle only."""
    import torch
    rng = np.random.default_rng(9)
    k, n = 1500, 700
    x = rng.standard_normal((k, n))
    dx = dev(x)
    sentinel = 7.0
    dc = torch.full((n, n), sentinel, dtype=torch.float64, device="cuda")
    assert zb.lib().zolo_ozgemm_dev(h.ptr, b"T", b"N", n, n, k, 1.0, dx.data_ptr(), k, dx.data_ptr(), k, 0.0,
                                    dc.data_ptr(), n, 1, 0, 8) == 0
    got = host(dc)
    ref = x.T @ x
    low = np.tril(np.ones((n, n), dtype=bool))
    bd = bound(x.T, x, np.zeros((n, n)), 1.0, 0.0, 8)
    assert np.all(np.abs(got - ref)[low] <= bd[low])
    assert np.all(got[~low] == sentinel)  # the strict upper triangle is untouched


@pytest.mark.parametrize("kfrom", [1, 2, 3])
def test_ozgemm_triangular_skip(h, kfrom):
    """kfrom_n = 1: op(B) lower; 2: op(A) upper; 3: both -- the skipped k ranges hold zeros."""
    rng = np.random.default_rng(20 + kfrom)
    n = 300
    a = rng.standard_normal((n, n))
    b = rng.standard_normal((n, n))
    if kfrom in (2, 3):
        a = np.triu(a)
    if kfrom in (1, 3):
        b = np.tril(b)
    c0 = rng.standard_normal((n, n))
    got = run(h, "N", "N", a, b, c0, -1.0, 1.0, 8, 0, kfrom)
    ref = -(a @ b) + c0
    assert np.all(np.abs(got - ref) <= bound(a, b, c0, -1.0, 1.0, 8))


def test_ozgemm_zero_rows_and_scales(h):
    """Zero rows and columns, and operands spanning 1e-200 .. 1e200 across rows."""
    rng = np.random.default_rng(3)
    m, n, k = 200, 150, 400
    a = rng.standard_normal((m, k)) * (10.0 ** rng.uniform(-200, 200, (m, 1)))
    a[5] = 0.0
    b = rng.standard_normal((k, n))
    b[:, 7] = 0.0
    got = run(h, "N", "N", a, b, np.zeros((m, n)), 1.0, 0.0, 8)
    ref = a @ b
    assert np.all(got[5] == 0.0) and np.all(got[:, 7] == 0.0)
    assert np.all(np.abs(got - ref) <= bound(a, b, np.zeros((m, n)), 1.0, 0.0, 8))


def test_ozgemm_bad_arguments(h):
    import torch
    d = torch.zeros(16, dtype=torch.float64, device="cuda")
    p = d.data_ptr()
    assert zb.lib().zolo_ozgemm_dev(h.ptr, b"N", b"N", 2, 2, 2, 1.0, p, 2, p, 2, 0.0, p, 2, 0, 0, 5) == -17
    assert zb.lib().zolo_ozgemm_dev(h.ptr, b"N", b"N", 2, 3, 2, 1.0, p, 2, p, 2, 0.0, p, 2, 1, 0, 8) == -15
    # K beyond exact INT32 accumulation for 8 planes
    assert zb.lib().zolo_ozgemm_dev(h.ptr, b"N", b"N", 2, 2, 20000, 1.0, p, 2, p, 2, 0.0, p, 2, 0, 0, 8) == -6
