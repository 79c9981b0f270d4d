"""The allocation-free Cholesky entry point (zolo_dpotrf_noalloc).

It exists for callers that cannot let the library call cudaMalloc (hosts whose
device memory belongs to another allocator, or that cannot accept cudaMalloc's
device-wide synchronisation); its scratch is a fixed static device array, so
n <= ZOLO_NOALLOC_MAX_N.  Checked through the C-ABI against the handle-based
zolo_dpotrf_dev on two calls in a row, with the Cholesky tolerance of the
kernel tests.  This file is collected last on purpose.
"""
import numpy as np
import pytest

import zolo_svd_b200 as zb
from oracle import zolo_oracle as zo

pytestmark = pytest.mark.gpu
MAX_N = 1024


def _spd(n, seed):
    rng = np.random.default_rng(seed)
    x = rng.standard_normal((n + 5, n))
    return x.T @ x + n * np.eye(n)


def test_dpotrf_noalloc_matches_handle_entry_point():
    import torch
    lib = zb.lib()
    h = zb.Handle(0)
    stream = torch.cuda.current_stream().cuda_stream
    for call, n in enumerate([300, MAX_N]):  # two calls in a row, the second at the maximum size
        a = _spd(n, 40 + call)
        d_ref = zb.colmajor_to_device(a)
        d_new = zb.colmajor_to_device(a)
        torch.cuda.synchronize()
        assert lib.zolo_dpotrf_dev(h.ptr, n, d_ref.data_ptr(), n) == 0
        assert lib.zolo_dpotrf_noalloc(n, d_new.data_ptr(), n, stream) == 0
        l_ref = np.tril(zb.device_to_colmajor(d_ref))
        l_new = np.tril(zb.device_to_colmajor(d_new))
        tol = 20 * n * zo.EPS * np.sqrt(np.abs(np.diag(a)).max())
        assert np.allclose(l_new, l_ref, rtol=0, atol=tol)
        assert np.allclose(l_new, np.linalg.cholesky(a), rtol=0, atol=tol)
    h.close()


def test_dpotrf_noalloc_rejects_oversize_and_reports_info():
    import torch
    lib = zb.lib()
    stream = torch.cuda.current_stream().cuda_stream
    big = torch.zeros((MAX_N + 1, MAX_N + 1), dtype=torch.float64, device="cuda")
    assert lib.zolo_dpotrf_noalloc(MAX_N + 1, big.data_ptr(), MAX_N + 1, stream) == -1
    n = 130
    a = np.eye(n)
    a[77, 77] = -2.0
    d = zb.colmajor_to_device(a)
    torch.cuda.synchronize()
    assert lib.zolo_dpotrf_noalloc(n, d.data_ptr(), n, stream) == 78  # INFO cleared and set per call
    d = zb.colmajor_to_device(np.eye(n))
    torch.cuda.synchronize()
    assert lib.zolo_dpotrf_noalloc(n, d.data_ptr(), n, stream) == 0


def test_dpotrf_noalloc_padded_leading_dimension():
    """An odd order with lda > n (the padding rows are neither read as data nor written)."""
    import torch
    lib = zb.lib()
    h = zb.Handle(0)
    stream = torch.cuda.current_stream().cuda_stream
    n, lda = 257, 260
    a = _spd(n, 77)
    buf = np.full((lda, n), 5.0)
    buf[:n] = a
    d_new = zb.colmajor_to_device(buf)
    d_ref = zb.colmajor_to_device(a)
    torch.cuda.synchronize()
    assert lib.zolo_dpotrf_dev(h.ptr, n, d_ref.data_ptr(), n) == 0
    assert lib.zolo_dpotrf_noalloc(n, d_new.data_ptr(), lda, stream) == 0
    got = zb.device_to_colmajor(d_new)
    l_ref = np.tril(zb.device_to_colmajor(d_ref))
    tol = 20 * n * zo.EPS * np.sqrt(np.abs(np.diag(a)).max())
    assert np.allclose(np.tril(got[:n]), l_ref, rtol=0, atol=tol)
    assert np.all(got[n:] == 5.0)
    assert lib.zolo_dpotrf_noalloc(n, None, lda, stream) == -2
    h.close()
