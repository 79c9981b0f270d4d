"""The r-term sharded Zolo-PD driver (zolo-svd_b200/sharded.py) on CPU gloo ranks: the
distribution of the Zolotarev terms over 2 and 3 ranks (round-robin, uneven), the
all-reduced sum and the shared scalar control give the serial oracle's iterate and branch
sequence.  The ranks evaluate their terms with a backend built on the oracle, so no GPU is
needed; the product path (DeviceBackend) is the same driver with the library's kernels."""
import os
import socket
import sys

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


class OracleBackend:
    """Terms and FormX2 from the oracle's restatement, on CPU tensors of shape (n, m)."""

    def zeros_like(self, x):
        return torch.zeros_like(x)

    def term(self, kind, x, m, n, c, a, out):
        from oracle import zolo_oracle as zo
        xm = x.numpy().T
        if kind == "QR":
            w = np.vstack([xm, np.sqrt(c) * np.eye(n)])
            q = zo.house_qr_q(w)
            z, info = (a / np.sqrt(c)) * (q[:m] @ q[m:].T), 0
        else:
            z, info = zo.spd_solve_right(xm.T @ xm + c * np.eye(n), xm)
            z = a * z
        out.copy_(torch.from_numpy(np.ascontiguousarray(z.T)))
        return info

    def formx2(self, x, z, m, n, fone):
        new = (x + z) / fone
        err = float(torch.linalg.norm(new - x))
        x.copy_(new)
        return err


def _rank(rank, world, port, m, n, kappa, out):
    sys.path.insert(0, ROOT)
    import tests.conftest  # noqa: F401  (registers zolo_svd_b200)
    import importlib
    sh = importlib.import_module("zolo_svd_b200.sharded")
    from oracle import zolo_oracle as zo
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        a, u, v = zo.make_matrix(n, np.geomspace(1.0, 1.0 / kappa, n), 555, m=m)
        al = float(np.linalg.norm(a))
        be, _ = zo.bounds_qr_condest(a / al)
        x = torch.from_numpy(np.ascontiguousarray(a.T))
        it, branches, info = sh.pzolopd1_sharded("N", 5, m, n, al, be, x, OracleBackend())
        out[rank] = (x.numpy().T.copy(), it, branches, info, al, be)
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_sharded_terms_match_serial_oracle(world):
    sys.path.insert(0, ROOT)
    from oracle import zolo_oracle as zo
    m, n, kappa = 90, 70, 1e10
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.start_processes(_rank, args=(world, _free_port(), m, n, kappa, out), nprocs=world, join=True,
                       start_method="spawn")
    res = dict(out)
    q0, it0, br0, info0, al, be = res[0]
    for r in range(1, world):
        q, it, br, info, _, _ = res[r]
        assert np.array_equal(q, q0) and it == it0 and br == br0  # every rank holds the same iterate
    a, u, v = zo.make_matrix(n, np.geomspace(1.0, 1.0 / kappa, n), 555, m=m)
    q_s, st = zo.pzolopd1("N", 5, a, al, be)
    assert it0 == st.iterations and br0 == st.branches and info0 == 0
    # the same iteration; only the order of the term sum differs (kappa eps sensitivity)
    assert np.linalg.norm(q0 - q_s) / np.sqrt(n) <= 100 * zo.EPS * kappa
    assert zo.orthogonality(q0) <= 10 * n * zo.EPS


def test_term_assignment_round_robin():
    sys.path.insert(0, ROOT)
    import importlib
    sh = importlib.import_module("zolo_svd_b200.sharded")
    for rk in range(1, 9):
        for world in range(1, 10):
            got = sorted(t for r in range(world) for t in sh.my_terms(rk, r, world))
            assert got == list(range(1, rk + 1))
            sizes = [len(sh.my_terms(rk, r, world)) for r in range(world)]
            assert max(sizes) - min(sizes) <= 1
