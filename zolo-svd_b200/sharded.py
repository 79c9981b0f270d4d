"""PZOLOPD1 with the r Zolotarev terms of each iteration sharded over the ranks of a
torch.distributed process group: the reference's group parallelism (pzolopd1.f90:298-374),
one GPU per group of terms instead of one MPI process group per term.

Rank p of P evaluates the terms ip = p + 1, p + 1 + P, ... (ZOLOQR, zoloqr.f90:82-112, or
ZOLOCHOL, zolochol.f90:87-113, on its own GPU through zolo_zoloqr_dev /
zolo_zolochol_dev), the partial sums are all-reduced (NCCL over NVLink: one n x m FP64
sum per iteration, the DGSUM2D of pzolopd1.f90:424-429, 447-451), and every rank applies
FormX2 (FormX2.f90:73-89) and the same scalar iteration control (pzolopd1.f90:381-397,
459-472), so the iterate stays bitwise identical on all ranks (an all-reduce returns the
same sum to every rank).

The term evaluation and FormX2 are a backend: ``DeviceBackend`` (the library's kernels
on the rank's GPU, the product path) or any object with the same three methods (the
tests run the distribution logic on CPU gloo ranks with a backend built on the oracle).
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from . import ZoloError, compute_coeff, fone_next, lib

EPS = float(np.finfo(np.float64).eps)


class DeviceBackend:
    """Terms and FormX2 on the rank's GPU; matrices are torch CUDA tensors holding the m x n
    column-major matrix (shape (n, m), X[j, i] = X(i, j))."""

    def __init__(self, handle):
        self.h = handle

    def zeros_like(self, x):
        import torch
        return torch.zeros_like(x)

    def term(self, kind: str, x, m: int, n: int, c: float, a: float, out) -> int:
        f = lib().zolo_zoloqr_dev if kind == "QR" else lib().zolo_zolochol_dev
        r = f(self.h.ptr, m, n, x.data_ptr(), m, c, a, out.data_ptr(), m)
        if r < 0:
            raise ZoloError("zolo_zoloqr_dev" if kind == "QR" else "zolo_zolochol_dev", r)
        return r

    def formx2(self, x, z, m: int, n: int, fone: float) -> float:
        err = C.c_double()
        r = lib().zolo_formx2_dev(self.h.ptr, m, n, fone, x.data_ptr(), m, z.data_ptr(), m, C.byref(err))
        if r != 0:
            raise ZoloError("zolo_formx2_dev", r)
        return err.value


def my_terms(rk: int, rank: int, world: int) -> list[int]:
    """The 1-based term indices rank `rank` of `world` evaluates (round-robin)."""
    return list(range(rank + 1, rk + 1, world))


def pzolopd1_sharded(sym: str, rk: int, m: int, n: int, alpha: float, beta: float, x, backend, group=None,
                     maxit: int = 6):
    """Zolo-PD of A/(alpha beta) on every rank of `group` (x holds A on entry, the polar factor
    on return).  Returns (iterations, branches, INFO of the first failed Cholesky, 0 if none)."""
    import torch.distributed as dist
    world = dist.get_world_size(group) if dist.is_initialized() else 1
    rank = dist.get_rank(group) if dist.is_initialized() else 0
    if m < n:
        raise ValueError("m < n")
    if sym.upper() != "N":
        raise ValueError("the sharded driver takes SYM = 'N' (the right solve of zolochol.f90:103-106)")
    if not (alpha > 0.0 and beta > 0.0):
        raise ValueError("alpha and beta must be positive")
    x.mul_(1.0 / (alpha * beta))
    con = 1.0 / beta
    tol2 = math.exp(math.log(10.0 * EPS / 2.0) / (2.0 * rk + 1.0))
    err, it, info = 1.0, 0, 0
    branches = []
    z = backend.zeros_like(x)
    zt = backend.zeros_like(x)
    mine = my_terms(rk, rank, world)
    while err > tol2 and it < maxit:
        coeff = compute_coeff(con, EPS, rk)
        maxc = float(np.max(coeff[: 2 * rk]))
        kind = "QR" if (it == 0 or con > 1.0e3) and maxc > 3.0e2 else "CH"
        branches.append(kind)
        z.zero_()
        for ip in mine:
            r = backend.term(kind, x, m, n, float(coeff[2 * ip - 2]), float(-coeff[2 * rk + ip - 1]), zt)
            if r > 0 and info == 0:
                info = r
            z.add_(zt)
        if world > 1:
            dist.all_reduce(z, op=dist.ReduceOp.SUM, group=group)
        fone, con = fone_next(con, coeff, rk)  # FONE and the next CON (pzolopd1.f90:459-472)
        err = backend.formx2(x, z, m, n, fone)
        it += 1
    if world > 1:
        # a factorization failure on any rank is reported by all
        import torch
        t = torch.tensor([info], dtype=torch.int64, device=z.device)
        dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
        info = int(t.item())
    return it, branches, info
