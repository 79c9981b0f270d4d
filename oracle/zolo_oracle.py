"""CPU oracle: a restatement of the reference's QDWH-PD / Zolo-PD / Zolo-SVD path.

TEST INFRASTRUCTURE ONLY.  Only ``tests/``, ``__graft_entry__.smoke()`` and the
``cpu_baseline`` / ``--impl reference`` legs of ``bench.py`` may import this
module, and only as the checker or the timed CPU baseline.  The product path
(the CUDA library behind ``include/zolo_b200.h``) never calls it.

Parity status: the reference (Fortran + MPI + ScaLAPACK + ELPA) cannot be built
or run in this environment and ships no golden vectors, so parity against the
reference's own outputs is UNPINNED.  What is pinned instead:
  * the Zolotarev coefficients, FONE and the CON recursion against an
    independent multi-precision evaluation (mpmath ellipk / ellipfun) --
    ``tests/golden/gen_golden.py`` writes those fixtures;
  * the polar factor, H and singular values against matrices built with a
    known decomposition A = U diag(s) V^T.

Every P-routine of the reference, run on a 1x1 process grid, is its LAPACK
D-routine; this module calls SciPy's bundled LAPACK (dgeqrf, dorgqr, dpotrf,
dgetrf, dgecon, dsyevd) for those.  Citations are ``file:line`` inside the
reference project (shengguolsg/Zolo-SVD).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np
import scipy.linalg as sla
from scipy.linalg import lapack

# DLAMCH('Precision') = eps * base = 2**-52
EPS = float(np.finfo(np.float64).eps)


# ---------------------------------------------------------------------------
# Zolotarev coefficients (Auxil_Zolo.f90)
# ---------------------------------------------------------------------------
def mellipke(alpha: float, tol: float) -> tuple[float, float]:
    """Complete elliptic integrals K, E by the AGM (Auxil_Zolo.f90:36-71)."""
    m = math.sin(alpha) * math.sin(alpha)
    a0 = 1.0
    b0 = math.cos(alpha)
    s0 = m
    i1 = 0
    mm = 1.0
    a1 = a0
    while mm > tol:
        a1 = (a0 + b0) / 2.0
        b1 = math.sqrt(a0 * b0)
        c1 = (a0 - b0) / 2.0
        i1 += 1
        w1 = (2.0 ** i1) * (c1 * c1)
        mm = w1
        s0 = s0 + w1
        a0 = a1
        b0 = b1
    k = math.pi / (2.0 * a1)
    e = k * (1.0 - s0 / 2.0)
    return k, e


def mellipj(u: float, alpha: float, tol: float) -> tuple[float, float, float]:
    """Jacobi sn, cn, dn by descending Landen / AGM (Auxil_Zolo.f90:73-128)."""
    mchunk = 1000
    m = math.sin(alpha) * math.sin(alpha)
    a = [0.0] * (mchunk + 2)
    b = [0.0] * (mchunk + 2)
    c = [0.0] * (mchunk + 2)
    phin = [0.0] * (mchunk + 2)
    c[1] = math.sin(alpha)
    b[1] = math.cos(alpha)
    a[1] = 1.0
    i = 1
    nin = 0
    while abs(c[i]) > tol and i < mchunk:
        i += 1
        a[i] = (a[i - 1] + b[i - 1]) * 0.5
        b[i] = math.sqrt(a[i - 1] * b[i - 1])
        c[i] = (a[i - 1] - b[i - 1]) * 0.5
        if abs(c[i]) <= tol and abs(c[i - 1]) > tol:
            nin = i - 1
    phin[1] = u
    phin[i] = (2.0 ** nin) * a[i] * u
    while i > 1:
        i -= 1
        phin[i] = phin[i + 1]
        if nin >= i:
            phin[i] = 0.5 * (math.asin(c[i + 1] * math.sin(phin[i + 1]) / a[i + 1]) + phin[i + 1])
    sn = math.sin(phin[1])
    cn = math.cos(phin[1])
    dn = math.sqrt(1.0 - m * sn * sn)
    return sn, cn, dn


def choosem(con: float) -> int:
    """Zolotarev degree from the condition number (Auxil_Zolo.f90:130-163)."""
    if con < 1.001:
        return 2
    if con <= 1.01:
        return 3
    if con <= 1.1:
        return 4
    if con <= 1.2:
        return 5
    if con <= 1.5:
        return 6
    if con <= 2:
        return 8
    if con < 6.5:
        return 2
    if con < 180:
        return 3
    if con < 1.5e4:
        return 4
    if con < 2e6:
        return 5
    if con < 1e9:
        return 6
    if con < 3e12:
        return 7
    return 8


def compute_coeff(con: float, tol: float, rk: int) -> np.ndarray:
    """c_1..c_2r and the partial-fraction weights (Auxil_Zolo.f90:165-200).

    Returns ``coeff`` of length 3*rk: coeff[0:2rk] = c_i, coeff[2rk+i] is the
    reference's un-negated weight (a_i = -coeff[2rk+i], zoloqr.f90:110).
    """
    coeff = np.zeros(3 * rk)
    kappa = 1.0 / con
    alpha = math.acos(kappa)
    kk, _ = mellipke(alpha, tol)
    rk2 = 2 * rk
    for i in range(1, rk2 + 1):
        t = float(i) * kk / (rk2 + 1.0)
        sn, cn, _ = mellipj(t, alpha, tol)
        coeff[i - 1] = sn ** 2 / cn ** 2
    for i in range(1, rk + 1):
        v = 1.0
        for j in range(1, rk + 1):
            v = v * (coeff[2 * i - 2] - coeff[2 * j - 1])
            if i != j:
                v = v / (coeff[2 * i - 2] - coeff[2 * j - 2])
        coeff[rk2 + i - 1] = v
    return coeff


def zolo_fone(coeff: np.ndarray, rk: int) -> float:
    """FONE = prod (1+c_2j)/(1+c_2j-1)  (pzolopd1.f90:459-462)."""
    f = 1.0
    for i in range(1, rk + 1):
        f = f * (1.0 + coeff[2 * i - 1]) / (1.0 + coeff[2 * i - 2])
    return f


def zolo_next_con(con: float, coeff: np.ndarray, rk: int, fone: float) -> float:
    """CON for the next iteration (pzolopd1.f90:468-472)."""
    fcon = con
    for i in range(1, rk + 1):
        fcon = fcon * (con * con + coeff[2 * i - 1]) / (con * con + coeff[2 * i - 2])
    return max(fcon / fone, 1.0)


def hfunc(x: float) -> float:
    """QDWH dynamical weight a(l) (hfunc.f90:2-42; the formula at 26-39)."""
    tol = 30.0 * EPS
    x2 = x * x
    if abs(x - 1.0) <= tol:
        ww = 0.0
    else:
        tmp = 4.0 * (1.0 - x2) / (x2 * x2)
        ww = math.exp(math.log(tmp) / 3.0)
    sum1 = math.sqrt(1.0 + ww)
    h = math.sqrt(8.0 - 4.0 * ww + 8.0 * (2.0 - x2) / (x2 * sum1))
    return sum1 + h / 2.0


def qdwh_weights(lowk: float) -> tuple[float, float, float, float]:
    """a_k, b_k, c_k and the next lower bound (pqdwhfacs.f90:361-368)."""
    ak = hfunc(lowk)
    bk = (ak - 1.0) * (ak - 1.0) / 4.0  # Fortran (AK-1)**2 with an integer power is a product
    ck = ak + bk - 1.0
    l2 = lowk * lowk
    lnext = lowk * (ak + bk * l2) / (1.0 + ck * l2)
    return ak, bk, ck, lnext


# ---------------------------------------------------------------------------
# Bounds (test_zolodrv1.f90:167-189, pqdwhfacs.f90:318-344)
# ---------------------------------------------------------------------------
def rcond1_lu(x: np.ndarray) -> tuple[float, int]:
    """rcond of x in the 1-norm with ANORM=1, as PDGETRF + PDGECON('1',...,ONE,...)."""
    lu, piv, info = lapack.dgetrf(np.asfortranarray(x))
    if info != 0:
        return 0.0, int(info)
    rc, info2 = lapack.dgecon(lu, 1.0, norm="1")
    return float(rc), int(info2)


def bounds_zolodrv(a: np.ndarray) -> tuple[float, float, int]:
    """ALPHA = ||A||_F, BETA = rcond_1(A/ALPHA)/sqrt(n) (test_zolodrv1.f90:179-189)."""
    n = a.shape[1]
    alpha = float(np.linalg.norm(a, "fro"))
    rc, info = rcond1_lu(a / alpha)
    return alpha, rc / math.sqrt(n), info


def bounds_pqdwhfacs(x0: np.ndarray) -> tuple[float, int]:
    """BETA = ||X0||_1 * rcond_1(X0) / sqrt(n) for X0 = A/alpha (pqdwhfacs.f90:325-344)."""
    n = x0.shape[1]
    temp_beta = float(np.abs(x0).sum(axis=0).max())
    rc, info = rcond1_lu(x0)
    return temp_beta * rc / math.sqrt(n), info


def bounds_qr_condest(x0: np.ndarray) -> tuple[float, int]:
    """sigma_min lower-bound estimate from R of X0 = QR: 1/(sqrt(n) * ||R^-1||_1).

    ||R^-1||_1 is evaluated exactly here (dtrtri), as on the GPU, which forms R^-1
    with its blocked triangular inverse and takes its exact norm.
    """
    n = x0.shape[1]
    r = np.triu(sla.qr(x0, mode="r")[0][:n, :n])
    if np.any(np.diag(r) == 0):
        return 0.0, 1
    rinv, info = lapack.dtrtri(r, lower=0)
    inv1 = float(np.abs(rinv).sum(axis=0).max())
    return 1.0 / (math.sqrt(n) * inv1), int(info)


# ---------------------------------------------------------------------------
# Per-term kernels
# ---------------------------------------------------------------------------
def house_qr_q(w: np.ndarray) -> np.ndarray:
    """Explicit Q (m x n) of a Householder QR: dgeqrf + dorgqr (mpdgeqrf.f / mpdorgqr.f)."""
    qr, tau, _, info = lapack.dgeqrf(np.asfortranarray(w))
    assert info == 0
    q, _, info = lapack.dorgqr(qr, tau)
    assert info == 0
    return q


def zoloqr(x: np.ndarray, coeff: np.ndarray, rk: int, ip: int) -> np.ndarray:
    """Term ip (1-based): (a_ip/sqrt(c)) Q1 Q2^T of [X; sqrt(c) I] (zoloqr.f90:82-112)."""
    n = x.shape[1]
    m = x.shape[0]
    c = coeff[2 * ip - 2]
    w = np.zeros((m + n, n), order="F")
    w[:m] = x
    w[m:] = math.sqrt(c) * np.eye(n)
    q = house_qr_q(w)
    akk = -coeff[2 * rk + ip - 1] / math.sqrt(c)
    return akk * (q[:m] @ q[m:].T)


def spd_solve_right(w: np.ndarray, x: np.ndarray) -> tuple[np.ndarray, int]:
    """X * W^{-1} for SPD W via POTRF of the upper factor (PDPOSV 'U' with PDTRAN)."""
    u, info = lapack.dpotrf(np.asfortranarray(w), lower=0)
    if info != 0:
        return np.full_like(x, np.nan), int(info)
    u = np.triu(u)
    # Y = X U^{-1} U^{-T}
    y = sla.solve_triangular(u, x.T, trans="T", lower=False)  # U^{-T} X^T
    y = sla.solve_triangular(u, y, trans="N", lower=False)  # U^{-1} U^{-T} X^T
    return np.ascontiguousarray(y.T), 0


def spd_solve_left(w: np.ndarray, x: np.ndarray) -> tuple[np.ndarray, int]:
    """W^{-1} X for SPD W (PDPOSV 'U' applied directly to X)."""
    u, info = lapack.dpotrf(np.asfortranarray(w), lower=0)
    if info != 0:
        return np.full_like(x, np.nan), int(info)
    u = np.triu(u)
    y = sla.solve_triangular(u, x, trans="T", lower=False)
    y = sla.solve_triangular(u, y, trans="N", lower=False)
    return y, 0


def zolochol(sym: str, x: np.ndarray, coeff: np.ndarray, rk: int, ip: int) -> tuple[np.ndarray, int]:
    """Term ip: a_ip X (X^T X + c I)^{-1} (zolochol.f90:87-113)."""
    n = x.shape[1]
    w = x.T @ x + coeff[2 * ip - 2] * np.eye(n)
    if sym.upper() == "S":
        z, info = spd_solve_left(w, x)
    else:
        z, info = spd_solve_right(w, x)
    return -coeff[2 * rk + ip - 1] * z, info


def formx2(x: np.ndarray, z: np.ndarray, fone: float) -> tuple[np.ndarray, float]:
    """X2 = (X + Z)/FONE and ERR = ||X2 - X||_F (FormX2.f90:73-89)."""
    x2 = (x + z) / fone
    err = float(np.linalg.norm(x - x2, "fro"))
    return x2, err


# ---------------------------------------------------------------------------
# Drivers
# ---------------------------------------------------------------------------
@dataclass
class PDStats:
    iterations: int = 0
    branches: list = field(default_factory=list)  # 'QR' / 'CH'
    con: list = field(default_factory=list)
    err: list = field(default_factory=list)
    alpha: float = 0.0
    beta: float = 0.0
    info: int = 0


def zolo_term(kind: str, sym: str, x: np.ndarray, coeff: np.ndarray, rk: int, ip: int) -> tuple[np.ndarray, int]:
    """Term ip of one Zolo-PD iteration: ZOLOQR (kind 'QR') or ZOLOCHOL (kind 'CH'), with INFO."""
    if kind == "QR":
        return zoloqr(x, coeff, rk, ip), 0
    return zolochol(sym, x, coeff, rk, ip)


def pzolopd1(sym: str, rk: int, a: np.ndarray, alpha: float, beta: float,
             maxit: int = 6, term_map=None) -> tuple[np.ndarray, PDStats]:
    """Zolo-PD (pzolopd1.f90:280-487).  The r terms of an iteration are evaluated by
    ``term_map(zolo_term, [(kind, sym, x, coeff, rk, ip), ...])`` -- serially by default; a
    process pool gives the reference's r concurrent process groups (pzolopd1.f90:298-374) --
    and summed in term order (the DGSUM2D of pzolopd1.f90:424-429, 447-451)."""
    if term_map is None:
        term_map = lambda fn, args: [fn(*x) for x in args]
    st = PDStats(alpha=alpha, beta=beta)
    scale = alpha * beta
    con = 1.0 / beta
    x = np.array(a, dtype=np.float64, order="F") / scale
    tol = EPS
    tol1 = 10.0 * EPS / 2.0
    tol2 = math.exp(math.log(tol1) / (2.0 * rk + 1.0))
    it = 0
    err = 1.0
    fone = 1.0
    while err > tol2 and it < maxit:
        coeff = compute_coeff(con, tol, rk)
        maxc = float(np.max(coeff[: 2 * rk]))
        z = np.zeros_like(x)
        kind = "QR" if (it == 0 or con > 1.0e3) and maxc > 3.0e2 else "CH"
        st.branches.append(kind)
        for zt, info in term_map(zolo_term, [(kind, sym, x, coeff, rk, ip) for ip in range(1, rk + 1)]):
            if info != 0 and st.info == 0:
                st.info = info
            z += zt
        st.con.append(con)
        fone = zolo_fone(coeff, rk)
        con = zolo_next_con(con, coeff, rk, fone)
        x, err = formx2(x, z, fone)
        st.err.append(err)
        it += 1
    st.iterations = it
    return x, st


def _qdwh_loop(sym: str, q: np.ndarray, lowk: float, maxit: int | None, left_solve_only: bool,
               st: PDStats) -> np.ndarray:
    """The QDWH iteration of pqdwhfacs.f90:359-457 (and zolopd.f90:348-440)."""
    n = q.shape[1]
    m = q.shape[0]
    tol1 = 10.0 * EPS / 2.0
    tol2 = math.exp(math.log(tol1) / 3.0)
    it = 0
    err = 1.0
    err2 = abs(1.0 - lowk)
    while (it == 0 or err > tol2 or err2 > tol1) and (maxit is None or it <= maxit):
        ak, bk, ck, lowk = qdwh_weights(lowk)
        st.con.append(ck)
        if ck > 100.0:
            st.branches.append("QR")
            sck = math.sqrt(ck)
            w = np.zeros((m + n, n), order="F")
            w[:m] = q
            w[m:] = (1.0 / sck) * np.eye(n)
            qq = house_qr_q(w)
            w2 = qq[:m] @ qq[m:].T
            akk = (ak - bk / ck) / sck
            bkk = bk / ck
            w2 = bkk * q + akk * w2
        else:
            st.branches.append("CH")
            g = ck * (q.T @ q) + np.eye(n)
            if left_solve_only or sym.upper() == "S":
                z, info = spd_solve_left(g, q)
            else:
                z, info = spd_solve_right(g, q)
            if info != 0 and st.info == 0:
                st.info = info
            akk = ak - bk / ck
            bkk = bk / ck
            w2 = bkk * q + akk * z
        err = float(np.linalg.norm(q - w2, "fro"))
        st.err.append(err)
        it += 1
        err2 = abs(1.0 - lowk)
        q = w2
    st.iterations = it
    return q


def polar_h(q: np.ndarray, a: np.ndarray) -> np.ndarray:
    """H = (Q^T A + (Q^T A)^T)/2 (pqdwhfacs.f90:460-466; ZoloCHK1.f90:80-83)."""
    h = q.T @ a
    return 0.5 * (h + h.T)


def pqdwhfacs(sym: str, a: np.ndarray, sigma: float = 0.0, polar: str = "T",
              bounds: str = "lu") -> tuple[np.ndarray, np.ndarray | None, PDStats]:
    """QDWH-PD of A - sigma I (pqdwhfacs.f90:296-466).

    ``bounds='lu'`` is the reference's PDGETRF + PDGECON estimate; ``'qr'`` is the
    QR + triangular-condition estimate the GPU path uses.
    """
    st = PDStats()
    q = np.array(a, dtype=np.float64, order="F")
    n = q.shape[1]
    if sigma != 0.0:
        q[np.arange(n), np.arange(n)] -= sigma
    alpha = float(np.linalg.norm(q, "fro"))
    q = q / alpha
    if bounds == "lu":
        beta, info = bounds_pqdwhfacs(q)
    else:
        temp_beta = float(np.abs(q).sum(axis=0).max())  # ||X0||_1, pqdwhfacs.f90:325
        beta, info = bounds_qr_condest(q)
        beta *= temp_beta
    st.alpha, st.beta = alpha, beta
    if info != 0:
        st.info = info
        return q, None, st
    q = _qdwh_loop(sym, q, beta, 12, False, st)
    h = polar_h(q, a) if polar.upper() == "T" else None
    return q, h, st


def zolopd(a: np.ndarray, sigma: float = 0.0, polar: str = "T",
           maxit: int = 100) -> tuple[np.ndarray, np.ndarray | None, PDStats]:
    """Older QDWH entry (zolopd.f90:290-440): BETA = rcond/sqrt(n), left SPD solve only.

    The reference loop has no iteration cap; ``maxit`` only guards this restatement.
    """
    st = PDStats()
    q = np.array(a, dtype=np.float64, order="F")
    n = q.shape[1]
    if sigma != 0.0:
        q[np.arange(n), np.arange(n)] -= sigma
    alpha = float(np.linalg.norm(q, "fro"))
    q = q / alpha
    rc, info = rcond1_lu(q)
    beta = rc / math.sqrt(n)
    st.alpha, st.beta = alpha, beta
    if info != 0:
        st.info = info
        return q, None, st
    q = _qdwh_loop("S", q, beta, maxit, True, st)
    h = polar_h(q, a) if polar.upper() == "T" else None
    return q, h, st


# ---------------------------------------------------------------------------
# SVD assembly, checks, spectral split
# ---------------------------------------------------------------------------
def zolochk1(a: np.ndarray, q: np.ndarray) -> dict:
    """H = sym(Q^T A), eig(H), U = Q V and the printed checks (ZoloCHK1.f90:80-177)."""
    h = polar_h(q, a)
    ev, v = sla.eigh(h, driver="evd")
    u = q @ v
    n = a.shape[1]
    norma = float(np.max(ev))
    res = float(np.linalg.norm(a @ v - u * ev[None, :], "fro"))
    orth_u = float(np.linalg.norm(u.T @ u - np.eye(n), "fro"))
    orth_v = float(np.linalg.norm(v.T @ v - np.eye(n), "fro"))
    return dict(h=h, ev=ev, v=v, u=u, res=res, res_rel=res / norma, orth_u=orth_u,
                orth_v=orth_v, orth_u_n=orth_u / n, orth_v_n=orth_v / n)


def backward_error(a: np.ndarray, q: np.ndarray, h: np.ndarray) -> float:
    """||A - Q H||_F / ||A||_F (ZoloCHK.f90:79-89, normalised)."""
    return float(np.linalg.norm(a - q @ h, "fro") / np.linalg.norm(a, "fro"))


def orthogonality(q: np.ndarray) -> float:
    """||Q^T Q - I||_F / sqrt(n)."""
    n = q.shape[1]
    return float(np.linalg.norm(q.T @ q - np.eye(n), "fro") / math.sqrt(n))


def pqdwhsubit(a: np.ndarray, q: np.ndarray, norma: float, rng: np.random.Generator,
               pp: int = 3) -> tuple[np.ndarray, np.ndarray, int, float]:
    """Subspace iteration split from the polar factor of A - sigma I (pqdwhsubit.f90:227-312).

    Returns (V, V^T A V, Rk, err).  C = (Q - I)/2 selects the eigenvalues below
    the shift (the code subtracts I although its comment says Q+I).
    """
    n = a.shape[0]
    tol1 = 10.0 * EPS / 2.0
    c = (q - np.eye(n)) / 2.0
    alpha = float(np.linalg.norm(c, "fro")) ** 2
    rk = int(round(alpha))
    kk = min(rk + pp, n)
    x = rng.random((n, kk))
    it = 1
    while True:
        x = house_qr_q(x)
        x = c @ x
        qr, tau, _, _ = lapack.dgeqrf(np.asfortranarray(x))
        # PDORGQR(N, N, kk, ...): full n x n Q from kk reflectors
        full = np.zeros((n, n), order="F")
        full[:, :kk] = qr
        tau_full = np.zeros(n)
        tau_full[:kk] = tau
        v, _, _ = lapack.dorgqr(full, tau_full)
        e = v.T @ (a @ v)
        err = float(np.linalg.norm(e[:rk, rk:], "fro")) / norma
        if err <= 4.0 * tol1 or it == 2:
            return v, e, rk, err
        x = c @ v[:, :rk]
        kk = rk
        it += 1


def zoloeig(a: np.ndarray, q: np.ndarray, rng: np.random.Generator) -> tuple[np.ndarray, np.ndarray, int]:
    """Partial eigendecomposition from a spectral split (ZoloEig.f90:78-102)."""
    norma = float(np.linalg.norm(a, "fro"))
    v, e, rk, _ = pqdwhsubit(a, q, norma, rng)
    ev, vv = sla.eigh(e[:rk, :rk], driver="evd")
    return ev, v[:, :rk] @ vv, rk


# ---------------------------------------------------------------------------
# Seeded synthetic matrices with a prescribed SVD
# ---------------------------------------------------------------------------
def haar(n: int, rng: np.random.Generator, m: int | None = None) -> np.ndarray:
    """Haar-distributed orthonormal columns: QR of N(0,1) with diag(R) > 0."""
    m = n if m is None else m
    g = rng.standard_normal((m, n))
    q, r = np.linalg.qr(g)
    return q * np.sign(np.diag(r))[None, :]


def make_matrix(n: int, s: np.ndarray, seed: int, m: int | None = None) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
    """A = (U * s) V^T with Haar U (m x n) and V (n x n); returns (A, U, V)."""
    rng = np.random.default_rng(seed)
    m = n if m is None else m
    u = haar(n, rng, m)
    v = haar(n, rng)
    a = (u * s[None, :]) @ v.T
    return np.asfortranarray(a), u, v
