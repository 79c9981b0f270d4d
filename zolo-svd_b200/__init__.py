"""zolo-svd_b200: B200-native QDWH-PD / Zolo-PD / Zolo-SVD.

Python mirror of the reference's entry points (shengguolsg/Zolo-SVD) over the
C-ABI of ``include/zolo_b200.h``:

* ``pqdwhfacs``  -- PQDWHFACS (pqdwhfacs.f90:2-3)
* ``zolopd``     -- ZOLOPD    (zolopd.f90:2-3)
* ``pzolopd1``   -- PZOLOPD1  (pzolopd1.f90:2)
* ``compute_coeff``, ``hfunc``, ``choosem`` -- Auxil_Zolo.f90 / hfunc.f90

The host-array functions take NumPy arrays (any layout; they are passed as
Fortran-ordered copies) and return INFO with the reference's conventions.  The
``*_dev`` functions take device pointers / CUDA tensors in column-major form
(see ``colmajor_to_device``).  Every computation runs in the CUDA library; if
the library is missing this module raises instead of falling back to the CPU.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libzolo_b200.so")
_lib = None

c_double_p = C.POINTER(C.c_double)
c_int_p = C.POINTER(C.c_int)


class Stats(C.Structure):
    _fields_ = [
        ("iterations", C.c_int),
        ("qr_iterations", C.c_int),
        ("chol_iterations", C.c_int),
        ("info", C.c_int),
        ("alpha", C.c_double),
        ("beta", C.c_double),
        ("last_err", C.c_double),
        ("ms_total", C.c_double),
        ("ms_bounds", C.c_double),
        ("ms_iter", C.c_double),
        ("ms_h", C.c_double),
        ("flops", C.c_double),
        ("launches", C.c_int64),
        ("con", C.c_double * 16),
        ("err", C.c_double * 16),
        ("branch", C.c_int * 16),
        ("flops_executed", C.c_double),
        ("ns_steps", C.c_int),
        ("ns_finish", C.c_int),
        ("ms_step", C.c_double * 16),
        ("ms_finish", C.c_double),
        ("terms", C.c_int * 16),
    ]

    def as_dict(self) -> dict:
        it = self.iterations
        return dict(iterations=it, qr_iterations=self.qr_iterations, chol_iterations=self.chol_iterations,
                    info=self.info, alpha=self.alpha, beta=self.beta, last_err=self.last_err,
                    ms_total=self.ms_total, ms_bounds=self.ms_bounds, ms_iter=self.ms_iter, ms_h=self.ms_h,
                    flops=self.flops, launches=int(self.launches),
                    con=list(self.con[: min(it, 16)]), err=list(self.err[: min(it, 16)]),
                    branches=[{1: "QR", 2: "CH", 3: "NS"}.get(b, "?")
                              for b in self.branch[: min(it + self.ns_steps, 16)]],
                    flops_executed=self.flops_executed, ns_steps=self.ns_steps, ns_finish=self.ns_finish,
                    ms_step=list(self.ms_step[: min(it, 16)]), ms_finish=self.ms_finish,
                    terms=list(self.terms[: min(it, 16)]))


# (name, restype, argtypes)
_SIGS = [
    ("zolo_version", C.c_char_p, []),
    ("zolo_create", C.c_int, [C.c_int, C.POINTER(C.c_void_p)]),
    ("zolo_destroy", C.c_int, [C.c_void_p]),
    ("zolo_set_stream", C.c_int, [C.c_void_p, C.c_void_p]),
    ("zolo_get_stats", C.c_int, [C.c_void_p, C.POINTER(Stats)]),
    ("zolo_default_handle", C.c_int, [C.POINTER(C.c_void_p)]),
    ("zolo_release_workspace", C.c_int, [C.c_void_p]),
    ("zolo_profile_enable", C.c_int, [C.c_void_p, C.c_int]),
    ("zolo_panel_cluster_size", C.c_int, [C.c_int, C.c_int]),
    ("zolo_profile_read", C.c_int, [C.c_void_p, c_double_p, C.c_int]),
    ("zolo_set_option", C.c_int, [C.c_void_p, C.c_int, C.c_int]),
    ("zolo_get_option", C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_int)]),
    ("zolo_compute_coeff", C.c_int, [C.c_double, C.c_double, C.c_int, c_double_p]),
    ("zolo_compute_coeff_kp", C.c_int, [C.c_double, C.c_double, C.c_int, c_double_p]),
    ("zolo_plan_terms", C.c_int, [C.c_double, C.c_int, C.c_int, C.c_int, C.c_int, C.POINTER(C.c_int),
                                  C.POINTER(C.c_int), C.c_int, C.POINTER(C.c_int)]),
    ("zolo_mellipke", None, [C.c_double, C.c_double, c_double_p, c_double_p]),
    ("zolo_mellipj", None, [C.c_double, C.c_double, C.c_double, c_double_p, c_double_p, c_double_p]),
    ("zolo_choosem", C.c_int, [C.c_double]),
    ("zolo_hfunc", C.c_double, [C.c_double]),
    ("zolo_fone_next", None, [C.c_double, c_double_p, C.c_int, c_double_p, c_double_p]),
    ("zolo_pqdwhfacs", None, [C.c_char, C.c_int, C.c_int, C.c_double, c_double_p, C.c_int, C.c_int, c_int_p,
                              c_double_p, C.c_int, C.c_int, c_int_p, c_double_p, C.c_int, c_int_p, c_double_p,
                              c_double_p, C.c_int, c_int_p, C.c_char]),
    ("zolo_zolopd", None, [C.c_int, C.c_int, C.c_double, c_double_p, C.c_int, C.c_int, c_int_p, c_double_p,
                           C.c_int, C.c_int, c_int_p, c_double_p, C.c_int, c_int_p, c_double_p, c_double_p,
                           C.c_int, c_int_p, C.c_char]),
    ("zolo_pzolopd1", None, [C.c_char, C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, c_double_p, C.c_int,
                             C.c_int, c_int_p, c_double_p, C.c_int, C.c_int, c_int_p, c_int_p, C.c_char]),
    ("zolo_pzolopd2", None, [C.c_char, C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, c_double_p, C.c_int,
                             C.c_int, c_int_p, c_double_p, C.c_int, C.c_int, c_int_p, c_int_p, C.c_char]),
    ("zolo_qdwh_batch_dev", C.c_int, [C.c_void_p, C.c_int, c_int_p, c_int_p, C.POINTER(C.c_void_p),
                                      C.POINTER(C.c_int64), C.POINTER(C.c_void_p), C.POINTER(C.c_int64),
                                      C.POINTER(C.c_void_p), C.POINTER(C.c_int64), c_int_p, c_int_p]),
    ("zolo_polar_dev", C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_int64, C.c_void_p,
                                 C.c_int64, C.c_void_p, C.c_int64]),
    ("zolo_qdwh_dev", C.c_int, [C.c_void_p, C.c_char, C.c_int, C.c_int, C.c_double, C.c_void_p, C.c_int64,
                                C.c_void_p, C.c_int64, C.c_void_p, C.c_int64, C.c_int, C.c_int, C.c_int]),
    ("zolo_pzolopd1_dev", C.c_int, [C.c_void_p, C.c_char, C.c_int, C.c_int, C.c_int, C.c_double, C.c_double,
                                    C.c_void_p, C.c_int64, C.c_void_p, C.c_int64, C.c_void_p, C.c_int64]),
    ("zolo_bounds_dev", C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_double, C.c_void_p, C.c_int64, C.c_int,
                                  c_double_p, c_double_p]),
    ("zolo_form_h_dev", C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_int64, C.c_void_p, C.c_int64,
                                  C.c_void_p, C.c_int64]),
    ("zolo_dgemm_dev", C.c_int, [C.c_void_p, C.c_char, C.c_char, C.c_int, C.c_int, C.c_int, C.c_double,
                                 C.c_void_p, C.c_int64, C.c_void_p, C.c_int64, C.c_double, C.c_void_p, C.c_int64,
                                 C.c_int, C.c_int]),
    ("zolo_ozgemm_dev", C.c_int, [C.c_void_p, C.c_char, C.c_char, C.c_int, C.c_int, C.c_int, C.c_double,
                                  C.c_void_p, C.c_int64, C.c_void_p, C.c_int64, C.c_double, C.c_void_p, C.c_int64,
                                  C.c_int, C.c_int, C.c_int]),
    ("zolo_batch_autotune", C.c_int, [C.c_void_p, c_double_p]),
    ("zolo_batch_stats", C.c_int, [C.c_void_p, c_double_p]),
    ("zolo_batch_schedule", C.c_int, [C.c_int, c_double_p, C.c_int, C.c_int, c_int_p, c_int_p, c_double_p, c_int_p,
                                      c_int_p, c_int_p]),
    ("zolo_batch_set_model", C.c_int, [C.c_void_p, c_double_p]),
    ("zolo_batch_plan", C.c_int, [C.c_int, c_int_p, c_int_p, c_double_p, C.c_int, C.c_int, c_int_p, c_int_p,
                                  c_int_p, c_double_p]),
    ("zolo_read_mm", C.c_int, [C.c_char_p, c_int_p, c_int_p, c_int_p, c_double_p, C.c_int64]),
    ("zolo_dpotrf_dev", C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_int64]),
    ("zolo_dtrsm_dev", C.c_int, [C.c_void_p, C.c_char, C.c_int, C.c_int, C.c_void_p, C.c_int64, C.c_void_p,
                                 C.c_int64, C.c_void_p, C.c_int64]),
    ("zolo_dtrtri_dev", C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_int64, C.c_void_p, C.c_int64]),
    ("zolo_dgeqrf_dev", C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_int64, C.c_void_p,
                                  C.c_void_p]),
    ("zolo_dorgqr_dev", C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_int64, C.c_void_p,
                                  C.c_void_p, C.c_int64]),
    ("zolo_zoloqr_dev", C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_int64, C.c_double, C.c_double,
                                  C.c_void_p, C.c_int64]),
    ("zolo_zolochol_dev", C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_int64, C.c_double, C.c_double,
                                    C.c_void_p, C.c_int64]),
    ("zolo_formx2_dev", C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_double, C.c_void_p, C.c_int64, C.c_void_p,
                                  C.c_int64, c_double_p]),
    ("zolo_dpotrf_noalloc", C.c_int, [C.c_int, C.c_void_p, C.c_int64, C.c_void_p]),
    ("zolo_syev_dev", C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p, C.c_int64]),
    ("zolo_svd_dev", C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_int64, C.c_void_p,
                               C.c_int64, C.c_void_p, C.c_void_p, C.c_int64]),
    ("zolo_zoloeig_dev", C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_int64, C.c_void_p, C.c_int64, c_int_p,
                                   C.c_void_p, C.c_void_p, C.c_int64]),
    ("zolo_zoloeig", None, [C.c_int, C.c_int, c_double_p, c_double_p, C.c_int, C.c_int, c_double_p, C.c_int,
                            c_double_p, C.c_int, c_double_p, c_int_p]),
]

OPT_SHARED_QR = 1
OPT_NS_FINISH = 2
OPT_CHOL_INVERSE = 3
OPT_BETA_FROB = 4
OPT_TERM_PLAN = 5
OPT_MIXED = 6
OPT_MIXED_SLICES = 7
OPT_OWN_BOUNDS = 8
OPT_INJECT_CHOL_FAIL = 9
OPT_NORM2_BOUND = 10
OPT_BATCH_GRAPH = 11
OPT_INJECT_BATCH_ERR = 12
OPT_EIG_ZOLO_MIN = 13
PROFILE_CLASSES = ["dgemm", "qr_panel", "potrf_leaf", "dgemm_m32", "dgemm_n64", "dgemm_rank_k", "dgemm_tri",
                   "ozgemm", "dgemm_k256", "ozgemm_slicing"]

EXPORTED = [s[0] for s in _SIGS] + ["pqdwhfacs_", "zolopd_", "pzolopd1_", "pzolopd2_", "zoloeig_"]


class ZoloError(RuntimeError):
    """A negative INFO from the library (argument error or GPU failure)."""

    def __init__(self, where: str, info: int):
        self.info = info
        if info <= -1000:
            msg = f"{where}: CUDA error {-1000 - info}"
        else:
            msg = f"{where}: INFO = {info}"
        super().__init__(msg)


def lib() -> C.CDLL:
    """Load the CUDA library (built in-tree); raise if it is missing."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: run `python zolo-svd_b200/build.py` "
                               "(this package has no CPU fallback)")
        l = C.CDLL(LIB_PATH)
        for name, res, args in _SIGS:
            f = getattr(l, name)
            f.restype = res
            f.argtypes = args
        _lib = l
    return _lib


def _dp(a: np.ndarray):
    return a.ctypes.data_as(c_double_p)


def _desc(m: int, n: int, nb: int = 64, lld: int | None = None) -> np.ndarray:
    return np.array([1, 0, m, n, nb, nb, 0, 0, max(1, m if lld is None else lld)], dtype=np.int32)


# ---------------------------------------------------------------------------
# host scalar routines
# ---------------------------------------------------------------------------
def compute_coeff(con: float, tol: float, rk: int) -> np.ndarray:
    out = np.zeros(3 * rk)
    r = lib().zolo_compute_coeff(con, tol, rk, _dp(out))
    if r != 0:
        raise ZoloError("zolo_compute_coeff", r)
    return out


def plan_terms(con: float, rk: int, m: int, n: int, prefactored: bool = True, maxlen: int = 16):
    """The term plan from CON on: ([(terms, "QR" | "CH"), ...], predicted Newton-Schulz steps)."""
    terms = (C.c_int * maxlen)()
    qr = (C.c_int * maxlen)()
    ns = C.c_int()
    k = lib().zolo_plan_terms(con, rk, m, n, 1 if prefactored else 0, terms, qr, maxlen, C.byref(ns))
    if k < 0:
        raise ZoloError("zolo_plan_terms", k)
    return [(terms[i], "QR" if qr[i] else "CH") for i in range(k)], ns.value


def compute_coeff_kp(con: float, tol: float, rk: int) -> np.ndarray:
    """Zolotarev coefficients from the complementary modulus 1/con (accurate at any con)."""
    out = np.zeros(3 * rk)
    r = lib().zolo_compute_coeff_kp(con, tol, rk, _dp(out))
    if r != 0:
        raise ZoloError("zolo_compute_coeff_kp", r)
    return out


def hfunc(x: float) -> float:
    return float(lib().zolo_hfunc(x))


def choosem(con: float) -> int:
    return int(lib().zolo_choosem(con))


def fone_next(con: float, coeff: np.ndarray, rk: int) -> tuple[float, float]:
    f, nx = C.c_double(), C.c_double()
    c = np.ascontiguousarray(coeff, dtype=np.float64)
    lib().zolo_fone_next(con, _dp(c), rk, C.byref(f), C.byref(nx))
    return f.value, nx.value


# ---------------------------------------------------------------------------
# reference-named host-array entry points
# ---------------------------------------------------------------------------
def workspace_query(m: int, n: int, nb: int = 64) -> tuple[int, int]:
    """LWORK = -1 query of PQDWHFACS: the minimal LWORK and LWORK2."""
    work = np.zeros(2)
    info = C.c_int(0)
    d = _desc(m, n, nb)
    dw = _desc(2 * n, n, nb)
    dummy = np.zeros(1)
    lib().zolo_pqdwhfacs(b"N", m, n, 0.0, _dp(dummy), 1, 1, d.ctypes.data_as(c_int_p), _dp(dummy), 1, 1,
                         d.ctypes.data_as(c_int_p), _dp(work), -1, dw.ctypes.data_as(c_int_p), _dp(dummy),
                         _dp(dummy), -1, C.byref(info), b"N")
    return int(work[0]), int(work[1])


def pqdwhfacs(sym: str, a: np.ndarray, sigma: float = 0.0, polar: str = "T", nb: int = 64):
    """PQDWHFACS on a host matrix: returns (Q, H or None, INFO)."""
    a = np.asfortranarray(a, dtype=np.float64)
    m, n = a.shape
    lw, lw2 = workspace_query(m, n, nb)
    q = np.zeros((m, n), order="F")
    work = np.zeros(max(lw, 2))
    work2 = np.zeros((max(lw2, n * n),))
    tau = np.zeros(max(n, 1))
    d = _desc(m, n, nb)
    dw = _desc(2 * n, n, nb)
    info = C.c_int(0)
    lib().zolo_pqdwhfacs(sym.encode()[:1], m, n, sigma, _dp(a), 1, 1, d.ctypes.data_as(c_int_p), _dp(q), 1, 1,
                         d.ctypes.data_as(c_int_p), _dp(work), len(work), dw.ctypes.data_as(c_int_p), _dp(tau),
                         _dp(work2), len(work2), C.byref(info), polar.encode()[:1])
    h = None
    if polar.upper().startswith("T") and info.value == 0:
        h = np.asfortranarray(work2[: m * n].reshape((m, n), order="F")[:n, :])
    return q, h, info.value


def zolopd(a: np.ndarray, sigma: float = 0.0, polar: str = "T", nb: int = 64):
    """ZOLOPD on a host matrix: returns (Q, H or None, INFO)."""
    a = np.asfortranarray(a, dtype=np.float64)
    m, n = a.shape
    lw, lw2 = workspace_query(m, n, nb)
    q = np.zeros((m, n), order="F")
    work = np.zeros(max(lw, 2))
    work2 = np.zeros((max(lw2, n * n),))
    tau = np.zeros(max(n, 1))
    d = _desc(m, n, nb)
    dw = _desc(2 * n, n, nb)
    info = C.c_int(0)
    lib().zolo_zolopd(m, n, sigma, _dp(a), 1, 1, d.ctypes.data_as(c_int_p), _dp(q), 1, 1,
                      d.ctypes.data_as(c_int_p), _dp(work), len(work), dw.ctypes.data_as(c_int_p), _dp(tau),
                      _dp(work2), len(work2), C.byref(info), polar.encode()[:1])
    h = None
    if polar.upper().startswith("T") and info.value == 0:
        h = np.asfortranarray(work2[: m * n].reshape((m, n), order="F")[:n, :])
    return q, h, info.value


def pzolopd1(sym: str, rk: int, a: np.ndarray, alpha: float, beta: float, polar: str = "N", nb: int = 64):
    """PZOLOPD1 on a host matrix: returns (Q, INFO)."""
    a = np.asfortranarray(a, dtype=np.float64)
    m, n = a.shape
    q = np.zeros((m, n), order="F")
    d = _desc(m, n, nb)
    info = C.c_int(0)
    lib().zolo_pzolopd1(sym.encode()[:1], rk, m, n, alpha, beta, _dp(a), 1, 1, d.ctypes.data_as(c_int_p), _dp(q),
                        1, 1, d.ctypes.data_as(c_int_p), C.byref(info), polar.encode()[:1])
    return q, info.value


def batch_plan(m, n, model=None, max_batch: int = 1024, mode: int = 0):
    """The bucket plan of the batched solver (host only): (bucket of each member, [(MB, NB)]
    per bucket, predicted ms).  mode 1 = the fixed size ladder."""
    m = np.ascontiguousarray(m, dtype=np.int32)
    n = np.ascontiguousarray(n, dtype=np.int32)
    k = len(n)
    bucket = np.zeros(k, dtype=np.int32)
    mb = np.zeros(max(k, 1), dtype=np.int32)
    nb = np.zeros(max(k, 1), dtype=np.int32)
    pred = C.c_double()
    mdl = None if model is None else np.ascontiguousarray(model, dtype=np.float64)
    r = lib().zolo_batch_plan(k, m.ctypes.data_as(c_int_p), n.ctypes.data_as(c_int_p),
                              None if mdl is None else _dp(mdl), max_batch, mode, bucket.ctypes.data_as(c_int_p),
                              mb.ctypes.data_as(c_int_p), nb.ctypes.data_as(c_int_p), C.byref(pred))
    if r < 0:
        raise ZoloError("zolo_batch_plan", r)
    return bucket, [(int(mb[b]), int(nb[b])) for b in range(r)], pred.value


MM_KINDS = {0: "general", 1: "symmetric", 2: "other"}


def read_mm(path: str):
    """A MatrixMarket file as a dense Fortran-order matrix, the reference's way
    (prepare_real_GEM / prepare_real_symm_MM): returns (A, kind)."""
    m, n, kind = C.c_int(), C.c_int(), C.c_int()
    r = lib().zolo_read_mm(path.encode(), C.byref(m), C.byref(n), C.byref(kind), None, 1)
    if r != 0:
        raise ZoloError("zolo_read_mm", r)
    a = np.zeros((m.value, n.value), order="F")
    r = lib().zolo_read_mm(path.encode(), C.byref(m), C.byref(n), C.byref(kind), _dp(a), max(1, m.value))
    if r != 0:
        raise ZoloError("zolo_read_mm", r)
    return a, MM_KINDS[kind.value]


def pzolopd_f77(sym: str, rk: int, m: int, n: int, alpha: float, beta: float, a_ptr: int, lda: int, q_ptr: int,
                ldq: int, routine: str = "pzolopd1_", nb: int = 64) -> int:
    """PZOLOPD1 / PZOLOPD2 through the gfortran-mangled symbol, as an unchanged Fortran driver
    calls it (test_zolodrv1.f90:198): every argument by reference, hidden CHARACTER lengths
    last, host arrays at raw addresses (column-major, leading dimensions lda, ldq), the
    library's default handle (options from the environment).  Returns INFO."""
    f = getattr(lib(), routine)
    f.restype = None
    da = _desc(m, n, nb, lda)
    dq = _desc(m, n, nb, ldq)
    iv = lambda v: C.byref(C.c_int(v))
    info = C.c_int(0)
    f(C.c_char_p(sym.encode()[:1]), iv(rk), iv(m), iv(n), C.byref(C.c_double(alpha)), C.byref(C.c_double(beta)),
      C.c_void_p(a_ptr), iv(1), iv(1), da.ctypes.data_as(c_int_p), C.c_void_p(q_ptr), iv(1), iv(1),
      dq.ctypes.data_as(c_int_p), C.byref(info), C.c_char_p(b"N"), C.c_size_t(1), C.c_size_t(1))
    return info.value


class DefaultHandle:
    """The library's default handle: the one the reference-named host-array entry points use,
    created on first use with its options read from the environment (ZOLO_FAST,
    ZOLO_OPT_<NAME>, ZOLO_DEVICE).  Never destroyed from here."""

    def __init__(self):
        self.ptr = C.c_void_p()
        r = lib().zolo_default_handle(C.byref(self.ptr))
        if r != 0:
            raise ZoloError("zolo_default_handle", r)

    get_option = lambda self, option: Handle.get_option(self, option)
    stats = lambda self: Handle.stats(self)


# ---------------------------------------------------------------------------
# device-pointer API
# ---------------------------------------------------------------------------
class Handle:
    """A library handle (one CUDA stream, cached workspace)."""

    def __init__(self, device: int = 0):
        self.ptr = C.c_void_p()
        r = lib().zolo_create(device, C.byref(self.ptr))
        if r != 0:
            raise ZoloError("zolo_create", r)

    def close(self):
        if self.ptr:
            lib().zolo_destroy(self.ptr)
            self.ptr = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_stream(self, stream_ptr: int):
        r = lib().zolo_set_stream(self.ptr, C.c_void_p(stream_ptr))
        if r != 0:
            raise ZoloError("zolo_set_stream", r)

    def stats(self) -> dict:
        s = Stats()
        lib().zolo_get_stats(self.ptr, C.byref(s))
        return s.as_dict()

    def release(self):
        lib().zolo_release_workspace(self.ptr)

    def set_option(self, option: int, value: int):
        """Algorithm option of this handle.  OPT_SHARED_QR: 1 (default) = one QR of X
        shared by the Zolotarev terms, 0 = one QR per stacked term as in zoloqr.f90.
        OPT_NS_FINISH: 0 (default) = the reference's stopping rule, 1 = finish with FP64
        Newton-Schulz steps once ||X^T X - I||_F / sqrt(n) <= 5e-3."""
        rc = lib().zolo_set_option(self.ptr, option, value)
        if rc != 0:
            raise ZoloError(f"zolo_set_option({option}, {value})", rc)

    def get_option(self, option: int) -> int:
        v = C.c_int()
        rc = lib().zolo_get_option(self.ptr, option, C.byref(v))
        if rc != 0:
            raise ZoloError(f"zolo_get_option({option})", rc)
        return v.value

    def profile(self, on: bool = True, serialize: bool = False):
        """Per-kernel-class timing on (CUDA events around every launch); serialize: each launch
        timed alone (device synchronized around it)."""
        lib().zolo_profile_enable(self.ptr, (2 if serialize else 1) if on else 0)

    def profile_read(self, reset: bool = True) -> dict:
        """Per kernel class: launches, device ms (CUDA events) and algorithmic flops."""
        out = np.zeros(3 * len(PROFILE_CLASSES))
        lib().zolo_profile_read(self.ptr, _dp(out), 1 if reset else 0)
        names = PROFILE_CLASSES
        return {nm: dict(launches=int(out[3 * i]), ms=float(out[3 * i + 1]), flops=float(out[3 * i + 2]))
                for i, nm in enumerate(names)}


def colmajor_to_device(a: np.ndarray, device="cuda"):
    """Copy an m x n host matrix to a CUDA tensor holding it column-major (ld = m).

    The tensor has shape (n, m): tensor[j, i] == a[i, j].
    """
    import torch
    return torch.from_numpy(np.ascontiguousarray(np.asarray(a, dtype=np.float64).T)).to(device)


def device_to_colmajor(t) -> np.ndarray:
    """Inverse of ``colmajor_to_device``."""
    return np.asfortranarray(t.detach().cpu().numpy().T)


def _ck(name: str, r: int) -> int:
    if r < 0:
        raise ZoloError(name, r)
    return r


def qdwh_dev(h: Handle, sym: str, m: int, n: int, sigma: float, dA: int, lda: int, dQ: int, ldq: int,
             dH: int = 0, ldh: int = 1, bounds_mode: int = 0, maxit: int = 12, left_solve: int = 0) -> int:
    return _ck("zolo_qdwh_dev", lib().zolo_qdwh_dev(h.ptr, sym.encode()[:1], m, n, sigma, dA, lda, dQ, ldq,
                                                   dH or None, ldh, bounds_mode, maxit, left_solve))


def qdwh_batch_dev(h: Handle, members, with_h: bool = True):
    """Batched QDWH-PD on device arrays.  `members` is a list of
    (m, n, dA, lda, dQ, ldq, dH, ldh) with device pointers (dH may be 0 when
    with_h is False).  Returns (info list, iterations list)."""
    k = len(members)
    m = (C.c_int * k)(*[x[0] for x in members])
    n = (C.c_int * k)(*[x[1] for x in members])
    a = (C.c_void_p * k)(*[x[2] for x in members])
    lda = (C.c_int64 * k)(*[x[3] for x in members])
    q = (C.c_void_p * k)(*[x[4] for x in members])
    ldq = (C.c_int64 * k)(*[x[5] for x in members])
    hh = (C.c_void_p * k)(*[x[6] for x in members]) if with_h else None
    ldh = (C.c_int64 * k)(*[x[7] for x in members]) if with_h else None
    info = (C.c_int * k)()
    its = (C.c_int * k)()
    _ck("zolo_qdwh_batch_dev", lib().zolo_qdwh_batch_dev(h.ptr, k, m, n, a, lda, q, ldq, hh, ldh, info, its))
    return list(info), list(its)


BATCH_STATS_KEYS = ("buckets", "max_iterations", "flops", "flops_useful", "ms", "predicted_ms", "graph_replays",
                    "graph_captures", "eager_scheduled", "sync_loops", "restarts", "resumes")


def batch_schedule(l0, maxit: int = 12) -> dict:
    """Step schedule of one batched bucket for members with lower bounds l0
    (zolo_batch_schedule; host only)."""
    k = len(l0)
    l = (C.c_double * max(k, 1))(*l0)
    steps = C.c_int()
    r = lib().zolo_batch_schedule(k, l, maxit, 0, C.byref(steps), None, None, None, None, None)
    if r not in (0, -4):
        raise ZoloError("zolo_batch_schedule", r)
    K = steps.value
    qr = (C.c_int * max(K, 1))()
    tab = (C.c_double * max(5 * k * K, 1))()
    uc, last, cond = (C.c_int * max(k, 1))(), (C.c_int * max(k, 1))(), (C.c_int * max(k, 1))()
    _ck("zolo_batch_schedule", lib().zolo_batch_schedule(k, l, maxit, K, C.byref(steps), qr, tab, uc, last, cond))
    import numpy as _np
    return {"steps": K, "qr": list(qr)[:K], "table": _np.array(tab[:5 * k * K]).reshape(K, 5, k),
            "count": list(uc)[:k], "last": list(last)[:k], "cond": list(cond)[:k]}


def batch_stats(h: Handle) -> dict:
    """Record of the handle's last qdwh_batch_dev call (zolo_batch_stats)."""
    out = (C.c_double * 12)()
    _ck("zolo_batch_stats", lib().zolo_batch_stats(h.ptr, out))
    return {k: (int(v) if k not in ("flops", "flops_useful", "ms", "predicted_ms") else float(v))
            for k, v in zip(BATCH_STATS_KEYS, out)}


def polar_dev(h: Handle, rk: int, m: int, n: int, dA: int, lda: int, dQ: int, ldq: int, dH: int = 0,
              ldh: int = 1) -> int:
    """Bounds + Zolo-PD (+ H) in one call, sharing the QR of A/alpha; returns INFO."""
    return _ck("zolo_polar_dev", lib().zolo_polar_dev(h.ptr, rk, m, n, dA, lda, dQ, ldq, dH or None, ldh))


def pzolopd1_dev(h: Handle, sym: str, rk: int, m: int, n: int, alpha: float, beta: float, dA: int, lda: int,
                 dQ: int, ldq: int, dH: int = 0, ldh: int = 1) -> int:
    return _ck("zolo_pzolopd1_dev", lib().zolo_pzolopd1_dev(h.ptr, sym.encode()[:1], rk, m, n, alpha, beta, dA, lda,
                                                           dQ, ldq, dH or None, ldh))


def syev_dev(h: Handle, n: int, dH: int, ldh: int, dW: int, dZ: int, ldz: int) -> int:
    """Symmetric eigendecomposition (ascending) on device arrays."""
    return _ck("zolo_syev_dev", lib().zolo_syev_dev(h.ptr, n, dH, ldh, dW, dZ, ldz))


def svd_dev(h: Handle, m: int, n: int, dA: int, lda: int, dU: int, ldu: int, dS: int, dV: int, ldv: int,
            algo: int = 0, rk: int = 8) -> int:
    """A = U diag(s) V^T (s ascending) via QDWH-PD (algo 0) or Zolo-PD (algo 1) + eigensolve of H."""
    return _ck("zolo_svd_dev", lib().zolo_svd_dev(h.ptr, algo, rk, m, n, dA, lda, dU, ldu, dS, dV, ldv))


def zoloeig(q: np.ndarray, a: np.ndarray, nblk: int = 64):
    """ZoloEig on host arrays: returns (eigenvalues, eigenvectors, V, V^T A V, INFO)."""
    a = np.asfortranarray(a, dtype=np.float64).copy(order="F")
    q = np.asfortranarray(q, dtype=np.float64).copy(order="F")
    n = a.shape[0]
    work = np.zeros(max(n * n, 1))
    work2 = np.zeros(max(n * n, 1))
    tau = np.zeros(max(n, 1))
    info = C.c_int(0)
    q_in = q.copy(order="F")
    lib().zolo_zoloeig(n, nblk, _dp(q), _dp(a), 0, 0, _dp(work), len(work), _dp(work2), len(work2), _dp(tau),
                       C.byref(info))
    rk = int(round(float(np.linalg.norm((q_in - np.eye(n)) / 2.0) ** 2))) if n else 0
    vecs = work[: n * rk].reshape((n, rk), order="F")
    return tau[:rk].copy(), vecs.copy(), q, a, info.value


def bounds_dev(h: Handle, m: int, n: int, dA: int, lda: int, mode: int = 1, sigma: float = 0.0):
    al, be = C.c_double(), C.c_double()
    r = lib().zolo_bounds_dev(h.ptr, m, n, sigma, dA, lda, mode, C.byref(al), C.byref(be))
    return al.value, be.value, _ck("zolo_bounds_dev", r)
