"""The C-ABI library without a GPU: it loads, exports every declared symbol, its
host scalar code matches the oracle bit for bit, and argument errors return the
reference's INFO codes before any device work."""
import ctypes as C
import os
import re

import numpy as np
import pytest

import zolo_svd_b200 as zb
from oracle import zolo_oracle as zo

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
HEADER = os.path.join(ROOT, "include", "zolo_b200.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    names = re.findall(r"^\s*(?:const\s+)?[\w\s\*]+?\b(\w+)\s*\(", src, flags=re.M)
    return sorted(set(n for n in names if n not in ("defined",)))


def test_library_loads_and_exports_all_declared_symbols():
    lib = zb.lib()
    names = declared_functions()
    assert len(names) >= 30
    for n in names:
        assert hasattr(lib, n), f"{n} declared in zolo_b200.h but not exported"
    for n in zb.EXPORTED:
        assert n in names, f"{n} bound in Python but not declared"


def test_version():
    assert b"sm_100a" in zb.lib().zolo_version()


@pytest.mark.parametrize("con", [1.5, 10.0, 1e2, 1e4, 1e8, 1e12, 1e16])
@pytest.mark.parametrize("rk", [1, 2, 3, 5, 8])
def test_compute_coeff_bitwise_equals_oracle(con, rk):
    c_lib = zb.compute_coeff(con, zo.EPS, rk)
    c_ora = zo.compute_coeff(con, zo.EPS, rk)
    np.testing.assert_array_equal(c_lib, c_ora)
    f_lib, n_lib = zb.fone_next(con, c_lib, rk)
    f_ora = zo.zolo_fone(c_ora, rk)
    assert f_lib == f_ora
    assert n_lib == zo.zolo_next_con(con, c_ora, rk, f_ora)


def test_hfunc_and_choosem_bitwise():
    for x in [1e-16, 1e-12, 1e-8, 1e-3, 0.1, 0.5, 0.9, 0.999999, 1.0]:
        assert zb.hfunc(x) == zo.hfunc(x)
    for con in [1.0001, 1.005, 1.05, 1.15, 1.3, 1.8, 3.0, 100.0, 1e4, 1e6, 1e8, 1e11, 1e14]:
        assert zb.choosem(con) == zo.choosem(con)


def test_mellip_bitwise():
    lib = zb.lib()
    for con in [2.0, 1e3, 1e9]:
        alpha = np.arccos(1.0 / con)
        k, e = C.c_double(), C.c_double()
        lib.zolo_mellipke(alpha, zo.EPS, C.byref(k), C.byref(e))
        assert (k.value, e.value) == zo.mellipke(alpha, zo.EPS)
        sn, cn, dn = C.c_double(), C.c_double(), C.c_double()
        lib.zolo_mellipj(0.3 * k.value, alpha, zo.EPS, C.byref(sn), C.byref(cn), C.byref(dn))
        assert (sn.value, cn.value, dn.value) == zo.mellipj(0.3 * k.value, alpha, zo.EPS)


def test_workspace_query_matches_reference_formula():
    # pqdwhfacs.f90:262-278 on a 1x1 grid: LWIN = max(5N+NB+1, 2N^2, 2MN), LWIN2 = max(NB(3N+NB)+1, MN)
    for n, nb in [(10, 4), (100, 64), (1024, 64)]:
        lw, lw2 = zb.workspace_query(n, n, nb)
        assert lw == max(5 * n + nb + 1, 2 * n * n)
        assert lw2 == max(nb * (3 * n + nb) + 1, n * n)


def test_argument_errors_before_device_work():
    a = np.zeros((3, 5))  # M < N
    q, h, info = zb.pqdwhfacs("N", a)
    assert info == -1
    q, info = zb.pzolopd1("N", 9, np.eye(4), 1.0, 0.5)
    assert info == -2  # RK outside 1..8
    q, info = zb.pzolopd1("N", 2, np.zeros((3, 5)), 1.0, 0.5)
    assert info == -3
    q, info = zb.pzolopd1("N", 2, np.eye(4), 0.0, 0.5)
    assert info == -5
    q, info = zb.pzolopd1("N", 2, np.eye(4), 1.0, -1.0)
    assert info == -6


def test_descriptor_validation():
    lib = zb.lib()
    n = 4
    a = np.asfortranarray(np.eye(n))
    q = np.zeros((n, n), order="F")
    work = np.zeros(100)
    work2 = np.zeros(100)
    tau = np.zeros(n)
    info = C.c_int(0)
    good = np.array([1, 0, n, n, 2, 2, 0, 0, n], dtype=np.int32)
    bad = good.copy()
    bad[0] = 2  # DTYPE_ must be 1
    ip = lambda d: d.ctypes.data_as(zb.c_int_p)
    lib.zolo_pqdwhfacs(b"N", n, n, 0.0, zb._dp(a), 1, 1, ip(bad), zb._dp(q), 1, 1, ip(good), zb._dp(work), 100,
                       ip(good), zb._dp(tau), zb._dp(work2), 100, C.byref(info), b"N")
    assert info.value == -801
    bad = good.copy()
    bad[8] = 1  # LLD_ < M
    lib.zolo_pqdwhfacs(b"N", n, n, 0.0, zb._dp(a), 1, 1, ip(good), zb._dp(q), 1, 1, ip(bad), zb._dp(work), 100,
                       ip(good), zb._dp(tau), zb._dp(work2), 100, C.byref(info), b"N")
    assert info.value == -1209
    lib.zolo_pqdwhfacs(b"N", n, n, 0.0, zb._dp(a), 2, 1, ip(good), zb._dp(q), 1, 1, ip(good), zb._dp(work), 100,
                       ip(good), zb._dp(tau), zb._dp(work2), 100, C.byref(info), b"N")
    assert info.value == -6
    # LWORK too small -> -12, LWORK2 too small -> -16 (pqdwhfacs.f90:286-294)
    lib.zolo_pqdwhfacs(b"N", n, n, 0.0, zb._dp(a), 1, 1, ip(good), zb._dp(q), 1, 1, ip(good), zb._dp(work), 5,
                       ip(good), zb._dp(tau), zb._dp(work2), 100, C.byref(info), b"N")
    assert info.value == -12
    lib.zolo_pqdwhfacs(b"N", n, n, 0.0, zb._dp(a), 1, 1, ip(good), zb._dp(q), 1, 1, ip(good), zb._dp(work), 100,
                       ip(good), zb._dp(tau), zb._dp(work2), 3, C.byref(info), b"N")
    assert info.value == -16


def test_fortran_symbol_query_path():
    """pqdwhfacs_ with the gfortran calling convention: LWORK = -1 query fills WORK(1:2)."""
    lib = zb.lib()
    f = lib.pqdwhfacs_
    f.restype = None
    n = 8
    iv = lambda v: C.byref(C.c_int(v))
    d = np.array([1, 0, n, n, 4, 4, 0, 0, n], dtype=np.int32)
    dw = np.array([1, 0, 2 * n, n, 4, 4, 0, 0, 2 * n], dtype=np.int32)
    work = np.zeros(2)
    dummy = np.zeros(1)
    info = C.c_int(7)
    f(C.c_char_p(b"N"), iv(n), iv(n), C.byref(C.c_double(0.0)), zb._dp(dummy), iv(1), iv(1),
      d.ctypes.data_as(zb.c_int_p), zb._dp(dummy), iv(1), iv(1), d.ctypes.data_as(zb.c_int_p), zb._dp(work), iv(-1),
      dw.ctypes.data_as(zb.c_int_p), zb._dp(dummy), zb._dp(dummy), iv(-1), C.byref(info), C.c_char_p(b"N"),
      C.c_size_t(1), C.c_size_t(1))
    assert info.value == 0
    assert work[0] == max(5 * n + 4 + 1, 2 * n * n)
    assert work[1] == max(4 * (3 * n + 4) + 1, n * n)


def test_fortran_interface_module_matches_header():
    """include/zolo_b200.f90 binds only exported C names, with the header's option values and
    the argument counts of the C prototypes (no Fortran compiler here: checked as text)."""
    import os
    import re
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    f90 = open(os.path.join(root, "include", "zolo_b200.f90")).read()
    hdr = open(os.path.join(root, "include", "zolo_b200.h")).read()
    lib = zb.lib()
    binds = re.findall(r'(?:subroutine|function)\s+(\w+)\(([^)]*)\)[^\n]*?(?:&\s*\n[^\n]*?)?bind\(C, name="(\w+)"\)',
                       f90)
    assert len(binds) >= 12
    for fname, args, cname in binds:
        assert fname == cname
        assert hasattr(lib, cname), cname
        proto = re.search(r"\b" + cname + r"\(([^;]*)\);", hdr)
        assert proto, cname
        n_c = len([x for x in proto.group(1).split(",") if x.strip()])
        n_f = len([x for x in args.replace("&", "").split(",") if x.strip()])
        assert n_c == n_f, (cname, n_c, n_f)
    for name, val in re.findall(r"integer\(c_int\), parameter :: (ZOLO_OPT_\w+) = (\d+)", f90):
        assert re.search(r"#define " + name + r" " + val + r"\b", hdr), name
