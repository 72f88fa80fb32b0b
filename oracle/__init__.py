"""ctypes bindings of the CPU oracle (oracle/liboracle.so).

TEST INFRASTRUCTURE ONLY.  tests/, ``__graft_entry__.smoke()`` and bench.py's
CPU-baseline / reference legs import this module as the checker or as the
timed CPU baseline; the product package never imports it.

All arrays follow the reference's [i][j] convention: numpy float64 arrays of
shape (ni+2, nj+2), C-contiguous (i = axial index, j = radial index).
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)
_u8p = ctypes.POINTER(ctypes.c_ubyte)


def build(force: bool = False) -> str:
    """Compile liboracle.so with the Makefile and, when the reference sources are
    present, the checker library oracle/_ref/libref.so compiled from them (ref.py)."""
    so = os.path.join(_HERE, "liboracle.so")
    if force or not os.path.exists(so) or _stale(so):
        subprocess.run(["make", "-C", _HERE, "-s"], check=True)
    from . import ref
    ref.build(force=force)
    return so


def _stale(so: str) -> bool:
    t = os.path.getmtime(so)
    for f in os.listdir(_HERE):
        if f.endswith((".c", ".h")) and os.path.getmtime(os.path.join(_HERE, f)) > t:
            return True
    return False


def lib() -> ctypes.CDLL:
    global _LIB
    if _LIB is None:
        so = os.path.join(_HERE, "liboracle.so")
        if not os.path.exists(so):
            build()
        _LIB = ctypes.CDLL(so)
        _declare(_LIB)
    return _LIB


def _declare(L):
    f = L.orc_active_mask
    f.argtypes = [ctypes.c_int, ctypes.c_int, _ip, _ip, ctypes.c_int, _u8p]
    f.restype = None
    L.orc_struct5_residual.argtypes = [ctypes.c_int, ctypes.c_int, _ip, _ip, ctypes.c_int] + [_dp] * 8 + [_dp, _dp]
    L.orc_struct5_residual.restype = None
    L.orc_struct5_direct.argtypes = [ctypes.c_int, ctypes.c_int, _ip, _ip, ctypes.c_int] + [_dp] * 7
    L.orc_struct5_direct.restype = ctypes.c_int
    L.orc_smg_solve.argtypes = ([ctypes.c_int, ctypes.c_int, _ip, _ip, ctypes.c_int] + [_dp] * 6 +
                                [ctypes.c_int, ctypes.c_double, ctypes.c_int, ctypes.c_int, _dp, _ip, _dp])
    L.orc_smg_solve.restype = ctypes.c_int
    L.orc_sor_solve.argtypes = ([ctypes.c_int, ctypes.c_int, _ip, _ip, ctypes.c_int] + [_dp] * 6 +
                                [ctypes.c_double, ctypes.c_int, ctypes.c_double, _dp, _ip, _dp])
    L.orc_sor_solve.restype = None
    L.orc_calc_res.argtypes = [ctypes.c_int, ctypes.c_int, _ip, _ip, ctypes.c_int, _dp, _dp,
                               ctypes.c_double, ctypes.c_int]
    L.orc_calc_res.restype = ctypes.c_double
    for name in ("orc_exp", "orc_erf"):
        getattr(L, name).argtypes = [ctypes.c_size_t, _dp, _dp]
        getattr(L, name).restype = None


def _elementwise(name, x):
    a = np.array(x, dtype=np.float64, order="C")   # keeps 0-d inputs 0-d
    out = np.empty_like(a)
    getattr(lib(), name)(a.size, a.ctypes.data_as(_dp), out.ctypes.data_as(_dp))
    return out if out.ndim else float(out)


def libm_exp(x):
    """exp() of the C library, element-wise (the reference's exp)."""
    return _elementwise("orc_exp", x)


def libm_erf(x):
    """erf() of the C library, element-wise (the reference's erf)."""
    return _elementwise("orc_erf", x)


def _d(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(_dp)


def _blocks(i_bl, j_bl):
    ib = np.ascontiguousarray(np.asarray(i_bl, dtype=np.int32).reshape(-1))
    jb = np.ascontiguousarray(np.asarray(j_bl, dtype=np.int32).reshape(-1))
    return ib, jb, ib.size // 2


def active_mask(ni, nj, i_bl, j_bl):
    ib, jb, nb = _blocks(i_bl, j_bl)
    m = np.zeros((ni + 2, nj + 2), dtype=np.uint8)
    lib().orc_active_mask(ni, nj, ib.ctypes.data_as(_ip), jb.ctypes.data_as(_ip), nb,
                          m.ctypes.data_as(_u8p))
    return m


def residual(sysd, x):
    """Return (r, ||r||_2, ||b||_2) of the box-union system for solution x."""
    ni, nj = sysd["ni"], sysd["nj"]
    ib, jb, nb = _blocks(sysd["i_bl"], sysd["j_bl"])
    r = np.zeros_like(x)
    rr = ctypes.c_double()
    bb = ctypes.c_double()
    lib().orc_struct5_residual(ni, nj, ib.ctypes.data_as(_ip), jb.ctypes.data_as(_ip), nb,
                               *[_d(sysd[k]) for k in ("aP", "aE", "aW", "aN", "aS", "b")],
                               _d(np.ascontiguousarray(x)), _d(r), ctypes.byref(rr), ctypes.byref(bb))
    return r, float(np.sqrt(rr.value)), float(np.sqrt(bb.value))


def direct_solve(sysd, solution=None):
    ni, nj = sysd["ni"], sysd["nj"]
    ib, jb, nb = _blocks(sysd["i_bl"], sysd["j_bl"])
    x = np.zeros((ni + 2, nj + 2)) if solution is None else solution
    rc = lib().orc_struct5_direct(ni, nj, ib.ctypes.data_as(_ip), jb.ctypes.data_as(_ip), nb,
                                  *[_d(sysd[k]) for k in ("aP", "aE", "aW", "aN", "aS", "b")], _d(x))
    if rc != 0:
        raise RuntimeError("oracle direct solve failed (zero pivot)")
    return x


def smg_solve(sysd, maxITR=30, error_cnv=1e-10, nu1=1, nu2=1, solution=None):
    ni, nj = sysd["ni"], sysd["nj"]
    ib, jb, nb = _blocks(sysd["i_bl"], sysd["j_bl"])
    x = np.zeros((ni + 2, nj + 2)) if solution is None else solution
    it = ctypes.c_int()
    rel = ctypes.c_double()
    rc = lib().orc_smg_solve(ni, nj, ib.ctypes.data_as(_ip), jb.ctypes.data_as(_ip), nb,
                             *[_d(sysd[k]) for k in ("aP", "aE", "aW", "aN", "aS", "b")],
                             maxITR, error_cnv, nu1, nu2, _d(x), ctypes.byref(it), ctypes.byref(rel))
    return x, rc, it.value, rel.value


def sor_solve(sysd, alpha=1.9, maxITR=2000, error_cnv=1e-8, solution=None):
    ni, nj = sysd["ni"], sysd["nj"]
    ib, jb, nb = _blocks(sysd["i_bl"], sysd["j_bl"])
    x = np.zeros((ni + 2, nj + 2)) if solution is None else solution
    n = ctypes.c_int()
    e = ctypes.c_double()
    lib().orc_sor_solve(ni, nj, ib.ctypes.data_as(_ip), jb.ctypes.data_as(_ip), nb,
                        *[_d(sysd[k]) for k in ("aP", "aE", "aW", "aN", "aS", "b")],
                        alpha, maxITR, error_cnv, _d(x), ctypes.byref(n), ctypes.byref(e))
    return x, n.value, e.value


def calc_res(ni, nj, i_bl, j_bl, val_new, val_old, EPS, flag_error):
    ib, jb, nb = _blocks(i_bl, j_bl)
    return lib().orc_calc_res(ni, nj, ib.ctypes.data_as(_ip), jb.ctypes.data_as(_ip), nb,
                              _d(val_new), _d(val_old), EPS, flag_error)
