"""Two-port helpers of the microwave feed (host): CmpMat2 (include/cmpMat2.hpp),
InitialModule::sParamToABCD / ABCDToSParam (include/initialModule.hpp:1689-1739)
and the S-parameter set-up with stub and cable corrections
(include/initialModule.hpp:107-192), through the library's C ABI.  Matrices are
2x2 complex numpy arrays [[A, B], [C, D]]; errors where the reference throws
raise CathodeError."""
from __future__ import annotations

import ctypes

import numpy as np

from . import capi

_C2 = ctypes.c_double * 2


def _c2(z) -> "ctypes.Array":
    z = complex(z)
    return _C2(z.real, z.imag)


def _m_in(T) -> capi.CMat2:
    T = np.asarray(T, dtype=complex)
    m = capi.CMat2()
    for k, z in zip(("A", "B", "C", "D"), (T[0, 0], T[0, 1], T[1, 0], T[1, 1])):
        setattr(m, k, _c2(z))
    return m


def _m_out(m: capi.CMat2) -> np.ndarray:
    v = [complex(getattr(m, k)[0], getattr(m, k)[1]) for k in ("A", "B", "C", "D")]
    return np.array([[v[0], v[1]], [v[2], v[3]]])


def cmat2_mul(X, Y) -> np.ndarray:
    out = capi.CMat2()
    capi.check(capi.load().cth_cmat2_mul(ctypes.byref(_m_in(X)), ctypes.byref(_m_in(Y)), ctypes.byref(out)),
               allow_positive=False)
    return _m_out(out)


def cmat2_inv(X) -> np.ndarray:
    out = capi.CMat2()
    capi.check(capi.load().cth_cmat2_inv(ctypes.byref(_m_in(X)), ctypes.byref(out)), allow_positive=False)
    return _m_out(out)


def sparam_to_abcd(S11, S21, S12, S22, Z0: float) -> np.ndarray:
    out = capi.CMat2()
    args = [_c2(z) for z in (S11, S21, S12, S22)]
    capi.check(capi.load().cth_sparam_to_abcd(*[ctypes.byref(a) for a in args], Z0, ctypes.byref(out)),
               allow_positive=False)
    return _m_out(out)


def abcd_to_sparam(T, Z0: float):
    s = [_C2() for _ in range(4)]
    capi.check(capi.load().cth_abcd_to_sparam(ctypes.byref(_m_in(T)), Z0, *[ctypes.byref(a) for a in s]),
               allow_positive=False)
    return tuple(complex(a[0], a[1]) for a in s)


def sparam_setup(prm: dict):
    """(S11, S21, S12, S22) after the stub and cable corrections, and the cable phase (deg)."""
    p = capi.SParamParams(**{k: prm[k] for k, _ in capi.SParamParams._fields_})
    S = (_C2 * 4)()
    ph = ctypes.c_double()
    capi.check(capi.load().cth_sparam_setup(ctypes.byref(p), ctypes.byref(S), ctypes.byref(ph)), allow_positive=False)
    return tuple(complex(S[k][0], S[k][1]) for k in range(4)), ph.value
