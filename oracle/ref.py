"""ctypes bindings of oracle/_ref/libref.so: the reference's own FluidModule and
InitialModule compiled from its unmodified headers (oracle/Makefile, target
``ref``; linear solves by refshim/solverFuncs.hpp, the exact box-union solve).

TEST INFRASTRUCTURE ONLY (the checker).  tests/ use it to pin the CPU
restatement (oracle/fluid.py) and the device path to the reference itself.

Arrays follow the reference: float64 (ni+2, nj+2), indexed [i][j].
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_ref", "libref.so")
# the same driver with the product's GPU drop-in (include/cathode_solver.hpp) as solverFuncs.hpp
DROPIN_PATH = os.path.join(_HERE, "_ref", "libref_dropin.so")
_LIBS: dict = {}

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)
_vp = ctypes.c_void_p
_cs = ctypes.c_char_p

# FluidModule methods reachable through RefCase.call (fluidModule.hpp:35-49) and "step"
METHODS = ("check_CFL", "solve_Uix_tmp", "solve_Uir_tmp", "solve_Uip_tmp", "solve_rhoi_constTe",
           "correct_Ui_constTe", "solve_phi_couple_wdTe_wSEE_PC", "solve_rhoe_wdTe_wSEE_PC",
           "solve_Te_wdTe_wSEE_PC", "update_rhon", "update_rhom", "update_transport_coef", "step")
MW_LISTS = tuple(f"Bnd{s}{f}" for f in "xrp" for s in "WESN")


def reference_dir() -> str:
    """The reference checkout used by the build recipe (env CATHODE_REFERENCE)."""
    return os.environ.get("CATHODE_REFERENCE", "/root/reference")


def build(force: bool = False) -> str | None:
    """Build libref.so (and libref_dropin.so, once the product library exists) when the
    reference sources are present; returns the path of libref.so or None."""
    ref = reference_dir()
    if not os.path.isdir(os.path.join(ref, "include")):
        return LIB_PATH if os.path.exists(LIB_PATH) else None
    targets = ["ref"]
    if os.path.exists(os.path.join(_HERE, "..", "02_cathode-08_modulerev_b200", "libcathode_b200.so")):
        targets.append("ref-dropin")
    args = ["make", "-C", _HERE, "-s", f"REF={ref}"] + targets
    if force:
        args.insert(1, "-B")
    subprocess.run(args, check=True, stderr=subprocess.DEVNULL)
    return LIB_PATH


def available(dropin: bool = False) -> bool:
    return os.path.exists(DROPIN_PATH if dropin else LIB_PATH)


def lib(dropin: bool = False) -> ctypes.CDLL:
    key = "dropin" if dropin else "exact"
    if key not in _LIBS:
        path = DROPIN_PATH if dropin else LIB_PATH
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} not built (needs the reference sources; oracle/Makefile ref)")
        L = ctypes.CDLL(path)
        L.ref_create.argtypes = [ctypes.c_int, ctypes.c_int]
        L.ref_create.restype = _vp
        L.ref_destroy.argtypes = [_vp]
        L.ref_set_quiet.argtypes = [_vp, ctypes.c_int]
        L.ref_set_param.argtypes = [_vp, _cs, ctypes.c_double]
        L.ref_get_param.argtypes = [_vp, _cs, _dp]
        L.ref_set_field.argtypes = [_vp, _cs, _dp]
        L.ref_get_field.argtypes = [_vp, _cs, _dp]
        L.ref_get_int_field.argtypes = [_vp, _cs, _ip]
        L.ref_set_table.argtypes = [_vp, _cs, _dp, ctypes.c_int]
        L.ref_table_size.argtypes = [_vp, _cs]
        L.ref_get_table.argtypes = [_vp, _cs, _dp]
        L.ref_make_boundary.argtypes = [_vp]
        L.ref_mw_list.argtypes = [_vp, _cs, _ip, ctypes.c_int]
        L.ref_call.argtypes = [_vp, _cs]
        L.ref_solver_mode.argtypes = [ctypes.c_int]
        L.ref_solver_mode.restype = None
        L.ref_capture.argtypes = [ctypes.c_int]
        L.ref_capture.restype = None
        L.ref_captured_plane.argtypes = [ctypes.c_int, ctypes.c_int, _dp, ctypes.c_int]
        L.ref_captured_blocks.argtypes = [ctypes.c_int, _ip, _ip, ctypes.c_int]
        L.ref_dropin_precision.argtypes = [ctypes.c_int]
        L.ref_dropin_stats.argtypes = [ctypes.POINTER(ctypes.c_long), ctypes.POINTER(ctypes.c_long),
                                       ctypes.POINTER(ctypes.c_double)]
        L.ref_output.argtypes = [_vp, _cs]
        L.ref_set_cfield.argtypes = [_vp, _cs, _dp]
        L.ref_get_cfield.argtypes = [_vp, _cs, _dp]
        L.ref_set_sparam.argtypes = [_vp, ctypes.c_int, ctypes.c_double, ctypes.c_double]
        L.ref_microwave.argtypes = [_vp, _cs, ctypes.c_double, ctypes.c_int, _dp]
        _LIBS[key] = L
    return _LIBS[key]


class RefCase:
    """One reference state (Params + GridCenter + GridInterfaceX/R + MicrowaveBC + tables)."""

    def __init__(self, ni: int, nj: int, quiet: bool = True, dropin: bool = False):
        """dropin=True: the reference's solves go to the product's GPU drop-in."""
        self.ni, self.nj = int(ni), int(nj)
        self._L = lib(dropin)
        self._h = self._L.ref_create(self.ni, self.nj)
        if not self._h:
            raise ValueError("ref_create failed")
        self._L.ref_set_quiet(self._h, int(quiet))

    def close(self):
        if self._h:
            self._L.ref_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # parameters -------------------------------------------------------------------------------
    def set_param(self, name: str, value: float) -> bool:
        return self._L.ref_set_param(self._h, name.encode(), float(value)) == 0

    def set_params(self, prm: dict) -> list:
        """Set every scalar entry of prm that is a Params member; returns the names not taken."""
        skipped = []
        for k, v in prm.items():
            if isinstance(v, (int, float, np.integer, np.floating)) and not isinstance(v, bool):
                if not self.set_param(k, v):
                    skipped.append(k)
            else:
                skipped.append(k)
        return skipped

    def param(self, name: str) -> float:
        v = ctypes.c_double()
        if self._L.ref_get_param(self._h, name.encode(), ctypes.byref(v)) != 0:
            raise KeyError(name)
        return v.value

    # planes -----------------------------------------------------------------------------------
    def set_field(self, name: str, a) -> None:
        a = np.ascontiguousarray(a, dtype=np.float64)
        if a.shape != (self.ni + 2, self.nj + 2):
            raise ValueError(f"{name}: shape {a.shape}")
        if self._L.ref_set_field(self._h, name.encode(), a.ctypes.data_as(_dp)) != 0:
            raise KeyError(name)

    def set_fields(self, fields: dict, names=None) -> list:
        skipped = []
        for k in (names or fields):
            v = fields[k]
            if isinstance(v, np.ndarray) and v.shape == (self.ni + 2, self.nj + 2):
                try:
                    self.set_field(k, v)
                except KeyError:
                    skipped.append(k)
            else:
                skipped.append(k)
        return skipped

    def field(self, name: str) -> np.ndarray:
        out = np.empty((self.ni + 2, self.nj + 2))
        if self._L.ref_get_field(self._h, name.encode(), out.ctypes.data_as(_dp)) != 0:
            raise KeyError(name)
        return out

    def int_field(self, name: str) -> np.ndarray:
        out = np.empty((self.ni + 2, self.nj + 2), np.int32)
        if self._L.ref_get_int_field(self._h, name.encode(), out.ctypes.data_as(_ip)) != 0:
            raise KeyError(name)
        return out

    def blocks(self, which: str, n: int = 6):
        """Block table (i_bl, j_bl) as (n, 2) arrays; which = 'flc', 'flx' or 'flr'."""
        return self.int_field(f"i_{which}_bl")[:n, :2].copy(), self.int_field(f"j_{which}_bl")[:n, :2].copy()

    # tables -----------------------------------------------------------------------------------
    def set_table(self, name: str, v) -> None:
        v = np.ascontiguousarray(v, dtype=np.float64)
        if self._L.ref_set_table(self._h, name.encode(), v.ctypes.data_as(_dp), v.size) != 0:
            raise KeyError(name)

    def table(self, name: str) -> np.ndarray:
        n = self._L.ref_table_size(self._h, name.encode())
        if n < 0:
            raise KeyError(name)
        out = np.empty(n)
        self._L.ref_get_table(self._h, name.encode(), out.ctypes.data_as(_dp))
        return out

    # geometry and methods ---------------------------------------------------------------------
    def make_boundary(self) -> None:
        self._L.ref_make_boundary(self._h)

    def mw_list(self, name: str) -> np.ndarray:
        """(n, 3) array of (i, j, code) of one MicrowaveBC list, e.g. 'BndWx'."""
        cols = []
        for p in "ijs":
            n = self._L.ref_mw_list(self._h, (p + name).encode(), None, 0)
            if n < 0:
                raise KeyError(name)
            buf = np.empty(max(n, 1), np.int32)
            self._L.ref_mw_list(self._h, (p + name).encode(), buf.ctypes.data_as(_ip), n)
            cols.append(buf[:n])
        return np.stack(cols, axis=1)

    def set_cfield(self, name: str, a) -> None:
        """A complex plane (E1x, E1r, E1p, J1x, J1r, J1p, J1x_exc, J1r_exc, J1p_exc)."""
        a = np.ascontiguousarray(a, dtype=np.complex128)
        if a.shape != (self.ni + 2, self.nj + 2):
            raise ValueError(f"{name}: shape {a.shape}")
        if self._L.ref_set_cfield(self._h, name.encode(), a.view(np.float64).ctypes.data_as(_dp)) != 0:
            raise KeyError(name)

    def cfield(self, name: str) -> np.ndarray:
        out = np.empty((self.ni + 2, self.nj + 2), np.complex128)
        if self._L.ref_get_cfield(self._h, name.encode(), out.view(np.float64).ctypes.data_as(_dp)) != 0:
            raise KeyError(name)
        return out

    def set_sparams(self, S11, S21, S12, S22) -> None:
        for k, v in enumerate((S11, S21, S12, S22)):
            self._L.ref_set_sparam(self._h, k, complex(v).real, complex(v).imag)

    def microwave(self, which: str, tol: float = 1e-12, maxit: int = 2000) -> dict:
        """The drop-in's EmfieldModule::solve_Microwave or update_energy_profile (drop-in build)."""
        out = (ctypes.c_double * 3)()
        rc = self._L.ref_microwave(self._h, which.encode(), float(tol), int(maxit), out)
        if rc != 0:
            raise RuntimeError(f"{which}: drop-in microwave call failed ({rc})")
        return dict(iterations=int(out[0]), residual=out[1], converged=int(out[2]))

    def output(self, directory: str) -> str:
        """OutputModule::output into directory/results; returns the restart file's path."""
        n = int(self.param("nOut"))
        if self._L.ref_output(self._h, os.fsencode(directory)) != 0:
            raise OSError("ref_output failed")
        return os.path.join(directory, "results", f"restart{n}.csv")

    def call(self, method: str) -> int:
        rc = self._L.ref_call(self._h, method.encode())
        if rc < 0:
            raise KeyError(method)
        if rc:
            raise RuntimeError(f"{method}: a linear solve failed (zero pivot)")
        return rc


def solver_mode(mode: int) -> None:
    """0 = exact solve for solver_SMG (default), 1 = the oracle's SMG restatement."""
    lib().ref_solver_mode(int(mode))


def solve_calls() -> int:
    return lib().ref_solve_calls()


def capture(on: bool = True) -> None:
    lib().ref_capture(int(on))


def captured_planes(ni: int, nj: int) -> list:
    """Recorded systems of a (ni, nj) case: dicts aP, aE, aW, aN, aS, b, i_bl, j_bl."""
    L = lib()
    out = []
    n = (ni + 2) * (nj + 2)
    for s in range(L.ref_captured_count()):
        d = {}
        for k, name in enumerate(("aP", "aE", "aW", "aN", "aS", "b")):
            buf = np.empty((ni + 2, nj + 2))
            if L.ref_captured_plane(s, k, buf.ctypes.data_as(_dp), n) != 0:
                raise ValueError("captured system has another size")
            d[name] = buf
        ib = np.empty(16, np.int32)
        jb = np.empty(16, np.int32)
        nb = L.ref_captured_blocks(s, ib.ctypes.data_as(_ip), jb.ctypes.data_as(_ip), 8)
        d["i_bl"], d["j_bl"] = ib[:2 * nb].reshape(nb, 2).copy(), jb[:2 * nb].reshape(nb, 2).copy()
        out.append(d)
    return out


def dropin_stats() -> dict:
    """The GPU drop-in's solve counts since the last call: calls, not_converged (maxITR
    reached above the tolerance), worst (largest final relative residual of those)."""
    c, n, w = ctypes.c_long(), ctypes.c_long(), ctypes.c_double()
    if lib(True).ref_dropin_stats(ctypes.byref(c), ctypes.byref(n), ctypes.byref(w)) != 0:
        raise RuntimeError("not the drop-in build")
    return dict(calls=c.value, not_converged=n.value, worst=w.value)


def dropin_precision(p: int) -> None:
    """Precision of the GPU drop-in's solver_SMG: 1 mixed (FP32 cycles + FP64 defect correction), 0 FP64."""
    if lib(True).ref_dropin_precision(int(p)) != 0:
        raise RuntimeError("not the drop-in build")
