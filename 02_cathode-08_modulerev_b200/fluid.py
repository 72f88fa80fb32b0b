"""Fluid state in HBM and the FluidModule kernels, over the C ABI.

``Fields`` owns a cth_fields store on a Grid: named device planes (the
reference's member names), the per-cell side flags of the fluid blocks and the
BolsigVec rate tables.  ``geometry`` helpers build the side flags for the
reference's cathode block layout (initialModule.hpp:219-263 with the flag
expressions repeated in every FluidModule sweep, e.g. fluidModule.hpp:2660-2686)
or for the r-z rectangle of the synthetic workloads.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import capi

F_BLX, F_BRX, F_BLR_WALL, F_BLR_CEN, F_BRR_WALL, F_BRR_OPEN = 1, 2, 4, 8, 16, 32
F_BRX_BIAS = 64  # the right wall of the cell is the biased electrode
TABLES = ("nu_elas_N", "nu_exc_N", "nu_excReso_N", "nu_excMeta_N", "nu_ionz_N", "nu_ionzStep_N",
          "nu_excStep_N", "nu_super_N", "rate_eloss_n_N", "rate_eloss_m_N", "nui_m_N")


def cathode_blocks(ni=194, nj=70, xR=0.0388, rmax=0.014):
    """Fluid cell blocks 0..4 of InitialModule::makeBoundary (initialModule.hpp:219-263)."""
    dx, dr = xR / ni, rmax / nj
    x2, x3, x4, x5, x6 = 13.4e-3, 17.8e-3, 22.8e-3, 27.8e-3, 7.8e-3
    r1, r3, r4, r5 = 0.6e-3, 4.0e-3, 9.0e-3, 2.0e-3
    lo = lambda v, d: int(v / d + 0.5) + 1
    hi = lambda v, d: int(v / d - 0.5) + 1
    ib = [[lo(x6, dx), hi(x2, dx)], [lo(x2, dx), hi(x4, dx)], [lo(x2, dx), hi(x3, dx)],
          [lo(x3, dx), hi(x5, dx)], [lo(x5, dx), hi(xR, dx)]]
    jb = [[lo(r3, dr), hi(r4, dr)], [lo(r5, dr), hi(r4, dr)], [lo(r1, dr), hi(r5, dr)],
          [lo(0.0, dr), hi(r5, dr)], [lo(0.0, dr), hi(rmax, dr)]]
    return np.array(ib, np.int32), np.array(jb, np.int32)


def cathode_flags(ni, nj, ib, jb) -> np.ndarray:
    """Side flags of the fluid cells of the cathode's five fluid blocks."""
    fl = np.zeros((ni + 2, nj + 2), np.uint8)
    for b in range(5):
        I, J = np.meshgrid(np.arange(ib[b][0], ib[b][1] + 1), np.arange(jb[b][0], jb[b][1] + 1), indexing="ij")
        bLx = (I != ib[0][0]) | (b != 0)
        bLx &= (I != ib[2][0]) | (J > jb[0][0] - 1)
        bLx &= (I != ib[3][0]) | (J > jb[2][0] - 1)
        bLx &= (I != ib[4][0]) | (J < jb[1][0])
        bRx = ((I != ib[1][1]) | (J < jb[1][0])) & (I != ib[4][1])
        bLrw = ((J != jb[0][0]) | (I > ib[0][1])) & ((J != jb[2][0]) | (I > ib[2][1]))
        bLrc = J != jb[3][0]
        bRrw = ((J != jb[0][1]) | (b > 2)) & ((J != jb[3][1]) | (I < ib[1][1] + 1) | (I > ib[3][1]))
        bRro = (J != jb[4][1]) | (b != 4)
        code = (F_BLX * bLx + F_BRX * bRx + F_BLR_WALL * bLrw + F_BLR_CEN * bLrc + F_BRR_WALL * bRrw +
                F_BRR_OPEN * bRro + F_BRX_BIAS * ((I == ib[4][1]) & (b == 4)))
        fl[ib[b][0]:ib[b][1] + 1, jb[b][0]:jb[b][1] + 1] = code.astype(np.uint8)
    return fl


def rectangle_flags(ni, nj) -> np.ndarray:
    """r-z rectangle: wall at z = 0, electrode at z = L, axis at r = 0, wall at r = R."""
    fl = np.zeros((ni + 2, nj + 2), np.uint8)
    I, J = np.meshgrid(np.arange(1, ni + 1), np.arange(1, nj + 1), indexing="ij")
    fl[1:ni + 1, 1:nj + 1] = (F_BLX * (I != 1) + F_BRX * (I != ni) + F_BLR_WALL + F_BLR_CEN * (J != 1) +
                              F_BRR_WALL * (J != nj) + F_BRR_OPEN + F_BRX_BIAS * (I == ni)).astype(np.uint8)
    return fl


class Fields:
    """A cth_fields store bound to a Grid."""

    def __init__(self, grid):
        L = capi.load()
        h = ctypes.c_void_p()
        capi.check(L.cth_fields_create(grid._h, ctypes.byref(h)), allow_positive=False)
        self._h, self._L, self.grid = h, L, grid

    def close(self):
        if getattr(self, "_h", None):
            self._L.cth_fields_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def ptr(self, name: str) -> int:
        p = self._L.cth_field(self._h, name.encode())
        if not p:
            raise capi.CathodeError(capi.CTH_ERR_ALLOC, capi.last_error())
        return p

    def upload(self, name: str, a: np.ndarray):
        g = self.grid
        a = np.ascontiguousarray(a, dtype=np.float64)
        assert a.shape == (g.ni + 2, g.nj + 2), name
        capi.check(self._L.cth_field_upload(self._h, name.encode(), a.ctypes.data), allow_positive=False)

    def download(self, name: str) -> np.ndarray:
        g = self.grid
        out = np.zeros((g.ni + 2, g.nj + 2))
        capi.check(self._L.cth_field_download(self._h, name.encode(), out.ctypes.data), allow_positive=False)
        return out

    def set_flags(self, flags: np.ndarray):
        f = np.ascontiguousarray(flags, dtype=np.uint8)
        capi.check(self._L.cth_flags_upload(self._h, f.ctypes.data), allow_positive=False)

    def set_table(self, name: str, values):
        v = np.ascontiguousarray(values, dtype=np.float64)
        capi.check(self._L.cth_table_upload(self._h, name.encode(), v.ctypes.data, v.size), allow_positive=False)

    def solve_phi_pc(self, prm: dict, stream=None) -> dict:
        """FluidModule::solve_phi_couple_wdTe_wSEE_PC on the device (fluidModule.hpp:2080-3075).

        prm holds the cth_phi_params fields (dTe_SEE included); returns the PC
        result (iterations, calcRes errors, inner-solver status)."""
        p = capi.PhiParams(**{k: prm[k] for k, _ in capi.PhiParams._fields_})
        res = capi.PCResult()
        s = 0 if stream is None else stream.cuda_stream
        capi.check(self._L.cth_solve_phi_pc(self._h, ctypes.byref(p), s, ctypes.byref(res)), allow_positive=False)
        return dict(ncount=res.ncount, solver_rc=res.solver_rc, error_phi=res.error_phi,
                    error_nUex=res.error_nUex, error_nUer=res.error_nUer, error_iter=list(res.error_iter),
                    solver=res.solver.as_dict())

    def set_ghost_rules(self, rules):
        """Rules (i0, i1, j0, j1, di, dj, rhoe_mode) applied after the electron sweeps."""
        a = np.ascontiguousarray(np.asarray(rules, dtype=np.int32).reshape(-1, 7))
        capi.check(self._L.cth_ghost_rules_upload(self._h, a.ctypes.data, a.shape[0]), allow_positive=False)

    def _sg(self, fn, prm, stream):
        p = capi.SGParams(**{k: prm[k] for k, _ in capi.SGParams._fields_})
        res = capi.PCResult()
        s = 0 if stream is None else stream.cuda_stream
        capi.check(fn(self._h, ctypes.byref(p), s, ctypes.byref(res)), allow_positive=False)
        return dict(ncount=res.ncount, solver_rc=res.solver_rc, errors=(res.error_phi, res.error_nUex, res.error_nUer),
                    error_iter=list(res.error_iter), solver=res.solver.as_dict(), Ii_Anode=res.Ii_Anode,
                    Ie_Anode=res.Ie_Anode, I_Anode=res.I_Anode)

    def solve_rhoe_pc(self, prm: dict, stream=None) -> dict:
        """FluidModule::solve_rhoe_wdTe_wSEE_PC on the device (fluidModule.hpp:3082-3970)."""
        return self._sg(self._L.cth_solve_rhoe_pc, prm, stream)

    def solve_Te_pc(self, prm: dict, stream=None) -> dict:
        """FluidModule::solve_Te_wdTe_wSEE_PC on the device (fluidModule.hpp:4006-4957)."""
        return self._sg(self._L.cth_solve_Te_pc, prm, stream)

    def update_transport_coef(self, prm: dict, stream=None):
        """FluidModule::update_transport_coef on the device (fluidModule.hpp:5799-5976)."""
        p = capi.TransportParams(**{k: prm[k] for k, _ in capi.TransportParams._fields_})
        s = 0 if stream is None else stream.cuda_stream
        capi.check(self._L.cth_update_transport_coef(self._h, ctypes.byref(p), s), allow_positive=False)
