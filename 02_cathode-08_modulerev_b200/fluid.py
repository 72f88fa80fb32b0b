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
import os

import numpy as np

from . import capi

F_BLX, F_BRX, F_BLR_WALL, F_BLR_CEN, F_BRR_WALL, F_BRR_OPEN = 1, 2, 4, 8, 16, 32
F_BRX_BIAS = 64  # the right wall of the cell is the biased electrode
F_BRR_INLET = 128  # the upper wall of the cell is the neutral gas inlet
TABLES = ("nu_elas_N", "nu_exc_N", "nu_excReso_N", "nu_excMeta_N", "nu_ionz_N", "nu_ionzStep_N",
          "nu_excStep_N", "nu_super_N", "rate_eloss_n_N", "rate_eloss_m_N", "nui_m_N")


def cathode_blocks(ni=194, nj=70, xR=0.0388, rmax=0.014):
    """Fluid cell blocks 0..4 of InitialModule::makeBoundary (initialModule.hpp:219-263)."""
    dx, dr = xR / ni, rmax / nj
    # formed as the reference forms them (initialModule.hpp:225-230): the sums round differently
    # from the literals, which moves a block edge where x / dx lands on .5 (97 x 35)
    x6 = 0.0e-3 + 7.8e-3
    x2, x3, x4, x5 = 5.6e-3 + 7.8e-3, 10.0e-3 + 7.8e-3, 15.0e-3 + 7.8e-3, 20.0e-3 + 7.8e-3
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


# optional trailing fields of the parameter blocks (no counterpart in the
# reference) and their defaults
_PARAM_DEFAULTS = {"warm_start": 0, "guess_max_relres": 1.0}


def _param_fields(cls, prm: dict) -> dict:
    return {k: (prm[k] if k in prm or k not in _PARAM_DEFAULTS else _PARAM_DEFAULTS[k]) for k, _ in cls._fields_}


def step_params(params: dict) -> capi.StepParams:
    """cth_step_params from a parameter dict (step fields + the sub-step blocks)."""
    P = capi.StepParams()
    for k in ("itime", "ndt_i", "ndt_n", "ndt_m", "flag_adp_dt", "dt", "CFL", "gtime"):
        setattr(P, k, params[k])
    for blk, cls in (("ion", capi.IonParams), ("phi", capi.PhiParams), ("rhoe", capi.SGParams),
                     ("eps", capi.SGParams), ("transport", capi.TransportParams)):
        setattr(P, blk, cls(**_param_fields(cls, params[blk])))
    net = params.get("net")
    P.net = net.handle if net is not None else None
    nb = params["neutral"]
    P.neutral = capi.NeutralParams(**{k: nb[k] for k, _ in capi.NeutralParams._fields_
                                      if k not in ("n_pos_box", "pos_box", "do_rhon", "do_rhom")})
    boxes = params.get("pos_boxes", [])
    P.neutral.n_pos_box = len(boxes)
    for q, bx in enumerate(boxes):
        for k in range(4):
            P.neutral.pos_box[q][k] = int(bx[k])
    return P


def step_params_back(P: capi.StepParams, params: dict):
    """Copy the step fields the step updates (itime, dt, CFL, gtime) back into the dict."""
    for k in ("itime", "dt", "CFL", "gtime"):
        params[k] = getattr(P, k)


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

    def set_warm_start(self, enable: bool, max_relres: float = 1.0):
        """Field-valued solves (ion velocities, rhoi, rhon, rhom) start from the
        field's current values (guess threshold max_relres); default off."""
        capi.check(self._L.cth_fields_set_warm_start(self._h, int(enable), float(max_relres)),
                   allow_positive=False)

    def plane(self, name: str):
        """Zero-copy torch view (nj+2, ld) float64 of a device plane (library layout)."""
        import torch
        g = self.grid

        class _View:
            pass
        v = _View()
        v.__cuda_array_interface__ = {"shape": (g.nj + 2, g.ld), "typestr": "<f8", "data": (self.ptr(name), False),
                                      "version": 3, "strides": None}
        return torch.as_tensor(v, device=f"cuda:{g.device}")

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

    def _many(self, arrays: dict, fn, writable: bool, stream):
        g = self.grid
        names = list(arrays)
        arrs = [arrays[k] for k in names]
        for k, a in zip(names, arrs):
            ok = (isinstance(a, np.ndarray) and a.dtype == np.float64 and a.flags.c_contiguous and
                  a.shape == (g.ni + 2, g.nj + 2) and (a.flags.writeable or not writable))
            if not ok:
                raise ValueError(f"{k}: need a C-contiguous float64 array of shape {(g.ni + 2, g.nj + 2)}")
        n = len(names)
        cn = (ctypes.c_char_p * n)(*[k.encode() for k in names])
        cp = (ctypes.c_void_p * n)(*[a.ctypes.data for a in arrs])
        s = 0 if stream is None else stream.cuda_stream
        capi.check(fn(self._h, cn, cp, n, s), allow_positive=False)

    def upload_many(self, arrays: dict, stream=None):
        """Upload {name: [i][j] array} in one batch (one synchronisation; pinned arrays copy fastest)."""
        self._many(arrays, self._L.cth_fields_upload_many, False, stream)

    def download_many(self, arrays: dict, stream=None):
        """Download into the given {name: [i][j] array} in one batch, after the work queued on `stream`."""
        self._many(arrays, self._L.cth_fields_download_many, True, stream)

    def set_download_plan(self, arrays: dict):
        """The following fluid steps copy these fields into the given [i][j] host
        arrays (pinned for full speed) as soon as each is final within the step,
        overlapping the remaining sweeps; download_wait() waits for them."""
        g = self.grid
        names = list(arrays)
        for k in names:
            a = arrays[k]
            if not (isinstance(a, np.ndarray) and a.dtype == np.float64 and a.flags.c_contiguous and
                    a.flags.writeable and a.shape == (g.ni + 2, g.nj + 2)):
                raise ValueError(f"{k}: need a writable C-contiguous float64 array of shape {(g.ni + 2, g.nj + 2)}")
        n = len(names)
        cn = (ctypes.c_char_p * max(n, 1))(*[k.encode() for k in names])
        cp = (ctypes.c_void_p * max(n, 1))(*[arrays[k].ctypes.data for k in names])
        self._plan = dict(arrays)  # the arrays must outlive the copies
        capi.check(self._L.cth_fields_set_download_plan(self._h, cn, cp, n), allow_positive=False)

    def download_wait(self):
        capi.check(self._L.cth_fields_download_wait(self._h), allow_positive=False)

    def set_upload_plan(self, arrays: dict):
        """The next fluid step copies these [i][j] host arrays (pinned for full
        speed) in at its start without a host synchronisation; rhoeps, rhon and
        rhom arrive while the sweeps before their first use run."""
        g = self.grid
        names = list(arrays)
        for k in names:
            a = arrays[k]
            if not (isinstance(a, np.ndarray) and a.dtype == np.float64 and a.flags.c_contiguous and
                    a.shape == (g.ni + 2, g.nj + 2)):
                raise ValueError(f"{k}: need a C-contiguous float64 array of shape {(g.ni + 2, g.nj + 2)}")
        n = len(names)
        cn = (ctypes.c_char_p * max(n, 1))(*[k.encode() for k in names])
        cp = (ctypes.c_void_p * max(n, 1))(*[arrays[k].ctypes.data for k in names])
        self._up_plan = dict(arrays)  # the arrays must outlive the copies
        capi.check(self._L.cth_fields_set_upload_plan(self._h, cn, cp, n), allow_positive=False)

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
        p = capi.PhiParams(**_param_fields(capi.PhiParams, prm))
        res = capi.PCResult()
        s = 0 if stream is None else stream.cuda_stream
        capi.check(self._L.cth_solve_phi_pc(self._h, ctypes.byref(p), s, ctypes.byref(res)), allow_positive=False)
        return dict(ncount=res.ncount, solver_rc=res.solver_rc, error_phi=res.error_phi,
                    error_nUex=res.error_nUex, error_nUer=res.error_nUer, error_iter=list(res.error_iter),
                    solver=res.solver.as_dict(), first=res.first.as_dict())

    def set_ion_geometry(self, geo: dict):
        """Upload the ion wall programs and residual boxes of a geometry dict."""
        for k, prog in enumerate(ion_programs(geo["seg"])):
            a = (capi.IonOp * max(1, len(prog)))()
            for q, o in enumerate(prog):
                for f, v in zip(capi.ION_OP_FIELDS, o):
                    setattr(a[q], f, int(v))
            capi.check(self._L.cth_ion_program_upload(self._h, k, ctypes.addressof(a), len(prog)),
                       allow_positive=False)
        for k, boxes in enumerate(ion_boxes(geo)):
            b = np.ascontiguousarray(np.asarray(boxes, dtype=np.int32).reshape(-1, 4))
            capi.check(self._L.cth_ion_boxes_upload(self._h, k, b.ctypes.data, b.shape[0]), allow_positive=False)

    def ion_step(self, grid_x, grid_r, prm: dict, stream=None) -> dict:
        """The ion sub-step (src/main.cpp:191-197) on the device; grid_x / grid_r are
        Grids of the x-face and r-face blocks."""
        p = capi.IonParams(**{k: prm[k] for k, _ in capi.IonParams._fields_})
        res = capi.IonResult()
        s = 0 if stream is None else stream.cuda_stream
        capi.check(self._L.cth_ion_step(self._h, grid_x._h, grid_r._h, ctypes.byref(p), s, ctypes.byref(res)),
                   allow_positive=False)
        return dict(error_rhoi=res.error_rhoi, error_Uix=res.error_Uix, error_Uir=res.error_Uir,
                    error_Uip=res.error_Uip, solver_rc=res.solver_rc, solver=[res.solver[k].as_dict() for k in range(4)])

    def update_neutrals(self, prm: dict, pos_boxes, stream=None) -> dict:
        """FluidModule::update_rhon then update_rhom on the device (fluidModule.hpp:4963-5792)."""
        p = capi.NeutralParams(**{k: prm[k] for k, _ in capi.NeutralParams._fields_
                                  if k not in ("n_pos_box", "pos_box", "do_rhon", "do_rhom")})
        p.do_rhon = int(prm.get("do_rhon", 1))
        p.do_rhom = int(prm.get("do_rhom", 1))
        p.n_pos_box = len(pos_boxes)
        for q, bx in enumerate(pos_boxes):
            for k in range(4):
                p.pos_box[q][k] = int(bx[k])
        res = capi.NeutralResult()
        s = 0 if stream is None else stream.cuda_stream
        capi.check(self._L.cth_update_neutrals(self._h, ctypes.byref(p), s, ctypes.byref(res)), allow_positive=False)
        return dict(error_rhon=res.error_rhon, error_rhom=res.error_rhom, solver_rc=res.solver_rc,
                    solver=[res.solver[k].as_dict() for k in range(2)])

    def fluid_step(self, grid_x, grid_r, params: dict, stream=None) -> dict:
        """One time step (src/main.cpp:170-251) through cth_fluid_step; params holds
        the step fields and the sub-step blocks (ion, phi, rhoe, eps, neutral,
        transport) as dicts, plus pos_boxes; itime, dt, CFL and gtime are updated."""
        P = step_params(params)
        R = capi.StepResult()
        s = 0 if stream is None else stream.cuda_stream
        capi.check(self._L.cth_fluid_step(self._h, grid_x._h, grid_r._h, ctypes.byref(P), s, ctypes.byref(R)),
                   allow_positive=False)
        step_params_back(P, params)
        return dict(solver_rc=R.solver_rc, ran_ion=R.ran_ion, net_ran=R.net_ran, cfl=R.cfl.CFL, dt=R.cfl.dt,
                    errors=dict(rhoi=R.ion.error_rhoi, Uix=R.ion.error_Uix, Uir=R.ion.error_Uir, Uip=R.ion.error_Uip,
                                phi=R.phi.error_phi, rhoe=R.rhoe.error_phi, rhoeps=R.eps.error_phi,
                                rhon=R.neutral.error_rhon, rhom=R.neutral.error_rhom),
                    anode=dict(Ii=R.rhoe.Ii_Anode, Ie=R.rhoe.Ie_Anode, I=R.rhoe.I_Anode),
                    iterations=dict(phi=R.phi.solver.iterations, rhoe=R.rhoe.solver.iterations,
                                    eps=R.eps.solver.iterations, rhoi=R.ion.solver[3].iterations,
                                    rhon=R.neutral.solver[0].iterations),
                    phi_first=R.phi.first.as_dict(),
                    guess=dict(Uix=R.ion.solver[0].guess, Uir=R.ion.solver[1].guess, Uip=R.ion.solver[2].guess,
                               rhoi=R.ion.solver[3].guess, rhon=R.neutral.solver[0].guess,
                               rhom=R.neutral.solver[1].guess),
                    all_iterations=dict(Uix=R.ion.solver[0].iterations, Uir=R.ion.solver[1].iterations,
                                        Uip=R.ion.solver[2].iterations, rhoi=R.ion.solver[3].iterations,
                                        rhon=R.neutral.solver[0].iterations, rhom=R.neutral.solver[1].iterations))

    def update_energy_profile(self, grid_x, grid_r, prm: dict, E1x, E1r, E1p, J1x, J1r, J1p, stream=None) -> dict:
        """Absorbed microwave power (emfieldModule.hpp:7630-7790): complex128 device
        planes (nj+2, ld) in, J planes and the store's Pabsx/Pabsr/Pabsp/Pabs out."""
        p = capi.EnergyParams(**{k: prm[k] for k, _ in capi.EnergyParams._fields_})
        r = capi.EnergyResult()
        s = 0 if stream is None else stream.cuda_stream
        ptr = [ctypes.c_void_p(t.data_ptr()) for t in (E1x, E1r, E1p, J1x, J1r, J1p)]
        capi.check(self._L.cth_update_energy_profile(self._h, grid_x._h, grid_r._h, ctypes.byref(p), *ptr, s,
                                                     ctypes.byref(r)), allow_positive=False)
        return {k: getattr(r, k) for k, _ in capi.EnergyResult._fields_}

    def mw_port_rescale(self, prm: dict, power_sum: float, E1x=None, E1r=None, E1p=None, J1x=None, J1r=None,
                        J1p=None, J1x_exc=None, J1r_exc=None, J1p_exc=None, stream=None) -> dict:
        """The port / reflection / rescale part of update_energy_profile
        (emfieldModule.hpp:7792-8105) on complex128 device planes; prm holds
        the cth_mw_port_params fields (S-parameters as complex numbers).
        Returns the reported quantities (complex ones as complex)."""
        p = capi.MWPortParams()
        for k, t in capi.MWPortParams._fields_:
            v = prm[k]
            if k.startswith("S"):
                getattr(p, k)[0], getattr(p, k)[1] = complex(v).real, complex(v).imag
            else:
                setattr(p, k, v)
        r = capi.MWPortResult()
        s = 0 if stream is None else stream.cuda_stream
        ptr = [ctypes.c_void_p(t.data_ptr()) if t is not None else None
               for t in (E1x, E1r, E1p, J1x, J1r, J1p, J1x_exc, J1r_exc, J1p_exc)]
        rc = self._L.cth_mw_port_rescale(self._h, ctypes.byref(p), float(power_sum), *ptr, s, ctypes.byref(r))
        capi.check(rc, allow_positive=False)
        out = {}
        for k, t in capi.MWPortResult._fields_:
            v = getattr(r, k)
            out[k] = complex(v[0], v[1]) if hasattr(v, "__len__") else v
        return out

    def check_cfl(self, dt: float, CFL: float, masse: float, rmin: float, dr: float, flag_adp_dt: int = 0,
                  stream=None) -> dict:
        """FluidModule::check_CFL (fluidModule.hpp:57-115); returns dt, CFL and the maxima."""
        c = capi.CFL(dt=dt, CFL=CFL, masse=masse, rmin=rmin, dr=dr, flag_adp_dt=flag_adp_dt)
        s = 0 if stream is None else stream.cuda_stream
        capi.check(self._L.cth_check_cfl(self._h, ctypes.byref(c), s), allow_positive=False)
        return {k: getattr(c, k) for k, _ in capi.CFL._fields_}

    def set_ghost_rules(self, rules):
        """Rules (i0, i1, j0, j1, di, dj, rhoe_mode) applied after the electron sweeps."""
        a = np.ascontiguousarray(np.asarray(rules, dtype=np.int32).reshape(-1, 7))
        capi.check(self._L.cth_ghost_rules_upload(self._h, a.ctypes.data, a.shape[0]), allow_positive=False)

    # restart files (the reference's restart<nOut>.csv) ----------------------------------------
    def write_restart(self, path: str, x, r, stream=None):
        """Queue the write of a restart file of the reference's format (OutputModule::output,
        outputModule.hpp:429-470); returns once the copies are queued on ``stream``.
        x, r: the cell-centre coordinates gc.x (ni+2) and gc.r (nj+2)."""
        g = self.grid
        x = np.ascontiguousarray(x, dtype=np.float64)
        r = np.ascontiguousarray(r, dtype=np.float64)
        if x.shape != (g.ni + 2,) or r.shape != (g.nj + 2,):
            raise ValueError("x must have ni+2 and r nj+2 entries")
        s = 0 if stream is None else stream.cuda_stream
        capi.check(self._L.cth_restart_write(self._h, os.fsencode(path), x.ctypes.data, r.ctypes.data, s),
                   allow_positive=False)

    def restart_wait(self):
        """Wait for the restart file being written; raises if writing it failed."""
        capi.check(self._L.cth_restart_wait(self._h), allow_positive=False)

    def read_restart(self, path: str, gx, gr, x, r, dx: float, dr: float, V_bias: float, stream=None) -> dict:
        """Read a restart file into the store with the reference's checks and
        post-processing (InputModule::input_restart_data, inputModule.hpp:667-1157)."""
        x = np.ascontiguousarray(x, dtype=np.float64)
        r = np.ascontiguousarray(r, dtype=np.float64)
        p = capi.RestartParams(dx=dx, dr=dr, V_bias=V_bias)
        info = capi.RestartInfo()
        s = 0 if stream is None else stream.cuda_stream
        capi.check(self._L.cth_restart_read(self._h, gx._h, gr._h, os.fsencode(path), x.ctypes.data, r.ctypes.data,
                                            ctypes.byref(p), s, ctypes.byref(info)), allow_positive=False)
        return dict(rows=info.rows, variables_read=info.variables_read, unknown_columns=info.unknown_columns)

    def set_energy_keep_walls(self, boxes):
        """r-face boxes (i0, i1, j0, j1) whose wall flux Gr_wall the energy sweep leaves unchanged
        (the cathode's lower wall x2, fluidModule.hpp:4428-4449); at most 4."""
        a = np.ascontiguousarray(np.asarray(boxes, dtype=np.int32).reshape(-1, 4))
        capi.check(self._L.cth_energy_keep_walls_upload(self._h, a.ctypes.data, a.shape[0]), allow_positive=False)

    def set_geometry(self, geo):
        """Side flags, electron ghost rules and the energy sweep's kept walls of a geometry dict."""
        self.set_flags(geo["flags"])
        self.set_ghost_rules(geo["ghosts"])
        self.set_energy_keep_walls(geo.get("energy_keep_walls", []))

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


# ---------------------------------------------------------------------------
# geometries: cell / face blocks, wall segments, ghost rules, ion wall programs
# ---------------------------------------------------------------------------

def cell_coordinates(ni, nj, dx, dr, xL=0.0, rmin=0.0):
    """Cell-centre coordinates gc.x (ni+2) and gc.r (nj+2) as InitialModule::iniParam
    forms them (initialModule.hpp:80-85): x_i = xL + (i - 0.5) dx, r_j = rmin + (j - 0.5) dr."""
    return xL + (np.arange(ni + 2) - 0.5) * dx, rmin + (np.arange(nj + 2) - 0.5) * dr


def cathode_geometry(ni=194, nj=70, xR=0.0388, rmax=0.014, width_neutIn=0.0055) -> dict:
    """The cathode's fluid blocks with their x-face and r-face blocks
    (initialModule.hpp:219-345), side flags, ghost rules of the electron sweeps
    (fluidModule.hpp:3884-3921, :4878-4914) and the named wall segments of the ion
    sweeps on the cell, x-face and r-face index sets (fluidModule.hpp:218-360,
    :700-800, :1130-1200)."""
    dx, dr = xR / ni, rmax / nj
    # formed as the reference forms them (initialModule.hpp:225-230): the sums round differently
    # from the literals, which moves a block edge where x / dx lands on .5 (97 x 35)
    x6 = 0.0e-3 + 7.8e-3
    x2, x3, x4, x5 = 5.6e-3 + 7.8e-3, 10.0e-3 + 7.8e-3, 15.0e-3 + 7.8e-3, 20.0e-3 + 7.8e-3
    r1, r3, r4, r5 = 0.6e-3, 4.0e-3, 9.0e-3, 2.0e-3
    lo = lambda v, d, k: int(v / d + 0.5) + k
    hi = lambda v, d, k: int(v / d - 0.5) + k
    ib, jb = cathode_blocks(ni, nj, xR, rmax)
    fxi = np.array([[lo(x6, dx, 2), hi(x2, dx, 2)], [lo(x2, dx, 2), hi(x4, dx, 1)], [lo(x2, dx, 2), hi(x3, dx, 2)],
                    [lo(x3, dx, 2), hi(x5, dx, 2)], [lo(x5, dx, 2), hi(xR, dx, 1)]], np.int32)
    fxj = np.array([[lo(r3, dr, 1), hi(r4, dr, 1)], [lo(r5, dr, 1), hi(r4, dr, 1)], [lo(r1, dr, 1), hi(r5, dr, 1)],
                    [lo(0.0, dr, 1), hi(r5, dr, 1)], [lo(0.0, dr, 1), hi(rmax, dr, 1)]], np.int32)
    fri = np.array([[lo(x6, dx, 1), hi(x2, dx, 1)], [lo(x2, dx, 1), hi(x4, dx, 1)], [lo(x2, dx, 1), hi(x3, dx, 1)],
                    [lo(x3, dx, 1), hi(x5, dx, 1)], [lo(x5, dx, 1), hi(xR, dx, 1)]], np.int32)
    frj = np.array([[lo(r3, dr, 2), hi(r4, dr, 1)], [lo(r5, dr, 1), hi(r4, dr, 1)], [lo(r1, dr, 2), hi(r5, dr, 1)],
                    [lo(0.0, dr, 2), hi(r5, dr, 1)], [lo(0.0, dr, 2), hi(rmax, dr, 1)]], np.int32)

    def segs(I, J, axis):
        t = dict(z0=(I[0][0], I[0][0], J[0][0], J[0][1]), z1=(I[2][0], I[2][0], J[2][0], J[0][0] - 1),
                 z2=(I[3][0], I[3][0], J[3][0], J[2][0] - 1), z4=(I[4][0], I[4][0], J[1][0], J[4][1]),
                 z3=(I[1][1], I[1][1], J[1][0], J[1][1]), z5=(I[4][1], I[4][1], J[4][0], J[4][1]),
                 x0=(I[0][0], I[0][1], J[0][0], J[0][0]), x2=(I[2][0], I[2][1], J[2][0], J[2][0]),
                 x1=(I[0][0], I[1][1], J[0][1], J[0][1]), x4=(I[1][1] + 1, I[3][1], J[3][1], J[3][1]),
                 x5=(I[4][0], I[4][1], J[4][1], J[4][1]),
                 x6=(I[3][0], I[4][1], J[3][0], J[3][0]) if axis else None)
        return {k: (tuple(int(v) for v in s) if s is not None else None) for k, s in t.items()}

    ghosts = [(ib[0][0], ib[0][0], jb[0][0], jb[0][1], -1, 0, 0), (ib[1][0], ib[1][0], jb[1][0], jb[0][0] - 1, -1, 0, 0),
              (ib[0][0], ib[0][1], jb[0][0], jb[0][0], 0, -1, 0), (ib[1][1], ib[1][1], jb[1][0], jb[1][1], 1, 0, 1),
              (ib[0][0], ib[1][1], jb[0][1], jb[0][1], 0, 1, 1)]
    seg = dict(c=segs(ib, jb, False), x=segs(fxi, fxj, False), r=segs(fri, frj, True))
    flags = cathode_flags(ni, nj, ib, jb)
    # neutral inlet: the cells of the x1 wall with x_i <= width_neutIn + x6 (fluidModule.hpp:5040-5041)
    i0, i1, j0, _ = seg["c"]["x1"]
    for i in range(i0, i1 + 1):
        if 0.0 + (i - 0.5) * dx <= width_neutIn + x6:
            flags[i, j0] |= F_BRR_INLET
    return dict(ni=ni, nj=nj, dx=dx, dr=dr, ib=ib, jb=jb, fxi=fxi, fxj=fxj, fri=fri, frj=frj, flags=flags,
                ghosts=[tuple(int(v) for v in g) for g in ghosts], seg=seg, x6=x6, xL=0.0,
                width_neutIn=width_neutIn, pos_boxes=[tuple(int(v) for v in (ib[b][0], ib[b][1], jb[b][0], jb[b][1]))
                                                      for b in range(2)],
                # the energy sweep's lower-wall loop x2 sets Gr there but leaves Gr_wall as it was
                # (fluidModule.hpp:4428-4449, unlike x0 at :4423): r-faces (i0, i1, j0, j1)
                energy_keep_walls=[(int(ib[2][0]), int(ib[2][1]), int(jb[2][0]), int(jb[2][0]))])


def block_union_size(ib, jb) -> int:
    """Number of (i, j) in the union of the blocks [ib[b][0], ib[b][1]] x [jb[b][0], jb[b][1]]."""
    cells = set()
    for (a, b), (c, d) in zip(np.asarray(ib), np.asarray(jb)):
        cells.update((i, j) for i in range(int(a), int(b) + 1) for j in range(int(c), int(d) + 1))
    return len(cells)


def cathode_microwave(ni=194, nj=70, xR=0.0388, rmax=0.014) -> dict:
    """The microwave geometry of the cathode for Microwave3: the six cell, x-face
    and r-face blocks (initialModule.hpp:219-345: the five fluid blocks and the
    coax feed, block 5) and the 12 boundary lists of MicrowaveBC as
    InitialModule::makeBoundary builds them (initialModule.hpp:420-1055), from
    the package's segment table data/mw_lists_cathode.json: one record per
    segment (field, side, code, a loop over i or j with the other index fixed,
    or one entry), bounds written over the cell blocks as ic[b][k] / jc[b][k]
    plus a constant, so that the table serves every resolution.
    Returns dict(blocks=((xi, xj), (ri, rj), (ci, cj)), lists={(field, side):
    [(i, j, code), ...]}, j_flc_00) for Microwave3(..., blocks=) and
    set_boundary."""
    import json
    import os
    import re
    dx, dr = xR / ni, rmax / nj
    x1, x6 = 0.0, 7.8e-3
    x2, x3, x4, x5 = 5.6e-3 + x6, 10.0e-3 + x6, 15.0e-3 + x6, 20.0e-3 + x6
    r1, r2, r3, r4, r5 = 0.6e-3, 2.0e-3, 4.0e-3, 9.0e-3, 2.0e-3
    lo = lambda v, d, k: int(v / d + 0.5) + k
    hi = lambda v, d, k: int(v / d - 0.5) + k
    zs = [(x6, x2), (x2, x4), (x2, x3), (x3, x5), (x5, xR), (x1, x2)]
    rs = [(r3, r4), (r5, r4), (r1, r5), (0.0, r5), (0.0, rmax), (r1, r2)]
    ci = np.array([[lo(a, dx, 1), hi(b, dx, 1)] for a, b in zs], np.int32)
    cj = np.array([[lo(a, dr, 1), hi(b, dr, 1)] for a, b in rs], np.int32)
    # x-faces: both ends one further (the face i-1/2 of the block's first cell is a wall),
    # except the right ends of blocks 1 and 4; r-faces: the lower end one further, except block 1
    xi = np.array([[lo(a, dx, 2), hi(b, dx, 1 if b_ in (1, 4) else 2)] for b_, (a, b) in enumerate(zs)], np.int32)
    rj = np.array([[lo(a, dr, 1 if b_ == 1 else 2), hi(b, dr, 1)] for b_, (a, b) in enumerate(rs)], np.int32)
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data", "mw_lists_cathode.json")
    with open(path) as f:
        table = json.load(f)
    blocks = {"ic": ci, "jc": cj}
    form = re.compile(r"([ij]c)\[(\d)\]\[([01])\]([+-]\d+)?")

    def ev(e):
        m = form.fullmatch(e)
        if not m:
            raise ValueError(f"segment table: unexpected bound {e!r}")
        return int(blocks[m.group(1)][int(m.group(2))][int(m.group(3))]) + int(m.group(4) or 0)

    lists = {(f_, sd): [] for f_ in "xrp" for sd in "WESN"}
    for sg in table["segments"]:
        key = (sg["field"], sg["side"])
        if sg["kind"] == "point":
            lists[key].append((ev(sg["i"]), ev(sg["j"]), sg["code"]))
            continue
        fix = ev(sg["fix"])
        for v in range(ev(sg["lo"]), ev(sg["hi"]) + 1):
            lists[key].append((fix, v, sg["code"]) if sg["var"] == "j" else (v, fix, sg["code"]))
    return dict(blocks=((xi, cj), (ci, rj), (ci, cj)), lists=lists, j_flc_00=int(cj[0][0]), ni=ni, nj=nj,
                dx=dx, dr=dr)


def rectangle_geometry(ni, nj, Lz=10e-3, Lr=5e-3, width_neutIn=0.0) -> dict:
    """The r-z rectangle as one fluid block: z = 0 grounded wall (the reference's
    z0), z = L the biased electrode (z5), r = R a grounded wall (x1) with the neutral
    inlet over z <= width_neutIn, r = 0 the axis."""
    one = lambda a, b: np.array([[a, b]], np.int32)
    empty = dict(z1=None, z2=None, z3=None, z4=None, x0=None, x2=None, x4=None, x5=None)
    seg = dict(c=dict(empty, z0=(1, 1, 1, nj), z5=(ni, ni, 1, nj), x1=(1, ni, nj, nj), x6=None),
               x=dict(empty, z0=(2, 2, 1, nj), z5=(ni, ni, 1, nj), x1=(2, ni, nj, nj), x6=None),
               r=dict(empty, z0=(1, 1, 2, nj), z5=(ni, ni, 2, nj), x1=(1, ni, nj, nj), x6=(1, ni, 2, 2)))
    ghosts = [(1, 1, 1, nj, -1, 0, 0), (ni, ni, 1, nj, 1, 0, 1), (1, ni, nj, nj, 0, 1, 1)]
    flags = rectangle_flags(ni, nj)
    dx = Lz / ni
    for i in range(1, ni + 1):
        if 0.0 + (i - 0.5) * dx <= width_neutIn:
            flags[i, nj] |= F_BRR_INLET
    return dict(ni=ni, nj=nj, dx=dx, dr=Lr / nj, ib=one(1, ni), jb=one(1, nj), fxi=one(2, ni), fxj=one(1, nj),
                fri=one(1, ni), frj=one(2, nj), flags=flags, ghosts=ghosts, seg=seg, x6=0.0, xL=0.0,
                width_neutIn=width_neutIn, pos_boxes=[(1, ni, 1, nj)], energy_keep_walls=[])


_K = dict(WALL_FOLD=1, ZERO_COEF=2, FOLD_SUB=3, OPEN_FOLD=4, SET_WALL=5, SET_ZERO=6, COPY=7, SET_OPEN=8)
_D = dict(W=0, E=1, S=2, N=3)


def _op(kind, s, di0=0, di1=0, dj0=0, dj1=0, di=0, dj=0, dir="W", sign=0, bias=0, pair=0, scale=0):
    if s is None:
        return None
    i0, i1, j0, j1 = s[0] + di0, s[1] + di1, s[2] + dj0, s[3] + dj1
    if i0 > i1 or j0 > j1:
        return None
    return (_K[kind], i0, i1, j0, j1, di, dj, _D[dir], sign, bias, pair, scale)


def ion_programs(seg: dict) -> list:
    """The wall programs of the ion momentum sweeps, in the reference's loop order:
    [Uix assembly, Uix after solve, Uir assembly, Uir after solve, Uip assembly,
    Uip after solve] (fluidModule.hpp:216-579, :675-1046, :1114-1399)."""
    X, R, C = seg["x"], seg["r"], seg["c"]
    left, right = ("z0", "z1", "z2", "z4"), ("z3", "z5")
    P = [[] for _ in range(6)]
    # Uix
    for n in left:
        P[0].append(_op("WALL_FOLD", X[n], dir="W", sign=-1, pair=0))
    for n in right:
        P[0].append(_op("WALL_FOLD", X[n], dir="E", sign=1, bias=int(n == "z5"), pair=0))
    for n in ("x0", "x2"):
        P[0].append(_op("ZERO_COEF", X[n], dir="S"))
    for n in ("x1", "x4", "x5"):
        P[0].append(_op("ZERO_COEF", X[n], dir="N"))
    for n in left:
        P[1].append(_op("SET_WALL", X[n], di=-1, sign=-1, pair=0))
    for n in right:
        P[1].append(_op("SET_WALL", X[n], di=1, sign=1, bias=int(n == "z5"), pair=0))
    P[1].append(_op("SET_ZERO", X["x0"], di1=-1, dj=-1))
    P[1].append(_op("SET_ZERO", X["x2"], di1=-1, dj=-1))
    P[1].append(_op("SET_ZERO", X["x1"], dj=-1))          # the row below the top row, as the reference writes it
    P[1].append(_op("SET_ZERO", X["x4"], di0=1, di1=-1, dj=1))
    P[1].append(_op("SET_ZERO", X["x5"], dj=1))
    # Uir
    for n in left:
        P[2].append(_op("ZERO_COEF", R[n], dir="W"))
    for n in right:
        P[2].append(_op("ZERO_COEF", R[n], dir="E"))
    for n in ("x0", "x2"):
        P[2].append(_op("WALL_FOLD", R[n], dir="S", sign=-1, pair=1))
    P[2].append(_op("ZERO_COEF", R["x6"], dir="S"))
    for n in ("x1", "x4"):
        P[2].append(_op("WALL_FOLD", R[n], dir="N", sign=1, pair=1))
    P[2].append(_op("OPEN_FOLD", R["x5"], dir="N"))
    for n, adj in (("z0", (0, 0)), ("z1", (0, -1)), ("z2", (0, -1)), ("z4", (1, 0))):
        P[3].append(_op("SET_ZERO", R[n], dj0=adj[0], dj1=adj[1], di=-1))
    for n, adj in (("z3", (1, 0)), ("z5", (0, 0))):
        P[3].append(_op("SET_ZERO", R[n], dj0=adj[0], dj1=adj[1], di=1))
    for n in ("x0", "x2"):
        P[3].append(_op("SET_WALL", R[n], dj=-1, sign=-1, pair=1))
    P[3].append(_op("SET_ZERO", R["x6"], dj=-1))
    for n in ("x1", "x4"):
        P[3].append(_op("SET_WALL", R[n], dj=1, sign=1, pair=1))
    P[3].append(_op("SET_OPEN", R["x5"], dj=1))
    # Uip
    for n in left:
        P[4].append(_op("FOLD_SUB", C[n], dir="W"))
    for n in right:
        P[4].append(_op("FOLD_SUB", C[n], dir="E"))
    for n in ("x0", "x2"):
        P[4].append(_op("FOLD_SUB", C[n], dir="S", scale=1))
    for n in ("x1", "x4", "x5"):
        P[4].append(_op("FOLD_SUB", C[n], dir="N", scale=2))
    for n in left:
        P[5].append(_op("COPY", C[n], di=-1))
    for n in right:
        P[5].append(_op("COPY", C[n], di=1))
    for n in ("x0", "x2"):
        P[5].append(_op("COPY", C[n], dj=-1, scale=1))
    for n in ("x1", "x4", "x5"):
        P[5].append(_op("COPY", C[n], dj=1, scale=2))
    return [[o for o in prog if o is not None] for prog in P]


def ion_boxes(geo: dict) -> list:
    """Residual boxes of correct_Ui_constTe (fluidModule.hpp:1960-2070): rhoi and Uip
    over the cell blocks, Uix over the x-face blocks extended by one face in i, Uir
    over the r-face blocks without their first face in j."""
    cells = [(a, b, c, e) for (a, b), (c, e) in zip(geo["ib"], geo["jb"])]
    xs = [(a, b + 1, c, e) for (a, b), (c, e) in zip(geo["fxi"], geo["fxj"])]
    rs = [(a, b, c + 1, e) for (a, b), (c, e) in zip(geo["fri"], geo["frj"])]
    return [cells, xs, rs, cells]
