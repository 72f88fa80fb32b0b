"""The time loop of src/main.cpp:170-257 on the device for the r-z rectangle
discharge: cth_fluid_step every step and, every ``ndiv_mw`` steps, the microwave
update of the loop's end (:254-257): EmfieldModule::solve_Microwave (the
magnetised 3-component system on the discharge's n_e, nu_m1 and magnet field,
its ghost pass) and update_energy_profile without the reflection model
(flag_mwRef = 0: the absorbed power rescaled to Pmw, the port excitation by the
root of the ratio), whose Pabs the following energy sweeps read.
"""
from __future__ import annotations

import numpy as np

from . import capi
from .solvers import Grid, Microwave3


def rect_port(mw_params: dict, Pmw: float) -> dict:
    """Port settings of the rectangle's microwave update: no feed block, so no
    reflection model (flag_mwRef = 0): the absorbed power is rescaled to Pmw."""
    return dict(dx=mw_params["dx"], dr=mw_params["dr"], rmin=mw_params.get("rmin", 0.0),
                omegam=mw_params["omegam"], r1=mw_params["r1"], r2=mw_params["r2"], Z0=50.0, Pmw=float(Pmw),
                S11=0j, S21=1 + 0j, S12=1 + 0j, S22=0j, flag_mwRef=0, i_ref=1, j_out=0, i_out0=0, i_out1=0, jf0=0,
                jf1=0)


class MicrowaveUpdate:
    """cth_mw_update: the microwave update of the time loop (src/main.cpp:254-257)
    on a field store -- assembly from rhoe, nu_m1, Bx, Br, epsr_mw, solve, ghost
    pass, update_energy_profile, port / rescale to port["Pmw"] -- every ``ndiv_mw``
    steps.  E3 / J3: (3, nj+2, ld) complex128 device planes (None: the library
    allocates them).  warm_start: each solve after the first starts from the
    previous update's fields when they pass the device-side residual test."""

    def __init__(self, fs, m3, mw_params: dict, port: dict, ndiv_mw=100, maxit=400, tol=1e-10, E3=None, J3=None,
                 warm_start=False):
        import ctypes
        self._L = capi.load()
        p = capi.MWUpdateParams()
        for k, _ in capi.MWParams._fields_:
            setattr(p.mw, k, float(mw_params.get(k, 0.0)))
        for k, _ in capi.MWPortParams._fields_:
            v = port[k]
            if k.startswith("S"):
                getattr(p.port, k)[0], getattr(p.port, k)[1] = complex(v).real, complex(v).imag
            else:
                setattr(p.port, k, v)
        p.ndiv_mw, p.maxit, p.tol, p.warm_start = int(ndiv_mw), int(maxit), float(tol), int(bool(warm_start))
        self._keep = (E3, J3)
        h = ctypes.c_void_p()
        capi.check(self._L.cth_mw_update_create(fs._h, m3._h, ctypes.byref(p),
                                                E3.data_ptr() if E3 is not None else None,
                                                J3.data_ptr() if J3 is not None else None, ctypes.byref(h)),
                   allow_positive=False)
        self._h = h

    def set_net(self, net):
        """A trained microwave network (learned.UNet with 9 input, 6 output
        channels) whose guess starts each solve after the first; None: none."""
        capi.check(self._L.cth_mw_update_set_net(self._h, net.handle if net is not None else None),
                   allow_positive=False)
        self._net = net

    def due(self, itime: int) -> bool:
        return bool(self._L.cth_mw_update_due(self._h, int(itime)))

    def run(self, gx, gr, stream=None) -> dict:
        import ctypes
        r = capi.MWUpdateResult()
        s = 0 if stream is None else stream.cuda_stream
        rc = self._L.cth_mw_update_run(self._h, gx._h, gr._h, s, ctypes.byref(r))
        capi.check(rc)
        return dict(solve=r.solve.as_dict(), power_sum=r.power_sum, ratio=r.ratio, J1r_exc=r.J1r_exc, rc=rc)

    def prepare(self, stream=None):
        """Build the solve's hierarchy and graph (assembly + solve only; the
        discharge's state is left as it was)."""
        capi.check(self._L.cth_mw_update_prepare(self._h, 0 if stream is None else stream.cuda_stream),
                   allow_positive=False)

    def close(self):
        if getattr(self, "_h", None):
            self._L.cth_mw_update_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


FIELDS = ("rhoe", "rhoi", "rhon", "rhom", "Te", "Bx", "Br", "rhoeps", "phi", "Ex", "Er", "nUex", "nUer", "Uix",
          "Uir", "Uip", "rhoUix", "rhoUir", "rhoUix_wall", "rhoUir_wall", "rhoUex", "rhoUer", "rhoUex_wall",
          "rhoUer_wall", "Gx", "Gr", "Gx_wall", "Gr_wall", "rhoUnx", "rhoUnr", "rhoUnx_wall", "rhoUnr_wall",
          "rhoUmx", "rhoUmr", "rhoUmx_wall", "rhoUmr_wall", "nu_ano", "nu_ano_IAT", "Pabs", "rhoe_old")


class RectangleDischarge:
    """The seeded discharge of workloads.discharge_state / discharge_params on the
    ni (z) x nj (r) rectangle with its microwave update every ``ndiv_mw`` steps.
    precision: CTH_PREC_MIXED or CTH_PREC_FP64 for every inner solve; tol /
    maxit override the inner solves' stopping rule when given; reuse_tol > 0
    keeps each equation's multigrid hierarchy while its operator changes by at
    most that much (Grid.set_reuse on the three grids)."""

    def __init__(self, pkg, ni, nj, seed=0, device=0, precision=capi.CTH_PREC_MIXED, tol=None, maxit=None,
                 ndiv_mw=100, Pmw=8.0, mw_tol=1e-10, mw_maxit=400, V_bias=None, reuse_tol=0.0):
        self.ni, self.nj, self.ndiv_mw, self.mw_tol, self.mw_maxit = ni, nj, ndiv_mw, mw_tol, mw_maxit
        geo = pkg.fluid.rectangle_geometry(ni, nj, width_neutIn=2.03e-3)
        ds = pkg.workloads.discharge_state(ni, nj, seed=seed)
        cfg = pkg.workloads.discharge_params(geo, ds["dr"], 5e-3)
        self.geo, self.cfg = geo, cfg
        self.init = {k: np.zeros((ni + 2, nj + 2)) for k in FIELDS}
        self.init.update(ds["fields"])
        self.init["rhoe_old"] = self.init["rhoe"].copy()
        self.g = Grid(ni, nj, geo["ib"], geo["jb"], device=device)
        self.gx = Grid(ni, nj, geo["fxi"], geo["fxj"], device=device)
        self.gr = Grid(ni, nj, geo["fri"], geo["frj"], device=device)
        for gg in (self.g, self.gx, self.gr):
            gg.set_reuse(reuse_tol)
        self.fs = pkg.Fields(self.g)
        self.fs.set_geometry(geo)
        self.fs.set_ion_geometry(geo)
        for k, v in cfg["tables"].items():
            self.fs.set_table(k, v)
        for k, v in cfg["see"].items():
            self.fs.set_table(k, v)
        self.fs.upload("epsr_mw", np.ones((ni + 2, nj + 2)))
        for k, v in self.init.items():
            self.fs.upload(k, v)
        P = {k: (dict(v) if isinstance(v, dict) else v) for k, v in cfg["params"].items()}
        for blk in ("ion", "rhoe", "eps", "neutral"):
            P[blk]["precision"] = precision
            if tol is not None:
                P[blk].update(error_cnv_SOR=tol)
            if maxit is not None:
                P[blk].update(maxITR_SOR=maxit)
        P["phi"]["precision"] = precision
        if V_bias is not None:
            P["phi"]["V_bias"] = float(V_bias)
        if tol is not None:
            P["phi"].update(error_cnv_SOR_phi=tol)
        if maxit is not None:
            P["phi"].update(maxITR_SOR_phi=maxit)
        self.P = P
        self.fs.update_transport_coef(P["transport"])
        wb = pkg.workloads.mw_er_rect(ni, nj, seed=2)
        self.mw_params = dict(wb["params"])
        self.J1r_exc = self.mw_params["J1r_exc"]
        self.m3 = Microwave3(ni, nj, device=device)
        self.e3 = self.m3.planes(3)
        self.j3 = self.m3.planes(3)
        self.port = rect_port(self.mw_params, Pmw)
        self.mw = MicrowaveUpdate(self.fs, self.m3, self.mw_params, self.port, ndiv_mw=ndiv_mw, maxit=mw_maxit,
                                  tol=mw_tol, E3=self.e3, J3=self.j3)

    def microwave(self, stream=None) -> dict:
        """solve_Microwave + update_energy_profile (flag_mwRef = 0) on the current state."""
        out = self.mw.run(self.gx, self.gr, stream=stream)
        self.J1r_exc = out["J1r_exc"]
        return out

    def step(self, stream=None) -> dict:
        r = self.fs.fluid_step(self.gx, self.gr, self.P, stream=stream)
        if r["solver_rc"] < 0:
            raise capi.CathodeError(r["solver_rc"], "fluid step failed")
        if self.mw.due(self.P["itime"]):
            r["mw"] = self.microwave(stream=stream)
        return r

    def fields(self, names) -> dict:
        return {k: self.fs.download(k) for k in names}

    def microwave_fields(self):
        """E1x, E1r, E1p as [i][j] complex arrays."""
        return [np.ascontiguousarray(self.e3[c, :, :self.ni + 2].cpu().numpy().T) for c in range(3)]

    def close(self):
        self.mw.close()
        self.m3.close()
        self.fs.close()
        for x in (self.g, self.gx, self.gr):
            x.close()
