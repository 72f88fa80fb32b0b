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


class _Plane:
    """A raw device pointer with the data_ptr() of a torch tensor."""

    def __init__(self, p):
        self.p = p

    def data_ptr(self):
        return self.p


FIELDS = ("rhoe", "rhoi", "rhon", "rhom", "Te", "Bx", "Br", "rhoeps", "phi", "Ex", "Er", "nUex", "nUer", "Uix",
          "Uir", "Uip", "rhoUix", "rhoUir", "rhoUix_wall", "rhoUir_wall", "rhoUex", "rhoUer", "rhoUex_wall",
          "rhoUer_wall", "Gx", "Gr", "Gx_wall", "Gr_wall", "rhoUnx", "rhoUnr", "rhoUnx_wall", "rhoUnr_wall",
          "rhoUmx", "rhoUmr", "rhoUmx_wall", "rhoUmr_wall", "nu_ano", "nu_ano_IAT", "Pabs", "rhoe_old")


class RectangleDischarge:
    """The seeded discharge of workloads.discharge_state / discharge_params on the
    ni (z) x nj (r) rectangle with its microwave update every ``ndiv_mw`` steps.
    precision: CTH_PREC_MIXED or CTH_PREC_FP64 for every inner solve; tol /
    maxit override the inner solves' stopping rule when given."""

    def __init__(self, pkg, ni, nj, seed=0, device=0, precision=capi.CTH_PREC_MIXED, tol=None, maxit=None,
                 ndiv_mw=100, Pmw=8.0, mw_tol=1e-10, mw_maxit=400):
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
        self.eprm = {k: self.mw_params.get(k, 0.0) for k in ("dx", "dr", "rmin", "omegam", "masse")}
        self.port = dict(dx=self.eprm["dx"], dr=self.eprm["dr"], rmin=self.eprm["rmin"], omegam=self.eprm["omegam"],
                         r1=self.mw_params["r1"], r2=self.mw_params["r2"], Z0=50.0, Pmw=Pmw, S11=0j, S21=1 + 0j,
                         S12=1 + 0j, S22=0j, flag_mwRef=0, i_ref=1, j_out=0, i_out0=0, i_out1=0, jf0=0, jf1=0)

    def microwave(self, stream=None) -> dict:
        """solve_Microwave + update_energy_profile (flag_mwRef = 0) on the current state."""
        fs = self.fs
        f3 = [_Plane(fs.ptr(k)) for k in ("rhoe", "nu_m1", "Bx", "Br", "epsr_mw")]
        prm = dict(self.mw_params, J1r_exc=self.J1r_exc)
        self.m3.assemble_dev(*f3, prm, stream=stream)
        st = self.m3.solve_dev(maxITR=self.mw_maxit, error_cnv=self.mw_tol, out=self.e3, stream=stream)[1]
        self.m3.fill_ghosts(self.e3, f3[4], prm, Er_dc=_Plane(fs.ptr("Er")), stream=stream)
        er = fs.update_energy_profile(self.gx, self.gr, self.eprm, self.e3[0], self.e3[1], self.e3[2], self.j3[0],
                                      self.j3[1], self.j3[2], stream=stream)
        pr = fs.mw_port_rescale(self.port, er["power_sum"], stream=stream)
        self.J1r_exc *= pr["J1r_exc_factor"]
        return dict(solve=st.as_dict(), power_sum=er["power_sum"], ratio=pr["ratio"])

    def step(self, stream=None) -> dict:
        r = self.fs.fluid_step(self.gx, self.gr, self.P, stream=stream)
        if r["solver_rc"] < 0:
            raise capi.CathodeError(r["solver_rc"], "fluid step failed")
        if self.P["itime"] % self.ndiv_mw == 0:
            r["mw"] = self.microwave(stream=stream)
        return r

    def fields(self, names) -> dict:
        return {k: self.fs.download(k) for k in names}

    def microwave_fields(self):
        """E1x, E1r, E1p as [i][j] complex arrays."""
        return [np.ascontiguousarray(self.e3[c, :, :self.ni + 2].cpu().numpy().T) for c in range(3)]

    def close(self):
        self.m3.close()
        self.fs.close()
        for x in (self.g, self.gx, self.gr):
            x.close()
