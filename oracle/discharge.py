"""The time loop of src/main.cpp:170-257 restated on the CPU for the r-z
rectangle discharge: oracle.fluid.fluid_step every step and every ``ndiv_mw``
steps the microwave update (solve_Microwave on the magnetised system of the
rectangle, its ghost pass, update_energy_profile with flag_mwRef = 0).

TEST INFRASTRUCTURE ONLY (the checker of the device loop,
02_cathode-08_modulerev_b200/discharge.py)."""
from __future__ import annotations

import numpy as np

from . import direct_solve
from . import fluid
from . import microwave as mw


class RectangleChain:
    """state: the initial fields ([i][j], the reference's names); cfg: the parameter
    blocks, tables and SEE yields of workloads.discharge_params; geo: the
    package's rectangle geometry (xL, x6, width_neutIn of the neutral inlet)."""

    def __init__(self, state, cfg, geo, ni, nj, ndiv_mw=100, Pmw=8.0, J1r_exc=0.212687):
        self.ni, self.nj, self.ndiv_mw, self.Pmw = ni, nj, ndiv_mw, Pmw
        self.og = fluid.rectangle_geometry(ni, nj)
        P = {k: (dict(v) if isinstance(v, dict) else v) for k, v in cfg["params"].items()}
        P["neutral"].update(xL=geo["xL"], x6=geo["x6"], width_neutIn=geo["width_neutIn"])
        self.P = P
        self.tables = cfg["tables"]
        self.see = (cfg["see"]["coefEISEE_eb_table"], cfg["see"]["coefEISEE_rd_table"],
                    cfg["see"]["coefEISEE_ts_table"], P["phi"]["dTe_SEE"])
        self.s = fluid.update_transport_coef(dict(state), self.tables, P["transport"], self.og["flags"])
        self.p = mw.er_rect_params(ni, nj, J1r_exc=J1r_exc)
        self.p["rmin"] = 0.0
        self.lists = mw.rect_mw_lists(ni, nj, self.p)
        zero = np.zeros((ni + 2, nj + 2), complex)
        self.E = [zero.copy(), zero.copy(), zero.copy()]
        self.J1r_exc = J1r_exc

    def _solve(self, aP, aE, aW, aN, aS, b, ib, jb):
        return direct_solve(dict(ni=self.ni, nj=self.nj, i_bl=ib, j_bl=jb, aP=aP, aE=aE, aW=aW, aN=aN, aS=aS, b=b))

    def microwave(self):
        ni, nj, s = self.ni, self.nj, self.s
        p = dict(self.p, J1r_exc=self.J1r_exc)
        epsr = np.ones((ni + 2, nj + 2))
        sysd = mw.mag_rect_system(s["rhoe"], s["nu_m1"], s["Bx"], s["Br"], epsr, p)
        E = mw.mag_rect_solve(sysd)
        start = [np.where(sysd["masks"][k], E[k], self.E[k]) for k in range(3)]
        self.E = list(mw.mag_ghosts(start, s["Er"], epsr, p, self.lists, 0))
        prof, Psum = mw.energy_profile(*self.E, s["rhoe"], s["nu_m1"], s["Bx"], s["Br"], p,
                                       [(2, ni, 1, nj)], [(1, ni, 2, nj)], [(1, ni, 1, nj)])
        port = dict(dx=p["dx"], dr=p["dr"], rmin=0.0, omegam=p["omegam"], r1=p["r1"], r2=p["r2"], Z0=50.0,
                    Pmw=self.Pmw, S11=0j, S21=1 + 0j, S12=1 + 0j, S22=0j, flag_mwRef=0, i_ref=1, j_out=0, i_out0=0,
                    i_out1=0, jf0=0, jf1=0)
        planes, res = mw.mw_port_rescale(*self.E, [prof["J1x"], prof["J1r"], prof["J1p"]], None, prof["Pabs"],
                                         sum(Psum), port)
        s["Pabs"] = planes["Pabs"]
        self.J1r_exc *= res["J1r_exc_factor"]
        return dict(power_sum=sum(Psum), ratio=res["ratio"])

    def step(self):
        self.s = fluid.fluid_step(self.s, self.P, self.og, self.see, self.tables, self._solve)
        if self.P["itime"] % self.ndiv_mw == 0:
            return self.microwave()
        return None
