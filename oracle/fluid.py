"""CPU restatement of the reference's fluid-side assembly (FluidModule).

TEST INFRASTRUCTURE ONLY (checker; the product never imports it).

Arrays follow the reference: (ni+2, nj+2) float64 [i][j]; x-face arrays at
i-1/2 and r-face arrays at j-1/2 use the same shape (fluidModule.hpp:156-173).
"""
from __future__ import annotations

import numpy as np

BOLTZ = 1.380649e-23
E0 = 1.60217662e-19
EPS0 = 8.8541878128e-12

# boundary flag bits of a cell (1 = the side is an ordinary interior face)
F_BLX, F_BRX, F_BLR_WALL, F_BLR_CEN, F_BRR_WALL, F_BRR_OPEN = 1, 2, 4, 8, 16, 32


def cathode_blocks(ni: int = 194, nj: int = 70, xR: float = 0.0388, rmax: float = 0.014):
    """Cell blocks of the reference's cathode geometry (initialModule.hpp:219-263)."""
    dx, dr = xR / ni, rmax / nj
    x2, x3, x4, x5, x6 = 5.6e-3 + 7.8e-3, 10.0e-3 + 7.8e-3, 15.0e-3 + 7.8e-3, 20.0e-3 + 7.8e-3, 7.8e-3
    r1, r3, r4, r5 = 0.6e-3, 4.0e-3, 9.0e-3, 2.0e-3
    ib = [[int(x6 / dx + 0.5) + 1, int(x2 / dx - 0.5) + 1],
          [int(x2 / dx + 0.5) + 1, int(x4 / dx - 0.5) + 1],
          [int(x2 / dx + 0.5) + 1, int(x3 / dx - 0.5) + 1],
          [int(x3 / dx + 0.5) + 1, int(x5 / dx - 0.5) + 1],
          [int(x5 / dx + 0.5) + 1, int(xR / dx - 0.5) + 1]]
    jb = [[int(r3 / dr + 0.5) + 1, int(r4 / dr - 0.5) + 1],
          [int(r5 / dr + 0.5) + 1, int(r4 / dr - 0.5) + 1],
          [int(r1 / dr + 0.5) + 1, int(r5 / dr - 0.5) + 1],
          [int(0.0 / dr + 0.5) + 1, int(r5 / dr - 0.5) + 1],
          [int(0.0 / dr + 0.5) + 1, int(rmax / dr - 0.5) + 1]]
    return np.array(ib, np.int32), np.array(jb, np.int32)


def cathode_flags(ni, nj, ib, jb) -> np.ndarray:
    """Per-cell side flags of the fluid blocks 0..4, the expressions repeated in
    every FluidModule sweep (e.g. fluidModule.hpp:2660-2686, :5838-5860)."""
    fl = np.zeros((ni + 2, nj + 2), np.uint8)
    for blk in range(5):
        for i in range(ib[blk][0], ib[blk][1] + 1):
            for j in range(jb[blk][0], jb[blk][1] + 1):
                bLx = (i != ib[0][0] or blk != 0)
                bLx = bLx and (i != ib[2][0] or j > jb[0][0] - 1)
                bLx = bLx and (i != ib[3][0] or j > jb[2][0] - 1)
                bLx = bLx and (i != ib[4][0] or j < jb[1][0])
                bRx = (i != ib[1][1] or j < jb[1][0])
                bRx = bRx and (i != ib[4][1])
                bLr_wall = (j != jb[0][0] or i > ib[0][1])
                bLr_wall = bLr_wall and (j != jb[2][0] or i > ib[2][1])
                bLr_cen = (j != jb[3][0])
                bRr_wall = (j != jb[0][1] or blk > 2)
                bRr_wall = bRr_wall and (j != jb[3][1] or i < ib[1][1] + 1 or i > ib[3][1])
                bRr_open = (j != jb[4][1] or blk != 4)
                fl[i, j] = (F_BLX * bLx | F_BRX * bRx | F_BLR_WALL * bLr_wall | F_BLR_CEN * bLr_cen |
                            F_BRR_WALL * bRr_wall | F_BRR_OPEN * bRr_open)
    return fl


def rectangle_flags(ni, nj) -> np.ndarray:
    """Rectangle: z = 0 wall, z = L electrode, r = 0 axis, r = R wall."""
    fl = np.zeros((ni + 2, nj + 2), np.uint8)
    i = np.arange(1, ni + 1)[:, None]
    j = np.arange(1, nj + 1)[None, :]
    fl[1:ni + 1, 1:nj + 1] = (F_BLX * (i != 1) | F_BRX * (i != ni) | F_BLR_WALL |
                              F_BLR_CEN * (j != 1) | F_BRR_WALL * (j != nj) | F_BRR_OPEN)
    return fl


def func_Te(value, Te, dTe):
    """miniFuncs.hpp:35-46 (elementwise)."""
    value = np.asarray(value)
    iL = np.trunc(Te / dTe).astype(np.int64)
    iR = iL + 1
    Te_L = iL * dTe
    ok = iR < value.size - 1
    iLc = np.clip(iL, 0, value.size - 1)
    iRc = np.clip(iR, 0, value.size - 1)
    interp = (value[iRc] - value[iLc]) / (dTe + 1e-100) * (Te - Te_L) + value[iLc]
    return np.where(ok, interp, value[-1])


def func_dTe(value, Te, dTe):
    """miniFuncs.hpp:53-68 (elementwise)."""
    value = np.asarray(value)
    iL = np.trunc(Te / dTe).astype(np.int64)
    iR = iL + 1
    hi = iR >= value.size - 1
    iL = np.where(hi, value.size - 2, iL)
    iR = np.where(hi, value.size - 1, iR)
    return (value[iR] - value[iL]) / (iR * dTe - iL * dTe + 1e-100)


def func_Ei(value, Ei, dEi, massi):
    """miniFuncs.hpp:75-91 (elementwise)."""
    value = np.asarray(value)
    iL = np.trunc(Ei / dEi).astype(np.int64)
    iR = iL + 1
    Ei_L = iL * dEi
    ok = iR < value.size - 1
    iLc = np.clip(iL, 0, value.size - 1)
    iRc = np.clip(iR, 0, value.size - 1)
    interp = (value[iRc] - value[iLc]) / (dEi + 1e-100) * (Ei - Ei_L) + value[iLc]
    imax = value.size - 1
    v_max = np.sqrt(imax * dEi / massi)
    v_tmp = np.sqrt(Ei / massi)
    ext = value[-1] / v_max * v_tmp
    return np.where(ok, interp, ext)


TABLES = ("nu_elas_N", "nu_exc_N", "nu_excReso_N", "nu_excMeta_N", "nu_ionz_N", "nu_ionzStep_N",
          "nu_excStep_N", "nu_super_N", "rate_eloss_n_N", "rate_eloss_m_N", "nui_m_N")


def update_transport_coef(f: dict, tb: dict, prm: dict, flags: np.ndarray) -> dict:
    """FluidModule::update_transport_coef (fluidModule.hpp:5799-5976).

    f: cell fields rhoe, rhoi, rhon, rhom, Te, Bx, Br, nu_ano, nu_ano_IAT, Uip;
       x-face fields Uix, rhoUex; r-face fields Uir, rhoUer.
    tb: rate tables (TABLES); prm: masse, massi, Ti, nu_eff, flag_Bohm,
    flag_Sagdeev, dTe, dEi, dr, rmin.  flags: per-cell side flags (0 = not a
    fluid cell).  Returns the updated fields."""
    ni, nj = f["rhoe"].shape[0] - 2, f["rhoe"].shape[1] - 2
    r = prm["rmin"] + (np.arange(nj + 2) - 0.5) * prm["dr"]
    out = {k: v.copy() for k, v in f.items()}
    blk = flags != 0
    rhoe_max = f["rhoe"][blk].max() if blk.any() else 0.0
    ratio_rhoe = 0.001
    me, mi, Ti = prm["masse"], prm["massi"], prm["Ti"]
    Mache = f.get("Mache", np.zeros_like(f["rhoe"])).copy()
    IAT = f["nu_ano_IAT"].copy()
    for i in range(1, ni + 1):
        for j in range(1, nj + 1):
            if not blk[i, j]:
                continue
            fl = int(flags[i, j])
            bLx = float(bool(fl & F_BLX)); bRx = float(bool(fl & F_BRX))
            bLr = float(bool(fl & F_BLR_WALL)); bRr = float(bool(fl & F_BRR_WALL))
            ut = np.sqrt(2.0 * BOLTZ * f["Te"][i, j] / me)
            rL = (r[j] + r[j - 1]) / 2.0
            rR = (r[j] + r[j + 1]) / 2.0
            rhoUex_t = (f["rhoUex"][i + 1, j] * bRx + f["rhoUex"][i, j] * bLx) / 2.0
            rhoUer_t = (rR * f["rhoUer"][i, j + 1] * bRr + rL * f["rhoUer"][i, j] * bLr) / (2.0 * r[j])
            Uex = rhoUex_t / (f["rhoe"][i, j] + rhoe_max * ratio_rhoe)
            Uer = rhoUer_t / (f["rhoe"][i, j] + rhoe_max * ratio_rhoe)
            Uix = (f["Uix"][i, j] + f["Uix"][i + 1, j]) / 2.0
            Uir = (rL * f["Uir"][i, j] + rR * f["Uir"][i, j + 1]) / (2.0 * r[j])
            Mache[i, j] = np.sqrt(Uex ** 2 + Uer ** 2) / (ut + 100.0)
            cs = np.sqrt(2.0 * BOLTZ * (f["Te"][i, j] + Ti) / mi)
            omega_pi = np.sqrt(f["rhoi"][i, j] * E0 * E0 / (mi * EPS0))
            ud = np.sqrt((Uex - Uix) ** 2 + (Uer - Uir) ** 2)
            IAT[i, j] = 0.01 * omega_pi * ud / cs * f["Te"][i, j] / Ti
    out["Mache"] = Mache
    out["nu_ano_IAT"] = IAT
    Te, dTe = f["Te"], prm["dTe"]
    rhon, rhom = f["rhon"], f["rhom"]
    out["nu_elas"] = rhon * func_Te(tb["nu_elas_N"], Te, dTe)
    out["nu_exc"] = rhon * func_Te(tb["nu_exc_N"], Te, dTe)
    out["nu_excReso"] = rhon * func_Te(tb["nu_excReso_N"], Te, dTe)
    out["nu_excMeta"] = rhon * func_Te(tb["nu_excMeta_N"], Te, dTe)
    out["nu_ionz"] = rhon * func_Te(tb["nu_ionz_N"], Te, dTe)
    out["nu_ionzStep"] = rhom * func_Te(tb["nu_ionzStep_N"], Te, dTe)
    out["nu_excStep"] = rhom * func_Te(tb["nu_excStep_N"], Te, dTe)
    out["nu_super"] = rhom * func_Te(tb["nu_super_N"], Te, dTe)
    nu_m_real = rhon * func_Te(tb["nu_elas_N"], Te, dTe)
    out["nu_m"] = nu_m_real + float(prm["flag_Bohm"]) * f["nu_ano"] + float(prm["flag_Sagdeev"]) * IAT
    out["nu_m1"] = nu_m_real + prm["nu_eff"]
    out["rate_ionize"] = f["rhoe"] * (out["nu_ionz"] + out["nu_ionzStep"])
    vv = np.zeros_like(Te)
    rL = ((r[1:nj + 1] + r[0:nj]) / 2.0)[None, :]
    rR = ((r[1:nj + 1] + r[2:nj + 2]) / 2.0)[None, :]
    Uix = (f["Uix"][1:ni + 1, 1:nj + 1] + f["Uix"][2:ni + 2, 1:nj + 1]) / 2.0
    Uir = (rL * f["Uir"][1:ni + 1, 1:nj + 1] + rR * f["Uir"][1:ni + 1, 2:nj + 2]) / (2.0 * r[1:nj + 1][None, :])
    Uip = f["Uip"][1:ni + 1, 1:nj + 1]
    vv[1:ni + 1, 1:nj + 1] = Uix * Uix + Uir * Uir + Uip * Uip
    out["nui_m"] = rhon * func_Ei(tb["nui_m_N"], mi * vv, prm["dEi"], mi)
    out["rate_eloss"] = rhon * func_Te(tb["rate_eloss_n_N"], Te, dTe) + rhom * func_Te(tb["rate_eloss_m_N"], Te, dTe)
    out["delossdeps"] = (2.0 / (3.0 * BOLTZ) * rhon * func_dTe(tb["rate_eloss_n_N"], Te, dTe) +
                         2.0 / (3.0 * BOLTZ) * rhom * func_dTe(tb["rate_eloss_m_N"], Te, dTe))
    num = out["nu_m"]
    out["mu_para"] = E0 / (me * num + 1e-100)
    Bmag = np.sqrt(f["Bx"] ** 2 + f["Br"] ** 2)
    Om = E0 * Bmag / (me * num + 1e-100)
    Omx = E0 * f["Bx"] / (me * num + 1e-100)
    Omr = E0 * f["Br"] / (me * num + 1e-100)
    deno = 1.0 + Om * Om
    out["mu_xx"] = out["mu_para"] * (1.0 + Omx * Omx) / deno
    out["mu_rr"] = out["mu_para"] * (1.0 + Omr * Omr) / deno
    out["mu_xr"] = out["mu_para"] * (Omx * Omr) / deno
    out["mu_perp"] = out["mu_para"] / deno
    out["mu_min"] = out["mu_para"] * 2.0 / deno
    return out


def synthetic_tables(n_e: int = 1801, n_i: int = 40, d_eps_eV: float = 150.0 / 1800, d_ei_eV: float = 1.0):
    """Rate tables on the reference's uniform mean-energy grid (input_BOLSIG_data,
    inputModule.hpp:1413-1655): electron tables at mean energy k*d_eps (eV), so
    Te = 2/3 eps; ionisation k = 1e-13 Te^0.5 exp(-12.13/Te) m^3/s with threshold
    12.13 eV, elastic 2e-13 m^3/s; ion momentum table 5.2e-16 m^3/s."""
    eps = np.arange(n_e) * d_eps_eV
    Te = 2.0 / 3.0 * eps
    with np.errstate(divide="ignore", over="ignore", invalid="ignore"):
        kion = np.where(Te > 0, 1e-13 * np.sqrt(Te) * np.exp(-12.13 / np.maximum(Te, 1e-30)), 0.0)
    kel = np.full(n_e, 2e-13)
    tb = {k: np.zeros(n_e) for k in TABLES if k != "nui_m_N"}
    tb["nu_elas_N"] = kel
    tb["nu_ionz_N"] = kion
    tb["nu_exc_N"] = 0.5 * kion
    tb["nu_ionzStep_N"] = 0.1 * kion
    tb["rate_eloss_n_N"] = kion * 12.13 + 0.5 * kion * 8.31
    tb["rate_eloss_m_N"] = 0.1 * kion * 3.9
    tb["nui_m_N"] = np.full(n_i, 5.2e-16)
    dTe = d_eps_eV * 2.0 / 3.0 * E0 / BOLTZ
    dEi = d_ei_eV * E0
    return tb, dTe, dEi


def bolsig_tables(text_e: str, text_i: str):
    """InputModule::input_BOLSIG_data (inputModule.hpp:1413-1655) on the two CSV
    texts: row 1 names each collision column's type, row 2 its threshold (eV),
    then one row per mean energy k*delta.  Columns of one type add into that
    type's rate table; the energy-loss tables sum rate*threshold over the ground
    state types (elastic .. ionisation) and over the stepwise / superelastic
    types.  Returns (tables, dTe, dEi) with dTe = delta*2/3*e/k_B (K) and
    dEi = delta_i*e (J)."""
    kinds = {"Elastic": 0, "Excitation": 1, "Excitation_reso": 2, "Excitation_meta": 3, "Ionization": 4,
             "Ionization_step": 5, "Excitation_step": 6}
    names = ("nu_elas_N", "nu_exc_N", "nu_excReso_N", "nu_excMeta_N", "nu_ionz_N", "nu_ionzStep_N",
             "nu_excStep_N", "nu_super_N")
    rows = [ln.split(",") for ln in text_e.splitlines() if ln.strip()]
    ctype = [kinds.get(c.strip(), 7) for c in rows[0][1:]]
    thr = np.array([float(v) for v in rows[1][1:]]) * E0
    data = np.array([[float(v) for v in r[1:len(ctype) + 1]] for r in rows[2:]])
    delta = float(rows[3][0]) - float(rows[2][0])
    tb = {k: np.zeros(data.shape[0]) for k in names + ("rate_eloss_n_N", "rate_eloss_m_N")}
    for c, t in enumerate(ctype):
        tb[names[t]] += data[:, c]
        tb["rate_eloss_n_N" if t <= 4 else "rate_eloss_m_N"] += data[:, c] * thr[c]
    rows_i = [ln.split(",") for ln in text_i.splitlines() if ln.strip()]
    data_i = np.array([[float(v) for v in r[1:len(rows_i[0])]] for r in rows_i[2:]])
    tb["nui_m_N"] = data_i.sum(axis=1)
    delta_i = float(rows_i[3][0]) - float(rows_i[2][0])
    return tb, delta * 2.0 / 3.0 * E0 / BOLTZ, delta_i * E0
