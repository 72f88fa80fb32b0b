"""CPU restatement of the reference's fluid-side assembly (FluidModule).

TEST INFRASTRUCTURE ONLY (checker; the product never imports it).

Arrays follow the reference: (ni+2, nj+2) float64 [i][j]; x-face arrays at
i-1/2 and r-face arrays at j-1/2 use the same shape (fluidModule.hpp:156-173).
"""
from __future__ import annotations

import numpy as np


def _exp(x):
    """exp() of the C library, as the reference evaluates it (numpy's vectorised exp
    differs by one ulp on a few per cent of arguments)."""
    import oracle
    return oracle.libm_exp(x)

BOLTZ = 1.380649e-23
E0 = 1.60217662e-19
EPS0 = 8.8541878128e-12

# boundary flag bits of a cell (1 = the side is an ordinary interior face);
# F_BRX_BIAS marks the cells whose right wall is the biased electrode
F_BLX, F_BRX, F_BLR_WALL, F_BLR_CEN, F_BRR_WALL, F_BRR_OPEN = 1, 2, 4, 8, 16, 32
F_BRX_BIAS = 64


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
                            F_BRR_WALL * bRr_wall | F_BRR_OPEN * bRr_open |
                            F_BRX_BIAS * (blk == 4 and i == ib[4][1]))
    return fl


def rectangle_flags(ni, nj) -> np.ndarray:
    """Rectangle: z = 0 wall, z = L electrode, r = 0 axis, r = R wall."""
    fl = np.zeros((ni + 2, nj + 2), np.uint8)
    i = np.arange(1, ni + 1)[:, None]
    j = np.arange(1, nj + 1)[None, :]
    fl[1:ni + 1, 1:nj + 1] = (F_BLX * (i != 1) | F_BRX * (i != ni) | F_BLR_WALL |
                              F_BLR_CEN * (j != 1) | F_BRR_WALL * (j != nj) | F_BRR_OPEN |
                              F_BRX_BIAS * (i == ni))
    return fl


def func_Te(value, Te, dTe):
    """miniFuncs.hpp:35-46 (elementwise).  Below the table (Te / dTe <= -1, where
    the reference reads before its vector) the first interval is extrapolated,
    as the device does."""
    value = np.asarray(value)
    iL = np.maximum(np.trunc(Te / dTe), 0).astype(np.int64)
    iR = iL + 1
    Te_L = iL * dTe
    ok = iR < value.size - 1
    iLc = np.clip(iL, 0, value.size - 1)
    iRc = np.clip(iR, 0, value.size - 1)
    interp = (value[iRc] - value[iLc]) / (dTe + 1e-100) * (Te - Te_L) + value[iLc]
    return np.where(ok, interp, value[-1])


def func_dTe(value, Te, dTe):
    """miniFuncs.hpp:53-68 (elementwise); below the table the first interval's slope."""
    value = np.asarray(value)
    iL = np.maximum(np.trunc(Te / dTe), 0).astype(np.int64)
    iR = iL + 1
    hi = iR >= value.size - 1
    iL = np.where(hi, value.size - 2, iL)
    iR = np.where(hi, value.size - 1, iR)
    return (value[iR] - value[iL]) / (iR * dTe - iL * dTe + 1e-100)


def func_Ei(value, Ei, dEi, massi):
    """miniFuncs.hpp:75-91 (elementwise); below the table the first interval extrapolated."""
    value = np.asarray(value)
    iL = np.maximum(np.trunc(Ei / dEi), 0).astype(np.int64)
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
    # anomalous frequency on the fluid cells (:5818-5908), evaluated for all grid cells
    # and kept where the cell is in a block
    I, J = slice(1, ni + 1), slice(1, nj + 1)
    fl = flags[I, J].astype(np.int64)
    bLx = ((fl & F_BLX) != 0).astype(float); bRx = ((fl & F_BRX) != 0).astype(float)
    bLr = ((fl & F_BLR_WALL) != 0).astype(float); bRr = ((fl & F_BRR_WALL) != 0).astype(float)
    Te = f["Te"][I, J]
    rj = r[J][None, :]
    rL = (r[1:nj + 1] + r[0:nj])[None, :] / 2.0
    rR = (r[1:nj + 1] + r[2:nj + 2])[None, :] / 2.0
    ut = np.sqrt(2.0 * BOLTZ * Te / me)
    rhoUex_t = (f["rhoUex"][2:ni + 2, J] * bRx + f["rhoUex"][I, J] * bLx) / 2.0
    rhoUer_t = (rR * f["rhoUer"][I, 2:nj + 2] * bRr + rL * f["rhoUer"][I, J] * bLr) / (2.0 * rj)
    den = f["rhoe"][I, J] + rhoe_max * ratio_rhoe
    Uex = rhoUex_t / den
    Uer = rhoUer_t / den
    Uix = (f["Uix"][I, J] + f["Uix"][2:ni + 2, J]) / 2.0
    Uir = (rL * f["Uir"][I, J] + rR * f["Uir"][I, 2:nj + 2]) / (2.0 * rj)
    cs = np.sqrt(2.0 * BOLTZ * (Te + Ti) / mi)
    omega_pi = np.sqrt(f["rhoi"][I, J] * E0 * E0 / (mi * EPS0))
    ud = np.sqrt((Uex - Uix) * (Uex - Uix) + (Uer - Uir) * (Uer - Uir))
    sel = blk[I, J]
    with np.errstate(all="ignore"):
        Mache[I, J] = np.where(sel, np.sqrt(Uex * Uex + Uer * Uer) / (ut + 100.0), Mache[I, J])
        IAT[I, J] = np.where(sel, 0.01 * omega_pi * ud / cs * Te / Ti, IAT[I, J])
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
        kion = np.where(Te > 0, 1e-13 * np.sqrt(Te) * _exp(-12.13 / np.maximum(Te, 1e-30)), 0.0)
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


def see_tables(text: str):
    """InputModule::input_SEE_data (inputModule.hpp:605-657): columns EB, RD, TS
    of coefEISEE.csv against mean energy; dTe_SEE = delta*0.5*e/k_B."""
    rows = [ln.split(",") for ln in text.splitlines() if ln.strip()][1:]
    a = np.array([[float(v) for v in r[:4]] for r in rows])
    return a[:, 1].copy(), a[:, 2].copy(), a[:, 3].copy(), (a[1, 0] - a[0, 0]) * 0.5 * E0 / BOLTZ


# ----------------------------------------------------------------------------
# geometry of the PC sweeps: cell blocks, face blocks and the wall segments in
# the order the reference visits them
# ----------------------------------------------------------------------------

def cathode_geometry(ni: int = 194, nj: int = 70, xR: float = 0.0388, rmax: float = 0.014) -> dict:
    """Cell blocks, x-/r-face blocks (initialModule.hpp:219-345) and the wall
    segments of solve_phi_couple_wdTe_wSEE_PC (fluidModule.hpp:2149-2240):
    kind L/R/RB (left, right, right at V_bias), D/U (lower, upper wall),
    O (upper open); each (kind, i0, i1, j0, j1) over cells."""
    dx, dr = xR / ni, rmax / nj
    x2, x3, x4, x5, x6 = 5.6e-3 + 7.8e-3, 10.0e-3 + 7.8e-3, 15.0e-3 + 7.8e-3, 20.0e-3 + 7.8e-3, 7.8e-3
    r1, r3, r4, r5 = 0.6e-3, 4.0e-3, 9.0e-3, 2.0e-3
    ib, jb = cathode_blocks(ni, nj, xR, rmax)
    lo = lambda v, d, k: int(v / d + 0.5) + k
    hi = lambda v, d, k: int(v / d - 0.5) + k
    fxi = [[lo(x6, dx, 2), hi(x2, dx, 2)], [lo(x2, dx, 2), hi(x4, dx, 1)], [lo(x2, dx, 2), hi(x3, dx, 2)],
           [lo(x3, dx, 2), hi(x5, dx, 2)], [lo(x5, dx, 2), hi(xR, dx, 1)]]
    fxj = [[lo(r3, dr, 1), hi(r4, dr, 1)], [lo(r5, dr, 1), hi(r4, dr, 1)], [lo(r1, dr, 1), hi(r5, dr, 1)],
           [lo(0.0, dr, 1), hi(r5, dr, 1)], [lo(0.0, dr, 1), hi(rmax, dr, 1)]]
    fri = [[lo(x6, dx, 1), hi(x2, dx, 1)], [lo(x2, dx, 1), hi(x4, dx, 1)], [lo(x2, dx, 1), hi(x3, dx, 1)],
           [lo(x3, dx, 1), hi(x5, dx, 1)], [lo(x5, dx, 1), hi(xR, dx, 1)]]
    frj = [[lo(r3, dr, 2), hi(r4, dr, 1)], [lo(r5, dr, 1), hi(r4, dr, 1)], [lo(r1, dr, 2), hi(r5, dr, 1)],
           [lo(0.0, dr, 2), hi(r5, dr, 1)], [lo(0.0, dr, 2), hi(rmax, dr, 1)]]
    segs = [("L", ib[0][0], ib[0][0], jb[0][0], jb[0][1]),          # z0
            ("L", ib[2][0], ib[2][0], jb[2][0], jb[0][0] - 1),      # z1
            ("L", ib[3][0], ib[3][0], jb[3][0], jb[2][0] - 1),      # z2
            ("L", ib[4][0], ib[4][0], jb[1][0], jb[4][1]),          # z4
            ("R", ib[1][1], ib[1][1], jb[1][0], jb[1][1]),          # z3
            ("RB", ib[4][1], ib[4][1], jb[4][0], jb[4][1]),         # z5
            ("D", ib[0][0], ib[0][1], jb[0][0], jb[0][0]),          # x0
            ("D", ib[2][0], ib[2][1], jb[2][0], jb[2][0]),          # x2
            ("U", ib[0][0], ib[1][1], jb[0][1], jb[0][1]),          # x1
            ("U", ib[1][1] + 1, ib[3][1], jb[3][1], jb[3][1]),      # x4
            ("O", ib[4][0], ib[4][1], jb[4][1], jb[4][1])]          # x5
    # ghost values set after the electron sweeps (fluidModule.hpp:3884-3921 for rhoe,
    # :4878-4914 for Te): (i0, i1, j0, j1, di, dj, rhoe_mode) with rhoe_mode 0 = zero,
    # 1 = copy of the cell; Te is always copied
    ghosts = [(ib[0][0], ib[0][0], jb[0][0], jb[0][1], -1, 0, 0),            # chamber
              (ib[1][0], ib[1][0], jb[1][0], jb[0][0] - 1, -1, 0, 0),        # magnet
              (ib[0][0], ib[0][1], jb[0][0], jb[0][0], 0, -1, 0),            # antenna
              (ib[1][1], ib[1][1], jb[1][0], jb[1][1], 1, 0, 1),             # right open
              (ib[0][0], ib[1][1], jb[0][1], jb[0][1], 0, 1, 1)]             # upper open
    # the energy sweep's lower-wall loop x2 (fluidModule.hpp:4428-4449) sets Gr but not Gr_wall:
    # r-face box (i0, i1, j0, j1) where Gr_wall keeps its value
    keep = [(int(ib[2][0]), int(ib[2][1]), int(jb[2][0]), int(jb[2][0]))]
    return dict(ni=ni, nj=nj, dx=dx, dr=dr, ib=ib, jb=jb, fxi=np.array(fxi), fxj=np.array(fxj),
                fri=np.array(fri), frj=np.array(frj), segs=segs, flags=cathode_flags(ni, nj, ib, jb),
                ghosts=ghosts, energy_keep_walls=keep)


def rectangle_geometry(ni: int, nj: int, Lz: float = 10e-3, Lr: float = 5e-3) -> dict:
    """The r-z rectangle as one fluid block: z = 0 wall (0 V, like z0), z = L
    biased electrode (like z5), r = R wall (like x1), r = 0 axis."""
    one = lambda a, b: np.array([[a, b]])
    segs = [("L", 1, 1, 1, nj), ("RB", ni, ni, 1, nj), ("U", 1, ni, nj, nj)]
    ghosts = [(1, 1, 1, nj, -1, 0, 0), (ni, ni, 1, nj, 1, 0, 1), (1, ni, nj, nj, 0, 1, 1)]
    return dict(ni=ni, nj=nj, dx=Lz / ni, dr=Lr / nj, ib=one(1, ni), jb=one(1, nj), fxi=one(2, ni),
                fxj=one(1, nj), fri=one(1, ni), frj=one(2, nj), segs=segs, flags=rectangle_flags(ni, nj),
                ghosts=ghosts)


def calc_res(new, old, ib, jb, eps, flag_error):
    """calcRes (miniFuncs.hpp:292-376) over the blocks (ib, jb)."""
    d = np.concatenate([(new[a:b + 1, c:e + 1] - old[a:b + 1, c:e + 1]).ravel()
                        for (a, b), (c, e) in zip(ib, jb)])
    o = np.concatenate([old[a:b + 1, c:e + 1].ravel() for (a, b), (c, e) in zip(ib, jb)])
    if flag_error == 0:
        return float(np.abs(d).max())
    if flag_error == 1:
        return float(np.sqrt(np.sum(d ** 2 / (o ** 2 + eps)) / d.size))
    if flag_error == 2:
        return float(np.abs(d).max() / np.abs(o).max())
    with np.errstate(divide="ignore", invalid="ignore"):   # an all-zero field gives NaN, as in the reference
        return float(np.sqrt(np.sum(d ** 2) / np.sum(o ** 2)))


PHI_FIELDS = ("phi", "Ex", "Er", "nUex", "nUer")


def _wall_flux(Te, rhoe, rhoe_old, rhoi, Ui, rhoUm, E_old, h, sign, prm, see):
    """Thermal + SEE electron flux through a wall face (fluidModule.hpp:2348-2457):
    sign -1 for a wall on the low side of the cell, +1 on the high side."""
    vth = np.sqrt(8.0 * BOLTZ * Te / (np.pi * prm["masse"]))
    delta_phi = np.fmax(sign * E_old * h / 2.0, 0.0)
    gpn = sign * 0.25 * vth * _exp(np.fmin(-E0 * delta_phi / (BOLTZ * Te + 1e-100), 100.0))
    eb, rd, ts, dTe_SEE = see
    c = func_Te(eb, Te, dTe_SEE) + func_Te(rd, Te, dTe_SEE) + func_Te(ts, Te, dTe_SEE)
    see_flux = -prm["coefIISEE_ts"] * rhoi * Ui - c * rhoe_old * gpn - prm["coefMISEE_ts"] * rhoUm
    return rhoe * gpn + see_flux


def solve_phi_pc(st: dict, prm: dict, geo: dict, see, solve) -> dict:
    """FluidModule::solve_phi_couple_wdTe_wSEE_PC (fluidModule.hpp:2080-3075).

    st: phi, Ex, Er, nUex, nUer, rhoe, rhoe_old, rhoi, Te, mu_para, mu_perp,
    mu_rr, mu_xr, mu_xx, rate_ionize, Uix, Uir, rhoUmx, rhoUmr (updated copies of
    phi, Ex, Er, nUex, nUer are returned with the residuals).  prm: dt, dx, dr,
    rmin, V_bias, masse, coefIISEE_ts, coefMISEE_ts, maxITR_HES_phi,
    error_cnv_HES_phi, flag_error.  see: (eb, rd, ts, dTe_SEE).
    solve(aP, aE, aW, aN, aS, b, ib, jb) -> block-cell solution (zero start).
    The sweeps run block by block over the face / cell blocks of ``geo`` and
    the wall segments in the reference's order."""
    ni, nj = geo["ni"], geo["nj"]
    dx, dr, dt = prm["dx"], prm["dr"], prm["dt"]
    r = prm["rmin"] + (np.arange(nj + 2) - 0.5) * dr
    fl = geo["flags"].astype(np.int64)
    bLx_c = (fl & F_BLX) != 0
    bRx_c = (fl & F_BRX) != 0
    bLr_c = ((fl & F_BLR_WALL) != 0) & ((fl & F_BLR_CEN) != 0)
    bRrw_c = (fl & F_BRR_WALL) != 0
    bRr_c = bRrw_c & ((fl & F_BRR_OPEN) != 0)
    g = {k: st[k] for k in st}
    phi, Ex, Er = st["phi"].copy(), st["Ex"].copy(), st["Er"].copy()
    nUex, nUer = st["nUex"].copy(), st["nUer"].copy()
    phi_old, Ex_old, Er_old, nUex_old, nUer_old = phi.copy(), Ex.copy(), Er.copy(), nUex.copy(), nUer.copy()
    dphi = phi - phi_old
    segs = geo["segs"]
    # ghost potentials of the walls, once before the iteration (:2149-2240)
    for kind, i0, i1, j0, j1 in segs:
        I, J = slice(i0, i1 + 1), slice(j0, j1 + 1)
        if kind == "L":
            phi[i0 - 1, J] = -phi[i0, J]
        elif kind == "R":
            phi[i0 + 1, J] = -phi[i0, J]
        elif kind == "RB":
            phi[i0 + 1, J] = 2.0 * prm["V_bias"] - phi[i0, J]
        elif kind in ("D",):
            phi[I, j0 - 1] = -phi[I, j0]
        elif kind == "U":
            phi[I, j0 + 1] = -phi[I, j0]
        else:
            phi[I, j0 + 1] = phi[I, j0]
    mu_para, mu_perp, rhoe, Te = g["mu_para"], g["mu_perp"], g["rhoe"], g["Te"]
    ncount = 0
    errs = (0.0, 0.0, 0.0)
    while True:
        ncount += 1
        phi_t, nUex_t, nUer_t = phi.copy(), nUex.copy(), nUer.copy()
        # predicted x flux on the x-face blocks (:2266-2343)
        for (a, b), (c, e) in zip(geo["fxi"], geo["fxj"]):
            I = np.arange(a, b + 1)[:, None]
            J = np.arange(c, e + 1)[None, :]
            rL = (r[J] + r[J - 1]) / 2.0
            rR = (r[J] + r[J + 1]) / 2.0
            mpa = (mu_para[I, J] + mu_para[I - 1, J]) / 2.0
            mpe = (mu_perp[I, J] + mu_perp[I - 1, J]) / 2.0
            mst = mpe * 1.0
            mrr = (g["mu_rr"][I, J] + g["mu_rr"][I - 1, J]) / 2.0
            mxr = (g["mu_xr"][I, J] + g["mu_xr"][I - 1, J]) / 2.0
            ixx = mrr / (mpa * mpe)
            ixr = -mxr / (mpa * mpe)
            rho_t = (rhoe[I, J] + rhoe[I - 1, J]) / 2.0
            dphidx = (phi[I, J] - phi[I - 1, J]) / dx
            dpedx = BOLTZ * (rhoe[I, J] * Te[I, J] - rhoe[I - 1, J] * Te[I - 1, J]) / dx
            bLr, bLrD = bLr_c[I, J], bLr_c[I - 1, J]
            bRr, bRrD = bRrw_c[I, J], bRrw_c[I - 1, J]
            nUer_i = (rR * nUer_t[I, J + 1] * bRr + rL * nUer_t[I, J] * bLr
                      + rR * nUer_t[I - 1, J + 1] * bRrD + rL * nUer_t[I - 1, J] * bLrD) / (4.0 * r[J])
            nUex[I, J] = (nUex_t[I, J] - (ixx * nUex_t[I, J] + ixr * nUer_i) * mst
                          + mst * (rho_t * dphidx - dpedx / E0))
        # x walls (:2346-2457)
        for kind, i0, i1, j0, j1 in segs:
            J = np.arange(j0, j1 + 1)
            if kind == "L":
                nUex[i0, J] = _wall_flux(Te[i0, J], rhoe[i0, J], g["rhoe_old"][i0, J], g["rhoi"][i0, J],
                                         g["Uix"][i0, J], g["rhoUmx"][i0, J], Ex_old[i0, J], dx, -1.0, prm, see)
            elif kind in ("R", "RB"):
                nUex[i0 + 1, J] = _wall_flux(Te[i0, J], rhoe[i0, J], g["rhoe_old"][i0, J], g["rhoi"][i0, J],
                                             g["Uix"][i0 + 1, J], g["rhoUmx"][i0 + 1, J], Ex_old[i0 + 1, J], dx,
                                             1.0, prm, see)
        # predicted r flux on the r-face blocks (:2459-2541)
        for (a, b), (c, e) in zip(geo["fri"], geo["frj"]):
            I = np.arange(a, b + 1)[:, None]
            J = np.arange(c, e + 1)[None, :]
            r_t = (r[J] + r[J - 1]) / 2.0
            mpa = (mu_para[I, J] + mu_para[I, J - 1]) / 2.0
            mpe = (mu_perp[I, J] + mu_perp[I, J - 1]) / 2.0
            mst = mpe * 1.0
            mxx = (g["mu_xx"][I, J] + g["mu_xx"][I, J - 1]) / 2.0
            mxr = (g["mu_xr"][I, J] + g["mu_xr"][I, J - 1]) / 2.0
            irr = mxx / (mpa * mpe)
            ixr = -mxr / (mpa * mpe)
            rho_t = (rhoe[I, J] + rhoe[I, J - 1]) / 2.0
            dphidr = (phi[I, J] - phi[I, J - 1]) / dr
            dpedr = BOLTZ * (rhoe[I, J] * Te[I, J] - rhoe[I, J - 1] * Te[I, J - 1]) / dr
            bLx, bLxD = bLx_c[I, J], bLx_c[I, J - 1]
            bRx, bRxD = bRx_c[I, J], bRx_c[I, J - 1]
            nUex_i = (r[J] * nUex_t[I + 1, J] * bRx + r[J] * nUex_t[I, J] * bLx
                      + r[J - 1] * nUex_t[I + 1, J - 1] * bRxD + r[J - 1] * nUex_t[I, J - 1] * bLxD) / (4.0 * r_t)
            nUer[I, J] = (nUer_t[I, J] - (ixr * nUex_i + irr * nUer_t[I, J]) * mst
                          + mst * (rho_t * dphidr - dpedr / E0))
        # r walls and the open top (:2544-2633)
        for kind, i0, i1, j0, j1 in segs:
            I = np.arange(i0, i1 + 1)
            if kind == "D":
                nUer[I, j0] = _wall_flux(Te[I, j0], rhoe[I, j0], g["rhoe_old"][I, j0], g["rhoi"][I, j0],
                                         g["Uir"][I, j0], g["rhoUmr"][I, j0], Er_old[I, j0], dr, -1.0, prm, see)
            elif kind == "U":
                nUer[I, j0 + 1] = _wall_flux(Te[I, j0], rhoe[I, j0], g["rhoe_old"][I, j0], g["rhoi"][I, j0],
                                             g["Uir"][I, j0 + 1], g["rhoUmr"][I, j0 + 1], Er_old[I, j0 + 1], dr,
                                             1.0, prm, see)
            elif kind == "O":
                nUer[I, j0 + 1] = g["rhoi"][I, j0] * g["Uir"][I, j0 + 1]
        # Poisson coefficients with dielectric relaxation (:2636-2716)
        sh = (ni + 2, nj + 2)
        aP, aE, aW, aN, aS, bb = (np.zeros(sh) for _ in range(6))
        for (a, b), (c, e) in zip(geo["ib"], geo["jb"]):
            I = np.arange(a, b + 1)[:, None]
            J = np.arange(c, e + 1)[None, :]
            rR = (r[J] + r[J + 1]) / 2.0
            rL = (r[J] + r[J - 1]) / 2.0
            qR = (r[J] + r[J + 1]) / 2.0 / r[J]
            qL = (r[J] + r[J - 1]) / 2.0 / r[J]
            mLx = (mu_perp[I, J] + mu_perp[I - 1, J]) / 2.0 * 1.0
            mRx = (mu_perp[I, J] + mu_perp[I + 1, J]) / 2.0 * 1.0
            mLr = (mu_perp[I, J] + mu_perp[I, J - 1]) / 2.0 * 1.0
            mRr = (mu_perp[I, J] + mu_perp[I, J + 1]) / 2.0 * 1.0
            nLx = (rhoe[I, J] + rhoe[I - 1, J]) / 2.0
            nRx = (rhoe[I, J] + rhoe[I + 1, J]) / 2.0
            nLr = (rhoe[I, J] + rhoe[I, J - 1]) / 2.0
            nRr = (rhoe[I, J] + rhoe[I, J + 1]) / 2.0
            bLx, bRx, bLr, bRr = bLx_c[I, J], bRx_c[I, J], bLr_c[I, J], bRr_c[I, J]
            aP[I, J] = (((EPS0 + E0 * dt * nRx * mRx * bRx) + (EPS0 + E0 * dt * nLx * mLx * bLx)) * dr * dr
                        + (qR * (EPS0 + E0 * dt * nRr * mRr * bRr) + qL * (EPS0 + E0 * dt * nLr * mLr * bLr))
                        * dx * dx)
            aE[I, J] = (EPS0 + E0 * dt * nRx * mRx * bRx) * dr * dr
            aW[I, J] = (EPS0 + E0 * dt * nLx * mLx * bLx) * dr * dr
            aN[I, J] = qR * (EPS0 + E0 * dt * nRr * mRr * bRr) * dx * dx
            aS[I, J] = qL * (EPS0 + E0 * dt * nLr * mLr * bLr) * dx * dx
            div = (nUex[I + 1, J] - nUex[I, J]) / dx + (qR * nUer[I, J + 1] - qL * nUer[I, J]) / dr
            lap = -(Ex[I + 1, J] - Ex[I, J]) / dx - (qR * Er[I, J + 1] - qL * Er[I, J]) / dr
            bb[I, J] = ((E0 * g["rhoi"][I, J] - E0 * rhoe[I, J] - E0 * dt * g["rate_ionize"][I, J]
                         + EPS0 * lap + E0 * dt * div) * dx * dx * dr * dr)
        # wall conditions on the coefficients (:2720-2816)
        for kind, i0, i1, j0, j1 in segs:
            I, J = slice(i0, i1 + 1), slice(j0, j1 + 1)
            if kind == "L":
                aP[i0, J] += aW[i0, J]; aW[i0, J] = 0.0
            elif kind in ("R", "RB"):
                aP[i0, J] += aE[i0, J]; aE[i0, J] = 0.0
            elif kind == "D":
                aP[I, j0] += aS[I, j0]; aS[I, j0] = 0.0
            elif kind == "U":
                aP[I, j0] += aN[I, j0]; aN[I, j0] = 0.0
            else:
                aP[I, j0] -= aN[I, j0]; aN[I, j0] = 0.0
        x = solve(aP, aE, aW, aN, aS, bb, geo["ib"], geo["jb"])
        for (a, b), (c, e) in zip(geo["ib"], geo["jb"]):
            dphi[a:b + 1, c:e + 1] = x[a:b + 1, c:e + 1]
        # ghost corrections and wall fields (:2836-2928)
        for kind, i0, i1, j0, j1 in segs:
            I, J = slice(i0, i1 + 1), slice(j0, j1 + 1)
            if kind == "L":
                dphi[i0 - 1, J] = -dphi[i0, J]
                Ex[i0, J] = Ex[i0, J] - (dphi[i0, J] - dphi[i0 - 1, J]) / dx
            elif kind in ("R", "RB"):
                dphi[i0 + 1, J] = -dphi[i0, J]
                Ex[i0 + 1, J] = Ex[i0 + 1, J] - (dphi[i0 + 1, J] - dphi[i0, J]) / dx
            elif kind == "D":
                dphi[I, j0 - 1] = -dphi[I, j0]
                Er[I, j0] = Er[I, j0] - (dphi[I, j0] - dphi[I, j0 - 1]) / dr
            elif kind == "U":
                dphi[I, j0 + 1] = -dphi[I, j0]
                Er[I, j0 + 1] = Er[I, j0 + 1] - (dphi[I, j0 + 1] - dphi[I, j0]) / dr
            else:
                dphi[I, j0 + 1] = dphi[I, j0]
                Er[I, j0 + 1] = 0.0
        phi = phi + dphi
        # fields and flux corrections on the face blocks (:2932-3024)
        for (a, b), (c, e) in zip(geo["fxi"], geo["fxj"]):
            I, J = slice(a, b + 1), slice(c, e + 1)
            Im = slice(a - 1, b)
            Ex[I, J] = -(phi[I, J] - phi[Im, J]) / dx
        for (a, b), (c, e) in zip(geo["fri"], geo["frj"]):
            I, J, Jm = slice(a, b + 1), slice(c, e + 1), slice(c - 1, e)
            Er[I, J] = -(phi[I, J] - phi[I, Jm]) / dr
        for (a, b), (c, e) in zip(geo["fxi"], geo["fxj"]):
            I, J, Im = slice(a, b + 1), slice(c, e + 1), slice(a - 1, b)
            mst = (mu_perp[I, J] + mu_perp[Im, J]) / 2.0 * 1.0
            rho_t = (rhoe[I, J] + rhoe[Im, J]) / 2.0
            nUex[I, J] = nUex[I, J] + mst * rho_t * ((dphi[I, J] - dphi[Im, J]) / dx)
        for (a, b), (c, e) in zip(geo["fri"], geo["frj"]):
            I, J, Jm = slice(a, b + 1), slice(c, e + 1), slice(c - 1, e)
            mst = (mu_perp[I, J] + mu_perp[I, Jm]) / 2.0 * 1.0
            rho_t = (rhoe[I, J] + rhoe[I, Jm]) / 2.0
            nUer[I, J] = nUer[I, J] + mst * rho_t * ((dphi[I, J] - dphi[I, Jm]) / dr)
        fe = prm["flag_error"]
        errs = (calc_res(phi, phi_t, geo["ib"], geo["jb"], 1e-100, fe),
                calc_res(nUex, nUex_t, geo["fxi"], geo["fxj"], 1e-100, fe),
                calc_res(nUer, nUer_t, geo["fri"], geo["frj"], 1e-100, fe))
        if max(errs) < prm["error_cnv_HES_phi"] or ncount >= prm["maxITR_HES_phi"]:
            break
    fe = prm["flag_error"]
    out = dict(phi=phi, Ex=Ex, Er=Er, nUex=nUex, nUer=nUer, ncount=ncount, errors_last=errs)
    out["error_phi"] = calc_res(phi, phi_old, geo["ib"], geo["jb"], 1e-100, fe)
    out["error_nUex"] = calc_res(nUex, nUex_old, geo["fxi"], geo["fxj"], 1e-100, fe)
    out["error_nUer"] = calc_res(nUer, nUer_old, geo["fri"], geo["frj"], 1e-100, fe)
    return out


# ----------------------------------------------------------------------------
# Scharfetter-Gummel predictor-correctors of the electron density and energy
# ----------------------------------------------------------------------------

LIM_EXP = 1.0e2  # fluidModule.hpp:3099
EPS_VD = 1.0e-3  # fluidModule.hpp:3100


def _sg(vd, z):
    """Upwind / downwind weights vd/(1-e^-z), vd/(e^z-1) with the exponent clipped at 100."""
    return vd / (1.0 - _exp(np.fmin(-z, LIM_EXP))), vd / (_exp(np.fmin(z, LIM_EXP)) - 1.0)


def _sg_face_x(Te, Ex, mu_perp, I, J, dx):
    mst = (mu_perp[I, J] + mu_perp[I - 1, J]) / 2.0 * 1.0
    Tt = (Te[I, J] + Te[I - 1, J]) / 2.0
    dT = (Te[I, J] - Te[I - 1, J]) / dx
    vd = mst * (-Ex[I, J] - BOLTZ / E0 * dT) + EPS_VD
    D = BOLTZ * Tt / E0 * mst
    return mst, vd, vd * dx / D


def _sg_face_r(Te, Er, mu_perp, I, J, dr):
    mst = (mu_perp[I, J] + mu_perp[I, J - 1]) / 2.0 * 1.0
    Tt = (Te[I, J] + Te[I, J - 1]) / 2.0
    dT = (Te[I, J] - Te[I, J - 1]) / dr
    vd = mst * (-Er[I, J] - BOLTZ / E0 * dT) + EPS_VD
    D = BOLTZ * Tt / E0 * mst
    return mst, vd, vd * dr / D


def _masks(geo):
    fl = geo["flags"].astype(np.int64)
    return dict(bLx=(fl & F_BLX) != 0, bRx=(fl & F_BRX) != 0, bLrw=(fl & F_BLR_WALL) != 0,
                bLr=((fl & F_BLR_WALL) != 0) & ((fl & F_BLR_CEN) != 0), bRrw=(fl & F_BRR_WALL) != 0,
                bRr=((fl & F_BRR_WALL) != 0) & ((fl & F_BRR_OPEN) != 0))


def _energy_wall(Te_old, Te, E, rhoeps, rhoeps_old, rhoe_old, rhoi, Ui, rhoUm, h, sign, prm, see):
    """Electron energy flux through a wall face (fluidModule.hpp:4175-4190)."""
    vth = np.sqrt(8.0 * BOLTZ * Te_old / (np.pi * prm["masse"]))
    delta_phi = np.fmax(sign * E * h / 2.0, 0.0)
    ex = _exp(np.fmin(-E0 * delta_phi / (BOLTZ * Te_old + 1e-100), LIM_EXP))
    gpn_eps = sign * vth * ex / 3.0 * 1.0
    eps_emit = 2.0 * E0 * prm["Te_emitSEE_eV"]
    gpn = sign * 0.25 * 1.0 * vth * ex
    eb, rd, ts, dTe_SEE = see
    ceb, crd, cts = func_Te(eb, Te, dTe_SEE), func_Te(rd, Te, dTe_SEE), func_Te(ts, Te, dTe_SEE)
    see_flux = (-eps_emit * prm["coefIISEE_ts"] * rhoi * Ui - (ceb + prm["ratioEngy_EISEE_rd"] * crd) * rhoeps_old * gpn_eps
                - eps_emit * cts * rhoe_old * gpn - eps_emit * prm["coefMISEE_ts"] * rhoUm)
    return rhoeps * gpn_eps + see_flux


def _apply_ghosts(a, geo, which):
    for i0, i1, j0, j1, di, dj, mode in geo["ghosts"]:
        I, J = slice(i0, i1 + 1), slice(j0, j1 + 1)
        It, Jt = slice(i0 + di, i1 + di + 1), slice(j0 + dj, j1 + dj + 1)
        if which == "rhoe" and mode == 0:
            a[It, Jt] = 0.0
        else:
            a[It, Jt] = a[I, J]


def solve_sg_pc(st: dict, prm: dict, geo: dict, see, solve, species: str) -> dict:
    """FluidModule::solve_rhoe_wdTe_wSEE_PC (species "rhoe", fluidModule.hpp:3082-3970)
    and solve_Te_wdTe_wSEE_PC (species "rhoeps", fluidModule.hpp:4006-4957).

    rhoe: st holds rhoe, rhoUex, rhoUer, rhoUex_wall, rhoUer_wall, Te, mu_para,
    mu_perp, mu_rr, mu_xr, mu_xx, Ex, Er, rhoi, Uix, Uir, rhoUmx, rhoUmr,
    rate_ionize, rhoUix_wall.  rhoeps: rhoeps, Gx, Gr, Gx_wall, Gr_wall, Te, rhoe,
    rhoe_old, rhoUex, rhoUer, Pabs, rate_eloss and the same mobility, field, ion
    and metastable arrays.  prm: dt, dx, dr, rmin, masse, coefIISEE_ts,
    coefMISEE_ts, Te_emitSEE_eV, ratioEngy_EISEE_rd, maxITR_HES, error_cnv_HES,
    flag_error.  Returns the updated arrays with the calcRes errors and, for rhoe,
    the anode currents Ii_Anode, Ie_Anode, I_Anode."""
    en = species == "rhoeps"
    nk, fxk, frk = ("rhoeps", "Gx", "Gr") if en else ("rhoe", "rhoUex", "rhoUer")
    fac = 5.0 / 3.0 if en else 1.0
    ni, nj = geo["ni"], geo["nj"]
    dx, dr, dt = prm["dx"], prm["dr"], prm["dt"]
    r = prm["rmin"] + (np.arange(nj + 2) - 0.5) * dr
    m = _masks(geo)
    g = dict(st)
    n = st[nk].copy()
    Fx, Fr = st[fxk].copy(), st[frk].copy()
    Fx_w, Fr_w = st[fxk + "_wall"].copy(), st[frk + "_wall"].copy()
    Te = st["Te"].copy()
    Te_old = Te.copy()
    n_old, Fx_old, Fr_old = n.copy(), Fx.copy(), Fr.copy()
    Tsg = Te_old if en else Te            # temperature of the SG weights
    rhoe_old = g["rhoe_old"] if en else n_old
    d = n - n_old
    mu_para, mu_perp, Ex, Er = g["mu_para"], g["mu_perp"], g["Ex"], g["Er"]
    ncount = 0
    while True:
        ncount += 1
        n_t, Fx_t, Fr_t = n.copy(), Fx.copy(), Fr.copy()
        for (a, b), (c, e) in zip(geo["fxi"], geo["fxj"]):
            I = np.arange(a, b + 1)[:, None]
            J = np.arange(c, e + 1)[None, :]
            rL = (r[J] + r[J - 1]) / 2.0
            rR = (r[J] + r[J + 1]) / 2.0
            mpa = (mu_para[I, J] + mu_para[I - 1, J]) / 2.0
            mpe = (mu_perp[I, J] + mu_perp[I - 1, J]) / 2.0
            mrr = (g["mu_rr"][I, J] + g["mu_rr"][I - 1, J]) / 2.0
            mxr = (g["mu_xr"][I, J] + g["mu_xr"][I - 1, J]) / 2.0
            ixx = mrr / (mpa * mpe)
            ixr = -mxr / (mpa * mpe)
            mst, vd, z = _sg_face_x(Tsg, Ex, mu_perp, I, J, dx)
            A, B = _sg(vd, z)
            Fr_i = (rR * Fr_t[I, J + 1] * m["bRrw"][I, J] + rL * Fr_t[I, J] * m["bLr"][I, J]
                    + rR * Fr_t[I - 1, J + 1] * m["bRrw"][I - 1, J] + rL * Fr_t[I - 1, J] * m["bLr"][I - 1, J]) / (4.0 * r[J])
            if en:
                Fx[I, J] = ((A * n[I - 1, J] - B * n[I, J]) * 5.0 / 3.0 + Fx_t[I, J]
                            - mst * (ixx * Fx_t[I, J] + ixr * Fr_i))
            else:
                Fx[I, J] = (A * n[I - 1, J] - B * n[I, J] + Fx_t[I, J] - mst * (ixx * Fx_t[I, J] + ixr * Fr_i))
        for kind, i0, i1, j0, j1 in geo["segs"]:
            J = np.arange(j0, j1 + 1)
            if kind not in ("L", "R", "RB"):
                continue
            c, f, sg = (i0, i0, -1.0) if kind == "L" else (i0, i0 + 1, 1.0)
            if en:
                v = _energy_wall(Te_old[c, J], Te[c, J], Ex[f, J], n[c, J], n_old[c, J], rhoe_old[c, J], g["rhoi"][c, J],
                                 g["Uix"][f, J], g["rhoUmx"][f, J], dx, sg, prm, see)
            else:
                v = _wall_flux(Te[c, J], n[c, J], n_old[c, J], g["rhoi"][c, J], g["Uix"][f, J], g["rhoUmx"][f, J],
                               Ex[f, J], dx, sg, prm, see)
            Fx[f, J] = v
            Fx_w[f, J] = v
        for (a, b), (c, e) in zip(geo["fri"], geo["frj"]):
            I = np.arange(a, b + 1)[:, None]
            J = np.arange(c, e + 1)[None, :]
            r_t = (r[J] + r[J - 1]) / 2.0
            mpa = (mu_para[I, J] + mu_para[I, J - 1]) / 2.0
            mpe = (mu_perp[I, J] + mu_perp[I, J - 1]) / 2.0
            mxx = (g["mu_xx"][I, J] + g["mu_xx"][I, J - 1]) / 2.0
            mxr = (g["mu_xr"][I, J] + g["mu_xr"][I, J - 1]) / 2.0
            irr = mxx / (mpa * mpe)
            ixr = -mxr / (mpa * mpe)
            mst, vd, z = _sg_face_r(Tsg, Er, mu_perp, I, J, dr)
            A, B = _sg(vd, z)
            Fx_i = (r[J] * Fx_t[I + 1, J] * m["bRx"][I, J] + r[J] * Fx_t[I, J] * m["bLx"][I, J]
                    + r[J - 1] * Fx_t[I + 1, J - 1] * m["bRx"][I, J - 1] + r[J - 1] * Fx_t[I, J - 1] * m["bLx"][I, J - 1]) / (4.0 * r_t)
            if en:
                Fr[I, J] = ((A * n[I, J - 1] - B * n[I, J]) * 5.0 / 3.0 + Fr_t[I, J]
                            - mst * (ixr * Fx_i + irr * Fr_t[I, J]))
            else:
                Fr[I, J] = (A * n[I, J - 1] - B * n[I, J] + Fr_t[I, J] - mst * (ixr * Fx_i + irr * Fr_t[I, J]))
        for kind, i0, i1, j0, j1 in geo["segs"]:
            I = np.arange(i0, i1 + 1)
            if kind in ("D", "U"):
                c, f, sg = (j0, j0, -1.0) if kind == "D" else (j0, j0 + 1, 1.0)
                if en:
                    v = _energy_wall(Te_old[I, c], Te[I, c], Er[I, f], n[I, c], n_old[I, c], rhoe_old[I, c],
                                     g["rhoi"][I, c], g["Uir"][I, f], g["rhoUmr"][I, f], dr, sg, prm, see)
                else:
                    v = _wall_flux(Te[I, c], n[I, c], n_old[I, c], g["rhoi"][I, c], g["Uir"][I, f], g["rhoUmr"][I, f],
                                   Er[I, f], dr, sg, prm, see)
                Fr[I, f] = v
                rec = np.ones(I.size, bool)
                if en:
                    for (a, b, c0, c1) in geo.get("energy_keep_walls", ()):
                        if c0 <= f <= c1:
                            rec &= ~((I >= a) & (I <= b))
                Fr_w[I[rec], f] = v[rec]
            elif kind == "O":
                if en:
                    Fr[I, j0 + 1] = 5.0 / 2.0 * BOLTZ * Te_old[I, j0] * np.fmax(g["rhoUer"][I, j0 + 1], 0.0)
                else:
                    Fr[I, j0 + 1] = g["rhoi"][I, j0] * g["Uir"][I, j0 + 1]
                Fr_w[I, j0 + 1] = 0.0
        sh = (ni + 2, nj + 2)
        aP, aE, aW, aN, aS, bb = (np.zeros(sh) for _ in range(6))
        for (a, b), (c, e) in zip(geo["ib"], geo["jb"]):
            I = np.arange(a, b + 1)[:, None]
            J = np.arange(c, e + 1)[None, :]
            rR = (r[J] + r[J + 1]) / 2.0
            rL = (r[J] + r[J - 1]) / 2.0
            qR = (r[J] + r[J + 1]) / 2.0 / r[J]
            qL = (r[J] + r[J - 1]) / 2.0 / r[J]
            _, vLx, zLx = _sg_face_x(Tsg, Ex, mu_perp, I, J, dx)
            _, vRx, zRx = _sg_face_x(Tsg, Ex, mu_perp, I + 1, J, dx)
            _, vLr, zLr = _sg_face_r(Tsg, Er, mu_perp, I, J, dr)
            _, vRr, zRr = _sg_face_r(Tsg, Er, mu_perp, I, J + 1, dr)
            bLx, bRx, bLr, bRr = m["bLx"][I, J], m["bRx"][I, J], m["bLr"][I, J], m["bRr"][I, J]
            ex = _exp
            tterm = 3.0 / 5.0 * dx * dr / dt if en else dx * dr / dt
            aP[I, J] = (vRx / (1.0 - ex(np.fmin(-zRx, LIM_EXP))) * bRx * dr
                        + vLx / (ex(np.fmin(zLx, LIM_EXP)) - 1.0) * bLx * dr
                        + qR * vRr / (1.0 - ex(np.fmin(-zRr, LIM_EXP))) * bRr * dx
                        + qL * vLr / (ex(np.fmin(zLr, LIM_EXP)) - 1.0) * bLr * dx + tterm)
            aE[I, J] = vRx / (ex(np.fmin(zRx, LIM_EXP)) - 1.0) * bRx * dr
            aW[I, J] = vLx / (1.0 - ex(np.fmin(-zLx, LIM_EXP))) * bLx * dr
            aN[I, J] = qR * vRr / (ex(np.fmin(zRr, LIM_EXP)) - 1.0) * bRr * dx
            aS[I, J] = qL * vLr / (1.0 - ex(np.fmin(-zLr, LIM_EXP))) * bLr * dx
            div = (Fx[I + 1, J] - Fx[I, J]) / dx + (qR * Fr[I, J + 1] - qL * Fr[I, J]) / dr
            if en:
                bLxw, bRxw, bLrw, bRrw = m["bLx"][I, J], m["bRx"][I, J], m["bLrw"][I, J], m["bRrw"][I, J]
                jx = -E0 * (g["rhoUex"][I + 1, J] * Ex[I + 1, J] * bRxw + g["rhoUex"][I, J] * Ex[I, J] * bLxw) / 2.0
                jr = -E0 * (rR * g["rhoUer"][I, J + 1] * Er[I, J + 1] * bRrw + rL * g["rhoUer"][I, J] * Er[I, J] * bLrw) / (2.0 * r[J])
                R1 = (-n[I, J] + n_old[I, J]) / dt
                R3 = g["Pabs"][I, J] - g["rhoe"][I, J] * g["rate_eloss"][I, J]
                bb[I, J] = 3.0 / 5.0 * (R1 + (jx + jr) + R3 + (-div)) * dx * dr
            else:
                bb[I, J] = (-div + g["rate_ionize"][I, J] - (n[I, J] - n_old[I, J]) / dt) * dx * dr
        x = solve(aP, aE, aW, aN, aS, bb, geo["ib"], geo["jb"])
        for (a, b), (c, e) in zip(geo["ib"], geo["jb"]):
            d[a:b + 1, c:e + 1] = x[a:b + 1, c:e + 1]
        for (a, b), (c, e) in zip(geo["fxi"], geo["fxj"]):
            I = np.arange(a, b + 1)[:, None]
            J = np.arange(c, e + 1)[None, :]
            _, vd, z = _sg_face_x(Tsg, Ex, mu_perp, I, J, dx)
            A, B = _sg(vd, z)
            Fx[I, J] = Fx[I, J] + ((A * d[I - 1, J] - B * d[I, J]) * 5.0 / 3.0 if en else A * d[I - 1, J] - B * d[I, J])
        for (a, b), (c, e) in zip(geo["fri"], geo["frj"]):
            I = np.arange(a, b + 1)[:, None]
            J = np.arange(c, e + 1)[None, :]
            _, vd, z = _sg_face_r(Tsg, Er, mu_perp, I, J, dr)
            A, B = _sg(vd, z)
            Fr[I, J] = Fr[I, J] + ((A * d[I, J - 1] - B * d[I, J]) * 5.0 / 3.0 if en else A * d[I, J - 1] - B * d[I, J])
        for (a, b), (c, e) in zip(geo["ib"], geo["jb"]):
            sl = (slice(a, b + 1), slice(c, e + 1))
            nn = n[sl] + d[sl]
            n[sl] = np.where(nn > 0.0, nn, n[sl])
        fe = prm["flag_error"]
        errs = (calc_res(n, n_t, geo["ib"], geo["jb"], 1e-100, fe),
                calc_res(Fx, Fx_t, geo["fxi"], geo["fxj"], 1e-100, fe),
                calc_res(Fr, Fr_t, geo["fri"], geo["frj"], 1e-100, fe))
        if max(errs) < prm["error_cnv_HES"] or ncount >= prm["maxITR_HES"]:
            break
    out = {nk: n, fxk: Fx, frk: Fr, fxk + "_wall": Fx_w, frk + "_wall": Fr_w, "ncount": ncount,
           "errors_last": errs}
    if en:
        for (a, b), (c, e) in zip(geo["ib"], geo["jb"]):
            sl = (slice(a, b + 1), slice(c, e + 1))
            n[sl] = np.where(n[sl] < 0.0, np.fmax(n_old[sl], 0.0), n[sl])
        blk = geo["flags"] != 0
        rhoe = g["rhoe"]
        rmax = rhoe[blk].max() if blk.any() else 0.0
        Te_max = 1000.0 * E0 / BOLTZ
        Te = Te.copy()
        for (a, b), (c, e) in zip(geo["ib"], geo["jb"]):
            sl = (slice(a, b + 1), slice(c, e + 1))
            Te[sl] = np.fmin(n[sl] / (3.0 / 2.0 * (rhoe[sl] + rmax * 0.001) * BOLTZ + 1e-100), Te_max)
        _apply_ghosts(Te, geo, "Te")
        out["Te"] = Te
        out["Te_old"] = Te_old
    else:
        _apply_ghosts(n, geo, "rhoe")
        Ii = Ie = 0.0
        for kind, i0, i1, j0, j1 in geo["segs"]:
            if kind != "RB":
                continue
            for j in range(j0, j1 + 1):
                di = g["rhoUix_wall"][i0 + 1, j] * 2.0 * np.pi * r[j] * dr * E0
                de = Fx_w[i0 + 1, j] * 2.0 * np.pi * r[j] * dr * (-E0)
                Ii += di
                Ie += de
        out.update(Ii_Anode=Ii, Ie_Anode=Ie, I_Anode=Ii + Ie, rhoe_old=n_old)
    fe = prm["flag_error"]
    out["error_" + nk] = calc_res(n, n_old, geo["ib"], geo["jb"], 1e-100, fe)
    out["error_" + fxk] = calc_res(Fx, Fx_old, geo["fxi"], geo["fxj"], 1e-100, fe)
    out["error_" + frk] = calc_res(Fr, Fr_old, geo["fri"], geo["frj"], 1e-100, fe)
    return out


def check_cfl(f: dict, prm: dict) -> dict:
    """FluidModule::check_CFL (fluidModule.hpp:57-115)."""
    rhoe, Te = f["rhoe"], f["Te"]
    ni, nj = rhoe.shape[0] - 2, rhoe.shape[1] - 2
    r = prm["rmin"] + (np.arange(nj + 2) - 0.5) * prm["dr"]
    rhoe_max = max(0.0, rhoe.max())
    mu_max = max(0.0, f["mu_para"].max())
    Te_max = max(0.0, Te.max())
    I, J = slice(1, ni + 1), slice(1, nj + 1)
    rL = (r[1:nj + 1] + r[0:nj]) / 2.0
    rR = (r[1:nj + 1] + r[2:nj + 2]) / 2.0
    ux = (f["rhoUex"][2:ni + 2, J] + f["rhoUex"][I, J]) / 2.0 / (rhoe[I, J] + 1e-100)
    ur = (rR * f["rhoUer"][I, 2:nj + 2] + rL * f["rhoUer"][I, J]) / (2.0 * r[J]) / (rhoe[I, J] + 1e-100)
    ue_max = max(0.0, np.sqrt(ux * ux + ur * ur).max()) + np.sqrt(8.0 * BOLTZ * Te_max / (np.pi * prm["masse"]))
    dt_min = EPS0 / (E0 * rhoe_max * mu_max)
    out = dict(rhoe_max=rhoe_max, mu_max=mu_max, Te_max=Te_max, ue_max=ue_max, dt_min=dt_min)
    if prm.get("flag_adp_dt", 0) == 1:
        out.update(dt=dt_min * prm["CFL"], CFL=prm["CFL"])
    else:
        out.update(dt=prm["dt"], CFL=prm["dt"] / dt_min)
    return out


# ----------------------------------------------------------------------------
# ion step: momentum (Uix, Uir, Uip), continuity and velocity correction
# ----------------------------------------------------------------------------

def ion_segments(geo: dict) -> dict:
    """Wall segments of the ion sweeps on the cell ('c'), x-face ('x') and r-face
    ('r') index spaces, named as in the reference (z0..z5 axial walls, x0..x5 radial
    walls, x6 the axis), each (i0, i1, j0, j1) or None.  Cathode: the loop bounds of
    fluidModule.hpp:218-360 (x faces), :700-800 (r faces), :1130-1200 (cells);
    rectangle: z0 at z = 0, z5 the biased electrode, x1 the wall at r = R, x6 the axis."""
    if len(geo["ib"]) == 5:
        ib, jb, fxi, fxj, fri, frj = geo["ib"], geo["jb"], geo["fxi"], geo["fxj"], geo["fri"], geo["frj"]

        def table(I, J, axis):
            t = dict(z0=(I[0][0], I[0][0], J[0][0], J[0][1]), z1=(I[2][0], I[2][0], J[2][0], J[0][0] - 1),
                     z2=(I[3][0], I[3][0], J[3][0], J[2][0] - 1), z4=(I[4][0], I[4][0], J[1][0], J[4][1]),
                     z3=(I[1][1], I[1][1], J[1][0], J[1][1]), z5=(I[4][1], I[4][1], J[4][0], J[4][1]),
                     x0=(I[0][0], I[0][1], J[0][0], J[0][0]), x2=(I[2][0], I[2][1], J[2][0], J[2][0]),
                     x1=(I[0][0], I[1][1], J[0][1], J[0][1]), x4=(I[1][1] + 1, I[3][1], J[3][1], J[3][1]),
                     x5=(I[4][0], I[4][1], J[4][1], J[4][1]))
            t["x6"] = (I[3][0], I[4][1], J[3][0], J[3][0]) if axis else None
            return {k: tuple(int(v) for v in s) if s is not None else None for k, s in t.items()}

        return dict(c=table(ib, jb, False), x=table(fxi, fxj, False), r=table(fri, frj, True))
    ni, nj = geo["ni"], geo["nj"]
    empty = dict(z1=None, z2=None, z3=None, z4=None, x0=None, x2=None, x4=None, x5=None)
    return dict(c=dict(empty, z0=(1, 1, 1, nj), z5=(ni, ni, 1, nj), x1=(1, ni, nj, nj), x6=None),
                x=dict(empty, z0=(2, 2, 1, nj), z5=(ni, ni, 1, nj), x1=(2, ni, nj, nj), x6=None),
                r=dict(empty, z0=(1, 1, 2, nj), z5=(ni, ni, 2, nj), x1=(1, ni, nj, nj), x6=(1, ni, 2, 2)))


def _pts(s, di0=0, di1=0, dj0=0, dj1=0):
    """Points of a segment with adjusted bounds, in loop order."""
    if s is None:
        return []
    i0, i1, j0, j1 = s
    return [(i, j) for i in range(i0 + di0, i1 + di1 + 1) for j in range(j0 + dj0, j1 + dj1 + 1)]


def _ui_wall(Uold, phi_a, phi_b, sign, bias, prm):
    dphi = (phi_a + phi_b) / 2.0 - bias
    return sign * np.sqrt(Uold ** 2 + max(2.0 * E0 * dphi / prm["massi"], 0.0))


def _erf(x):
    import oracle
    return oracle.libm_erf(x)


def ion_step(st: dict, prm: dict, geo: dict, solve_c, solve_x, solve_r) -> dict:
    """The ion sub-step of the time loop (src/main.cpp:191-197): solve_Uix_tmp,
    solve_Uir_tmp, solve_Uip_tmp (fluidModule.hpp:123-1404), solve_rhoi_constTe
    (:1405-1755) and correct_Ui_constTe (:1763-2072).

    st: Uix, Uir, Uip, rhoi, phi, Ex, Er, Bx, Br, rate_ionize, nui_m, rhoUix, rhoUir,
    rhoUix_wall, rhoUir_wall.  prm: dt, ndt_i, dx, dr, rmin, rmax, massi, Ti,
    V_bias, Te_rep_eV, CFL, flag_error.  solve_c / solve_x / solve_r(aP, aE, aW, aN,
    aS, b, ib, jb) return the block solutions of the cell, x-face and r-face
    systems (zero start)."""
    ni, nj = geo["ni"], geo["nj"]
    dx, dr = prm["dx"], prm["dr"]
    dt_i = prm["dt"] * float(prm["ndt_i"])
    massi, Ti = prm["massi"], prm["Ti"]
    r = prm["rmin"] + (np.arange(nj + 2) - 0.5) * dr
    S = ion_segments(geo)
    m = _masks(geo)
    g = {k: v.copy() for k, v in st.items()}
    phi = g["phi"]
    Uix_old, Uir_old, Uip_old, rhoi_old = g["Uix"].copy(), g["Uir"].copy(), g["Uip"].copy(), g["rhoi"].copy()
    sh = (ni + 2, nj + 2)

    # --- solve_Uix_tmp (:123-594) -------------------------------------------
    aP, aE, aW, aN, aS, b = (np.zeros(sh) for _ in range(6))
    for (a0, a1), (c0, c1) in zip(geo["fxi"], geo["fxj"]):
        I = np.arange(a0, a1 + 1)[:, None]
        J = np.arange(c0, c1 + 1)[None, :]
        rL = (r[J] + r[J - 1]) / 2.0
        rR = (r[J] + r[J + 1]) / 2.0
        qL, qR = rL / r[J], rR / r[J]
        ULx = (Uix_old[I, J] + Uix_old[I - 1, J]) / 2.0
        URx = (Uix_old[I, J] + Uix_old[I + 1, J]) / 2.0
        ULr = (Uir_old[I, J] + Uir_old[I - 1, J]) / 2.0
        URr = (Uir_old[I, J + 1] + Uir_old[I - 1, J + 1]) / 2.0
        rho_t = (g["rhoi"][I, J] + g["rhoi"][I - 1, J]) / 2.0
        riz = (g["rate_ionize"][I, J] + g["rate_ionize"][I - 1, J]) / 2.0
        nui = (g["nui_m"][I, J] + g["nui_m"][I - 1, J]) / 2.0
        dndx = (g["rhoi"][I, J] - g["rhoi"][I - 1, J]) / dx
        Uip_t = (Uip_old[I, J] + Uip_old[I - 1, J]) / 2.0
        Br_t = (g["Br"][I, J] + g["Br"][I - 1, J]) / 2.0
        lor = -E0 * Uip_t * Br_t
        aE[I, J] = -(URx - np.abs(URx)) / (2.0 * dx)
        aW[I, J] = (ULx + np.abs(ULx)) / (2.0 * dx)
        aN[I, J] = -qR * (URr - np.abs(URr)) / (2.0 * dr)
        aS[I, J] = qL * (ULr + np.abs(ULr)) / (2.0 * dr)
        aP[I, J] = 1.0 / dt_i + riz / (rho_t + 1e-100) + nui + aE[I, J] + aW[I, J] + aN[I, J] + aS[I, J]
        b[I, J] = (Uix_old[I, J] / dt_i + (E0 * g["Ex"][I, J] + lor) / massi
                   - BOLTZ * Ti / (massi * rho_t + 1e-100) * dndx)
    X = S["x"]
    for name, sign, coef, bias in (("z0", -1, aW, 0), ("z1", -1, aW, 0), ("z2", -1, aW, 0), ("z4", -1, aW, 0),
                                   ("z3", 1, aE, 0), ("z5", 1, aE, 1)):
        for i, j in _pts(X[name]):
            Uw = _ui_wall(Uix_old[i, j], phi[i, j], phi[i - 1, j], sign, prm["V_bias"] * bias, prm)
            b[i, j] = b[i, j] + coef[i, j] * Uw
            coef[i, j] = 0.0
    for name, coef in (("x0", aS), ("x2", aS), ("x1", aN), ("x4", aN), ("x5", aN)):
        for i, j in _pts(X[name]):
            coef[i, j] = 0.0
    x = solve_x(aP, aE, aW, aN, aS, b, geo["fxi"], geo["fxj"])
    for (a0, a1), (c0, c1) in zip(geo["fxi"], geo["fxj"]):
        g["Uix"][a0:a1 + 1, c0:c1 + 1] = x[a0:a1 + 1, c0:c1 + 1]
    for name, sign, di, bias in (("z0", -1, -1, 0), ("z1", -1, -1, 0), ("z2", -1, -1, 0), ("z4", -1, -1, 0),
                                 ("z3", 1, 1, 0), ("z5", 1, 1, 1)):
        for i, j in _pts(X[name]):
            g["Uix"][i + di, j] = _ui_wall(Uix_old[i, j], phi[i, j], phi[i - 1, j], sign, prm["V_bias"] * bias, prm)
    for i, j in _pts(X["x0"], di1=-1):
        g["Uix"][i, j - 1] = 0.0
    for i, j in _pts(X["x2"], di1=-1):
        g["Uix"][i, j - 1] = 0.0
    for i, j in _pts(X["x1"]):
        g["Uix"][i, j - 1] = 0.0          # the reference writes the row below the top row here
    for i, j in _pts(X["x4"], di0=1, di1=-1):
        g["Uix"][i, j + 1] = 0.0
    for i, j in _pts(X["x5"]):
        g["Uix"][i, j + 1] = 0.0

    # --- solve_Uir_tmp (:601-1053) ------------------------------------------
    aP, aE, aW, aN, aS, b = (np.zeros(sh) for _ in range(6))
    for (a0, a1), (c0, c1) in zip(geo["fri"], geo["frj"]):
        I = np.arange(a0, a1 + 1)[:, None]
        J = np.arange(c0, c1 + 1)[None, :]
        r_t = (r[J] + r[J - 1]) / 2.0
        rL = (r[J - 1] + r[J - 2]) / 2.0
        rR = (r[J + 1] + r[J]) / 2.0
        ULx = (r[J] * Uix_old[I, J] + r[J - 1] * Uix_old[I, J - 1]) / (2.0 * r_t)
        URx = (r[J] * Uix_old[I + 1, J] + r[J - 1] * Uix_old[I + 1, J - 1]) / (2.0 * r_t)
        ULr = (r_t * Uir_old[I, J] + rL * Uir_old[I, J - 1]) / (2.0 * r[J - 1])
        URr = (r_t * Uir_old[I, J] + rR * Uir_old[I, J + 1]) / (2.0 * r[J])
        rho_t = (g["rhoi"][I, J] + g["rhoi"][I, J - 1]) / 2.0
        riz = (g["rate_ionize"][I, J] + g["rate_ionize"][I, J - 1]) / 2.0
        nui = (g["nui_m"][I, J] + g["nui_m"][I, J - 1]) / 2.0
        dndr = (g["rhoi"][I, J] - g["rhoi"][I, J - 1]) / dr
        Bx_t = (r[J] * g["Bx"][I, J] + r[J - 1] * g["Bx"][I, J - 1]) / (2.0 * r_t)
        Uip_t = (r[J] * Uip_old[I, J] + r[J - 1] * Uip_old[I, J - 1]) / (2.0 * r_t)
        lor = E0 * Uip_t * Bx_t
        cen = -Uip_t * Uip_t / r_t
        aE[I, J] = -(URx - np.abs(URx)) / (2.0 * dx)
        aW[I, J] = (ULx + np.abs(ULx)) / (2.0 * dx)
        aN[I, J] = -r[J] / r_t * (URr - np.abs(URr)) / (2.0 * dr)
        aS[I, J] = r[J - 1] / r_t * (ULr + np.abs(ULr)) / (2.0 * dr)
        aP[I, J] = 1.0 / dt_i + riz / (rho_t + 1e-100) + nui + aE[I, J] + aW[I, J] + aN[I, J] + aS[I, J]
        b[I, J] = (Uir_old[I, J] / dt_i + (E0 * g["Er"][I, J] + lor) / massi
                   - BOLTZ * Ti / (massi * rho_t + 1e-100) * dndr + cen)
    R = S["r"]
    for name, coef in (("z0", aW), ("z1", aW), ("z2", aW), ("z4", aW), ("z3", aE), ("z5", aE)):
        for i, j in _pts(R[name]):
            coef[i, j] = 0.0
    for name, sign, coef in (("x0", -1, aS), ("x2", -1, aS)):
        for i, j in _pts(R[name]):
            Uw = _ui_wall(Uir_old[i, j], phi[i, j], phi[i, j - 1], sign, 0.0, prm)
            b[i, j] = b[i, j] + coef[i, j] * Uw
            coef[i, j] = 0.0
    for i, j in _pts(R["x6"]):
        aS[i, j] = 0.0
    for name in ("x1", "x4"):
        for i, j in _pts(R[name]):
            Uw = _ui_wall(Uir_old[i, j], phi[i, j], phi[i, j - 1], 1, 0.0, prm)
            b[i, j] = b[i, j] + aN[i, j] * Uw
            aN[i, j] = 0.0
    for i, j in _pts(R["x5"]):
        r_t = (r[j] + r[j - 1]) / 2.0
        rR = (r[j + 1] + r[j]) / 2.0
        b[i, j] = b[i, j] + aN[i, j] * r_t / rR * max(Uir_old[i, j], 0.0)
        aN[i, j] = 0.0
    x = solve_r(aP, aE, aW, aN, aS, b, geo["fri"], geo["frj"])
    for (a0, a1), (c0, c1) in zip(geo["fri"], geo["frj"]):
        g["Uir"][a0:a1 + 1, c0:c1 + 1] = x[a0:a1 + 1, c0:c1 + 1]
    for name, di, adj in (("z0", -1, (0, 0)), ("z1", -1, (0, -1)), ("z2", -1, (0, -1)), ("z4", -1, (1, 0)),
                          ("z3", 1, (1, 0)), ("z5", 1, (0, 0))):
        for i, j in _pts(R[name], dj0=adj[0], dj1=adj[1]):
            g["Uir"][i + di, j] = 0.0
    for name in ("x0", "x2"):
        for i, j in _pts(R[name]):
            g["Uir"][i, j - 1] = _ui_wall(Uir_old[i, j], phi[i, j], phi[i, j - 1], -1, 0.0, prm)
    for i, j in _pts(R["x6"]):
        g["Uir"][i, j - 1] = 0.0
    for name in ("x1", "x4"):
        for i, j in _pts(R[name]):
            g["Uir"][i, j + 1] = _ui_wall(Uir_old[i, j], phi[i, j], phi[i, j - 1], 1, 0.0, prm)
    for i, j in _pts(R["x5"]):
        r_t = (r[j] + r[j - 1]) / 2.0
        rR = (r[j + 1] + r[j]) / 2.0
        g["Uir"][i, j + 1] = r_t / rR * max(Uir_old[i, j], 0.0)

    # --- solve_Uip_tmp (:1054-1404) -----------------------------------------
    aP, aE, aW, aN, aS, b = (np.zeros(sh) for _ in range(6))
    for (a0, a1), (c0, c1) in zip(geo["ib"], geo["jb"]):
        I = np.arange(a0, a1 + 1)[:, None]
        J = np.arange(c0, c1 + 1)[None, :]
        rL = (r[J] + r[J - 1]) / 2.0
        rR = (r[J] + r[J + 1]) / 2.0
        qL, qR = rL / r[J], rR / r[J]
        ULx, URx = Uix_old[I, J], Uix_old[I + 1, J]
        ULr, URr = Uir_old[I, J], Uir_old[I, J + 1]
        Ux_t = (Uix_old[I + 1, J] + Uix_old[I, J]) / 2.0
        Ur_t = (rL * Uir_old[I, J] + rR * Uir_old[I, J + 1]) / (2.0 * r[J])
        lor = E0 * (Ux_t * g["Br"][I, J] - Ur_t * g["Bx"][I, J])
        cen = g["Uip"][I, J] * Ur_t / r[J]
        aE[I, J] = -(URx - np.abs(URx)) / (2.0 * dx)
        aW[I, J] = (ULx + np.abs(ULx)) / (2.0 * dx)
        aN[I, J] = -qR * (URr - np.abs(URr)) / (2.0 * dr)
        aS[I, J] = qL * (ULr + np.abs(ULr)) / (2.0 * dr)
        aP[I, J] = (1.0 / dt_i + g["rate_ionize"][I, J] / (g["rhoi"][I, J] + 1e-100) + g["nui_m"][I, J]
                    + aE[I, J] + aW[I, J] + aN[I, J] + aS[I, J])
        b[I, J] = Uip_old[I, J] / dt_i + lor / massi + cen
    C = S["c"]
    for name, coef in (("z0", aW), ("z1", aW), ("z2", aW), ("z4", aW), ("z3", aE), ("z5", aE)):
        for i, j in _pts(C[name]):
            aP[i, j] = aP[i, j] - coef[i, j]
            coef[i, j] = 0.0
    for name in ("x0", "x2"):
        for i, j in _pts(C[name]):
            aP[i, j] = aP[i, j] - aS[i, j] * r[j] / r[j - 1]
            aS[i, j] = 0.0
    for name in ("x1", "x4", "x5"):
        for i, j in _pts(C[name]):
            aP[i, j] = aP[i, j] - aN[i, j] * r[j] / r[j + 1]
            aN[i, j] = 0.0
    x = solve_c(aP, aE, aW, aN, aS, b, geo["ib"], geo["jb"])
    for (a0, a1), (c0, c1) in zip(geo["ib"], geo["jb"]):
        g["Uip"][a0:a1 + 1, c0:c1 + 1] = x[a0:a1 + 1, c0:c1 + 1]
    for name, di in (("z0", -1), ("z1", -1), ("z2", -1), ("z4", -1), ("z3", 1), ("z5", 1)):
        for i, j in _pts(C[name]):
            g["Uip"][i + di, j] = g["Uip"][i, j]
    for name in ("x0", "x2"):
        for i, j in _pts(C[name]):
            g["Uip"][i, j - 1] = r[j] / r[j - 1] * g["Uip"][i, j]
    for name in ("x1", "x4", "x5"):
        for i, j in _pts(C[name]):
            g["Uip"][i, j + 1] = r[j] / r[j + 1] * g["Uip"][i, j]

    # --- solve_rhoi_constTe (:1405-1755) ------------------------------------
    Uix, Uir = g["Uix"], g["Uir"]
    Te_rep = prm["Te_rep_eV"] * E0 / BOLTZ
    nu_star = 1.0 / prm["rmax"] * np.sqrt(BOLTZ * Te_rep / massi)
    vth = np.sqrt(8.0 * BOLTZ * Ti / (np.pi * massi))
    um = np.sqrt(2.0 * BOLTZ * Ti / massi)
    sq = np.sqrt(np.pi)
    aP, aE, aW, aN, aS, b = (np.zeros(sh) for _ in range(6))
    nui_m = g["nui_m"]
    for (a0, a1), (c0, c1) in zip(geo["ib"], geo["jb"]):
        I = np.arange(a0, a1 + 1)[:, None]
        J = np.arange(c0, c1 + 1)[None, :]
        rL = (r[J] + r[J - 1]) / 2.0
        rR = (r[J] + r[J + 1]) / 2.0
        qL, qR = rL / r[J], rR / r[J]
        ULx, URx, ULr, URr = Uix[I, J], Uix[I + 1, J], Uir[I, J], Uir[I, J + 1]
        D = lambda nu: BOLTZ * (Ti + Te_rep) / (massi * (nu + nu_star) + 1e-100)
        DLx = D((nui_m[I, J] + nui_m[I - 1, J]) / 2.0)
        DRx = D((nui_m[I, J] + nui_m[I + 1, J]) / 2.0)
        DLr = D((nui_m[I, J] + nui_m[I, J - 1]) / 2.0)
        DRr = D((nui_m[I, J] + nui_m[I, J + 1]) / 2.0)
        bLx, bRx, bLr, bRr = m["bLx"][I, J], m["bRx"][I, J], m["bLr"][I, J], m["bRrw"][I, J]
        bLrw = m["bLrw"][I, J]
        utx = ULx / (um + 1e-100)
        GLx = np.where(bLx, 0.0, -0.25 * vth * (_exp(-utx * utx) + utx * sq * (_erf(utx) - 1.0)))
        utx = URx / (um + 1e-100)
        GRx = np.where(bRx, 0.0, 0.25 * vth * (_exp(-utx * utx) + utx * sq * (_erf(utx) + 1.0)))
        utr = ULr / (um + 1e-100)
        GLr = np.where(bLrw, 0.0, -0.25 * vth * (_exp(-utr * utr) + utr * sq * (_erf(utr) - 1.0)))
        utr = URr / (um + 1e-100)
        GRr = np.where(bRr, 0.0, 0.25 * vth * (_exp(-utr * utr) + utr * sq * (_erf(utr) + 1.0)))
        aP[I, J] = ((URx + np.abs(URx)) / (2.0 * dx) * bRx - (ULx - np.abs(ULx)) / (2.0 * dx) * bLx
                    + qR * (URr + np.abs(URr)) / (2.0 * dr) * bRr - qL * (ULr - np.abs(ULr)) / (2.0 * dr) * bLr
                    + ((DRx * bRx + DLx * bLx) / (dx * dx) + (qR * DRr * bRr + qL * DLr * bLr) / (dr * dr))
                    - GLx / dx + GRx / dx - qL * GLr / dr + qR * GRr / dr + 1.0 / dt_i)
        aE[I, J] = (-(URx - np.abs(URx)) / (2.0 * dx) + DRx / (dx * dx)) * bRx
        aW[I, J] = ((ULx + np.abs(ULx)) / (2.0 * dx) + DLx / (dx * dx)) * bLx
        aN[I, J] = (-qR * (URr - np.abs(URr)) / (2.0 * dr) + qR * DRr / (dr * dr)) * bRr
        aS[I, J] = (qL * (ULr + np.abs(ULr)) / (2.0 * dr) + qL * DLr / (dr * dr)) * bLr
        ro = rhoi_old
        div = ((DRx * ro[I + 1, J] * bRx - (DRx * bRx + DLx * bLx) * ro[I, J] + DLx * ro[I - 1, J] * bLx) / (dx * dx)
               + (qR * DRr * ro[I, J + 1] * bRr - (qR * DRr * bRr + qL * DLr * bLr) * ro[I, J]
                  + qL * DLr * ro[I, J - 1] * bLr) / (dr * dr))
        b[I, J] = ro[I, J] / dt_i + g["rate_ionize"][I, J] - div
    for i, j in _pts(C["x5"]):
        aP[i, j] = aP[i, j] - aN[i, j]
        aN[i, j] = 0.0
    x = solve_c(aP, aE, aW, aN, aS, b, geo["ib"], geo["jb"])
    rhoi = g["rhoi"]
    for (a0, a1), (c0, c1) in zip(geo["ib"], geo["jb"]):
        rhoi[a0:a1 + 1, c0:c1 + 1] = x[a0:a1 + 1, c0:c1 + 1]

    def gpn(u, sign):
        ut = u / (um + 1e-100)
        return sign * 0.25 * vth * (_exp(-ut * ut) + ut * sq * (_erf(ut) + sign * 1.0))

    for name in ("z0", "z1", "z2", "z4"):
        for i, j in _pts(C[name]):
            g["rhoUix_wall"][i, j] = rhoi[i, j] * gpn(Uix[i, j], -1.0)
    for name in ("z3", "z5"):
        for i, j in _pts(C[name]):
            g["rhoUix_wall"][i + 1, j] = rhoi[i, j] * gpn(Uix[i + 1, j], 1.0)
    for name in ("x0", "x2"):
        for i, j in _pts(C[name]):
            g["rhoUir_wall"][i, j] = rhoi[i, j] * gpn(Uir[i, j], -1.0)
    for name in ("x1", "x4"):
        for i, j in _pts(C[name]):
            g["rhoUir_wall"][i, j + 1] = rhoi[i, j] * gpn(Uir[i, j + 1], 1.0)
    for i, j in _pts(C["x5"]):
        g["rhoUir"][i, j + 1] = rhoi[i, j] * Uir[i, j + 1]
        g["rhoUir_wall"][i, j + 1] = 0.0
    for (a0, a1), (c0, c1) in zip(geo["ib"], geo["jb"]):
        sl = (slice(a0, a1 + 1), slice(c0, c1 + 1))
        rhoi[sl] = np.where(rhoi[sl] < 0.0, np.fmax(rhoi_old[sl], 0.0), rhoi[sl])
    for i, j in _pts(C["x5"]):
        rhoi[i, j + 1] = rhoi[i, j]

    # --- correct_Ui_constTe (:1763-2072) -------------------------------------
    for (a0, a1), (c0, c1) in zip(geo["fxi"], geo["fxj"]):
        I = np.arange(a0, a1 + 1)[:, None]
        J = np.arange(c0, c1 + 1)[None, :]
        D = BOLTZ * (Ti + Te_rep) / (massi * ((nui_m[I, J] + nui_m[I - 1, J]) / 2.0 + nu_star) + 1e-100)
        rho_t = (rhoi[I, J] + rhoi[I - 1, J]) / 2.0
        dndx_old = (rhoi_old[I, J] - rhoi_old[I - 1, J]) / dx
        dndx = (rhoi[I, J] - rhoi[I - 1, J]) / dx
        U = Uix[I, J]
        flux = rhoi[I - 1, J] * (U + np.abs(U)) / 2.0 + rhoi[I, J] * (U - np.abs(U)) / 2.0
        g["rhoUix"][I, J] = flux - D * (dndx - dndx_old)
        Uix[I, J] = U - D / (rho_t + 1e-100) * (dndx - dndx_old)
    for blk, ((a0, a1), (c0, c1)) in enumerate(zip(geo["fri"], geo["frj"])):
        top = c1 + (1 if (blk == 4 or (len(geo["fri"]) == 1 and S["c"]["x5"] is not None)) else 0)
        I = np.arange(a0, a1 + 1)[:, None]
        J = np.arange(c0, top + 1)[None, :]
        D = BOLTZ * (Ti + Te_rep) / (massi * ((nui_m[I, J] + nui_m[I, J - 1]) / 2.0 + nu_star) + 1e-100)
        rho_t = (rhoi[I, J] + rhoi[I, J - 1]) / 2.0
        dndr_old = (rhoi_old[I, J] - rhoi_old[I, J - 1]) / dr
        dndr = (rhoi[I, J] - rhoi[I, J - 1]) / dr
        U = Uir[I, J]
        flux = rhoi[I, J - 1] * (U + np.abs(U)) / 2.0 + rhoi[I, J] * (U - np.abs(U)) / 2.0
        g["rhoUir"][I, J] = flux - D * (dndr - dndr_old)
        Uir[I, J] = U - D / (rho_t + 1e-100) * (dndr - dndr_old)
    out = {k: g[k] for k in ("Uix", "Uir", "Uip", "rhoi", "rhoUix", "rhoUir", "rhoUix_wall", "rhoUir_wall")}
    out.update(Uix_old=Uix_old, Uir_old=Uir_old, Uip_old=Uip_old, rhoi_old=rhoi_old)
    out.update(ion_errors(out, prm, geo))
    return out


def ion_boxes(geo: dict) -> dict:
    """Index boxes of the ion residuals of correct_Ui_constTe (fluidModule.hpp:1960-2070):
    rhoi and Uip over the cell blocks, Uix over the x-face blocks extended by one
    face in i, Uir over the r-face blocks without their first face in j."""
    cells = [(a, b, c, e) for (a, b), (c, e) in zip(geo["ib"], geo["jb"])]
    xs = [(a, b + 1, c, e) for (a, b), (c, e) in zip(geo["fxi"], geo["fxj"])]
    rs = [(a, b, c + 1, e) for (a, b), (c, e) in zip(geo["fri"], geo["frj"])]
    return dict(rhoi=cells, Uix=xs, Uir=rs, Uip=cells)


def ion_errors(o: dict, prm: dict, geo: dict) -> dict:
    """The ion residuals of correct_Ui_constTe (fluidModule.hpp:1960-2070)."""
    bx = ion_boxes(geo)
    CFL = prm["CFL"]
    out = {}
    for k, eps_l2 in (("rhoi", 1e10), ("Uix", 1e-6), ("Uir", 1e-6), ("Uip", 1e-6)):
        nw = np.concatenate([o[k][a:b + 1, c:e + 1].ravel() for a, b, c, e in bx[k]])
        od = np.concatenate([o[k + "_old"][a:b + 1, c:e + 1].ravel() for a, b, c, e in bx[k]])
        if prm["flag_error"] == 0:
            out["error_" + k] = float(np.abs((nw - od) / (nw + od + 1e-100) * 2.0 / CFL).max())
        else:
            out["error_" + k] = float(np.sqrt(np.sum((nw - od) ** 2 / (od ** 2 + eps_l2) / CFL) / nw.size))
    return out


# ----------------------------------------------------------------------------
# neutrals: ground-state (rhon) and metastable (rhom) diffusion
# ----------------------------------------------------------------------------

def _neutral_masks(geo, prm, i, j, blk):
    """Side flags of update_rhon / update_rhom for cell (i, j) of block blk
    (fluidModule.hpp:5021-5041, :5478-5501); the x1 wall of blocks 0-2 has a
    neutral inlet where x_i <= width_neutIn + x6."""
    fl = int(geo["flags"][i, j])
    x = prm["xL"] + (i - 0.5) * prm["dx"]
    inlet = (fl & F_BRR_WALL) == 0 and geo["seg_x1"] is not None and \
        geo["seg_x1"][0] <= i <= geo["seg_x1"][1] and j == geo["seg_x1"][2] and x <= prm["width_neutIn"] + prm["x6"]
    return dict(bLx=float((fl & F_BLX) != 0), bRx=float((fl & F_BRX) != 0), bLrw=float((fl & F_BLR_WALL) != 0),
                bLr=float((fl & F_BLR_WALL) != 0 and (fl & F_BLR_CEN) != 0),
                bRrw=float((fl & F_BRR_WALL) != 0), bRro=float((fl & F_BRR_OPEN) != 0), inlet=inlet)


def update_neutrals(st: dict, prm: dict, geo: dict, solve) -> dict:
    """FluidModule::update_rhon (fluidModule.hpp:4963-5410) then update_rhom
    (:5416-5792).  st: rhon, rhom, rhoUnx, rhoUnr, rhoUnx_wall, rhoUnr_wall, rhoUmx,
    rhoUmr, rhoUmx_wall, rhoUmr_wall, rhoUix_wall, rhoUir_wall, rhoe, nu_excStep,
    nu_super, nu_excMeta, nu_exc, nu_ionz, nu_ionzStep.  prm: dt, ndt_n, ndt_m, dx,
    dr, rmin, xL, x6, width_neutIn, fn_In, Tn, ri, massi, DmN, flag_error.  The
    cell loops follow the blocks; the walls follow the named segments of the
    reference (z0..z5, x0..x5)."""
    ni, nj = geo["ni"], geo["nj"]
    dx, dr = prm["dx"], prm["dr"]
    r = prm["rmin"] + (np.arange(nj + 2) - 0.5) * dr
    C = ion_segments(geo)["c"]
    geo = dict(geo, seg_x1=C["x1"])
    g = {k: v.copy() for k, v in st.items()}
    sh = (ni + 2, nj + 2)
    nb = len(geo["ib"])

    # --- update_rhon -----------------------------------------------------------
    dt_n = prm["dt"] * float(prm["ndt_n"])
    sigma = np.pi * (2.0 * prm["ri"]) * (2.0 * prm["ri"])
    DnN = 2.0 / (3.0 * sigma) * np.sqrt(BOLTZ * prm["Tn"] / (np.pi * prm["massi"]))
    rhon_old, Unx_old, Unr_old = g["rhon"].copy(), g["rhoUnx"].copy(), g["rhoUnr"].copy()
    aP, aE, aW, aN, aS, b = (np.zeros(sh) for _ in range(6))
    x1 = geo["seg_x1"]
    for blk in range(nb):
        I = np.arange(geo["ib"][blk][0], geo["ib"][blk][1] + 1)[:, None]
        J = np.arange(geo["jb"][blk][0], geo["jb"][blk][1] + 1)[None, :]
        rL = (r[J] + r[J - 1]) / 2.0
        rR = (r[J] + r[J + 1]) / 2.0
        qL = (r[J] + r[J - 1]) / 2.0 / r[J]
        qR = (r[J] + r[J + 1]) / 2.0 / r[J]
        DLx = DnN / ((rhon_old[I, J] + rhon_old[I - 1, J]) / 2.0 + 1e-100)
        DRx = DnN / ((rhon_old[I, J] + rhon_old[I + 1, J]) / 2.0 + 1e-100)
        DLr = DnN / ((rhon_old[I, J] + rhon_old[I, J - 1]) / 2.0 + 1e-100)
        DRr = DnN / ((rhon_old[I, J] + rhon_old[I, J + 1]) / 2.0 + 1e-100)
        fl = geo["flags"][I, J].astype(np.int64)
        bLx = ((fl & F_BLX) != 0).astype(float)
        bRx = ((fl & F_BRX) != 0).astype(float)
        bLrw = ((fl & F_BLR_WALL) != 0).astype(float)
        bLr = (((fl & F_BLR_WALL) != 0) & ((fl & F_BLR_CEN) != 0)).astype(float)
        bRrw = ((fl & F_BRR_WALL) != 0).astype(float)
        bRro = ((fl & F_BRR_OPEN) != 0).astype(float)
        x = prm["xL"] + (I - 0.5) * dx
        inlet = ((fl & F_BRR_WALL) == 0) & (x <= prm["width_neutIn"] + prm["x6"]) & (x1 is not None)
        if x1 is not None:
            inlet &= (I >= x1[0]) & (I <= x1[1]) & (J == x1[2])
        bRr_wall = np.where(inlet, 1.0, bRrw)
        bRr_in = np.where(inlet, 0.0, 1.0)
        bRr = bRr_wall * bRr_in * bRro
        W = g
        GLx = np.where(bLx == 0, -W["rhoUix_wall"][I, J] - W["rhoUmx_wall"][I, J], 0.0)
        GRx = np.where(bRx == 0, -W["rhoUix_wall"][I + 1, J] - W["rhoUmx_wall"][I + 1, J], 0.0)
        GLr = np.where(bLrw == 0, -W["rhoUir_wall"][I, J] - W["rhoUmr_wall"][I, J], 0.0)
        GRr = np.where(bRr_wall == 0, -W["rhoUir_wall"][I, J + 1] - W["rhoUmr_wall"][I, J + 1], 0.0)
        Gin = np.where(bRr_in == 0, -W["rhoUir_wall"][I, J + 1] - W["rhoUmr_wall"][I, J + 1] - prm["fn_In"], 0.0)
        Gop = np.where(bRro == 0, np.fmax(rL / rR * Unr_old[I, J], 0.0), 0.0)
        aP[I, J] = ((DRx * bRx + DLx * bLx) * dr * dr + (qR * DRr * bRr + qL * DLr * bLr) * dx * dx
                    + dx * dx * dr * dr / dt_n)
        aE[I, J] = DRx * dr * dr * bRx
        aW[I, J] = DLx * dr * dr * bLx
        aN[I, J] = qR * DRr * dx * dx * bRr
        aS[I, J] = qL * DLr * dx * dx * bLr
        G = (g["nu_excStep"][I, J] + g["nu_super"][I, J]) * g["rhoe"][I, J]
        L = (g["nu_excMeta"][I, J] + 0.5 * g["nu_exc"][I, J] + g["nu_ionz"][I, J]) * g["rhoe"][I, J]
        b[I, J] = (rhon_old[I, J] / dt_n * dx * dx * dr * dr + (G - L) * dx * dx * dr * dr
                   + (GLx) * dr * dx * dr - (GRx) * dr * dx * dr + qL * (GLr) * dx * dx * dr
                   - qR * (GRr + Gop + Gin) * dx * dx * dr)
    x = solve(aP, aE, aW, aN, aS, b, geo["ib"], geo["jb"])
    rhon = g["rhon"]
    for (a0, a1), (c0, c1) in zip(geo["ib"], geo["jb"]):
        rhon[a0:a1 + 1, c0:c1 + 1] = x[a0:a1 + 1, c0:c1 + 1]
    for (a0, a1), (c0, c1) in zip(geo["fxi"], geo["fxj"]):
        I, J, Im = slice(a0, a1 + 1), slice(c0, c1 + 1), slice(a0 - 1, a1)
        D = DnN / ((rhon_old[I, J] + rhon_old[Im, J]) / 2.0 + 1e-100)
        g["rhoUnx"][I, J] = -D * (rhon[I, J] - rhon[Im, J]) / dx
    for (a0, a1), (c0, c1) in zip(geo["fri"], geo["frj"]):
        I, J, Jm = slice(a0, a1 + 1), slice(c0, c1 + 1), slice(c0 - 1, c1)
        D = DnN / ((rhon_old[I, J] + rhon_old[I, Jm]) / 2.0 + 1e-100)
        g["rhoUnr"][I, J] = -D * (rhon[I, J] - rhon[I, Jm]) / dr
    for name in ("z0", "z1", "z2", "z4"):
        for i, j in _pts(C[name]):
            v = -g["rhoUix_wall"][i, j] - g["rhoUmx_wall"][i, j]
            g["rhoUnx"][i, j] = v
            g["rhoUnx_wall"][i, j] = v
    for name in ("z3", "z5"):
        for i, j in _pts(C[name]):
            v = -g["rhoUix_wall"][i + 1, j] - g["rhoUmx_wall"][i + 1, j]
            g["rhoUnx"][i + 1, j] = v
            g["rhoUnx_wall"][i + 1, j] = v
    for name in ("x0", "x2"):
        for i, j in _pts(C[name]):
            v = -g["rhoUir_wall"][i, j] - g["rhoUmr_wall"][i, j]
            g["rhoUnr"][i, j] = v
            g["rhoUnr_wall"][i, j] = v
    for i, j in _pts(C["x1"]):
        x = prm["xL"] + (i - 0.5) * dx
        if x < prm["width_neutIn"] + prm["x6"]:
            g["rhoUnr"][i, j + 1] = -g["rhoUir_wall"][i, j + 1] - g["rhoUmr_wall"][i, j + 1] - prm["fn_In"]
        else:
            v = -g["rhoUir_wall"][i, j + 1] - g["rhoUmr_wall"][i, j + 1]
            g["rhoUnr"][i, j + 1] = v
            g["rhoUnr_wall"][i, j + 1] = v
    for i, j in _pts(C["x4"]):
        v = -g["rhoUir_wall"][i, j + 1] - g["rhoUmr_wall"][i, j + 1]
        g["rhoUnr"][i, j + 1] = v
        g["rhoUnr_wall"][i, j + 1] = v
    for i, j in _pts(C["x5"]):
        rL = (r[j] + r[j - 1]) / 2.0
        rR = (r[j] + r[j + 1]) / 2.0
        g["rhoUnr"][i, j + 1] = max(rL / rR * Unr_old[i, j], 0.0)
        g["rhoUnr_wall"][i, j + 1] = 0.0
    for (a0, a1), (c0, c1) in zip(geo["ib"], geo["jb"]):
        sl = (slice(a0, a1 + 1), slice(c0, c1 + 1))
        rhon[sl] = np.where(rhon[sl] < 0.0, np.fmax(rhon_old[sl], 0.0), rhon[sl])
    fe = prm["flag_error"]
    err_n = calc_res(rhon, rhon_old, geo["ib"], geo["jb"], 1e-100, fe)

    # --- update_rhom -----------------------------------------------------------
    dt_m = prm["dt"] * float(prm["ndt_m"])
    vth = np.sqrt(8.0 * BOLTZ * prm["Tn"] / (np.pi * prm["massi"]))
    rhom_old, Umr_old = g["rhom"].copy(), g["rhoUmr"].copy()
    DmN = prm["DmN"]
    aP, aE, aW, aN, aS, b = (np.zeros(sh) for _ in range(6))
    for blk in range(nb):
        I = np.arange(geo["ib"][blk][0], geo["ib"][blk][1] + 1)[:, None]
        J = np.arange(geo["jb"][blk][0], geo["jb"][blk][1] + 1)[None, :]
        rL = (r[J] + r[J - 1]) / 2.0
        rR = (r[J] + r[J + 1]) / 2.0
        qL = (r[J] + r[J - 1]) / 2.0 / r[J]
        qR = (r[J] + r[J + 1]) / 2.0 / r[J]
        DLx = DmN / ((rhon[I, J] + rhon[I - 1, J]) / 2.0 + 1e-100)
        DRx = DmN / ((rhon[I, J] + rhon[I + 1, J]) / 2.0 + 1e-100)
        DLr = DmN / ((rhon[I, J] + rhon[I, J - 1]) / 2.0 + 1e-100)
        DRr = DmN / ((rhon[I, J] + rhon[I, J + 1]) / 2.0 + 1e-100)
        fl = geo["flags"][I, J].astype(np.int64)
        bLx = ((fl & F_BLX) != 0).astype(float)
        bRx = ((fl & F_BRX) != 0).astype(float)
        bLrw = ((fl & F_BLR_WALL) != 0).astype(float)
        bLr = (((fl & F_BLR_WALL) != 0) & ((fl & F_BLR_CEN) != 0)).astype(float)
        bRrw = ((fl & F_BRR_WALL) != 0).astype(float)
        bRro = ((fl & F_BRR_OPEN) != 0).astype(float)
        bRr = bRrw * bRro
        GLx = np.where(bLx == 0, -0.25 * vth, 0.0)
        GRx = np.where(bRx == 0, 0.25 * vth, 0.0)
        GLr = np.where(bLrw == 0, -0.25 * vth, 0.0)
        GRr = np.where(bRrw == 0, 0.25 * vth, 0.0)
        Gop = np.where(bRro == 0, rL / rR * Umr_old[I, J], 0.0)
        aP[I, J] = ((DRx * bRx + DLx * bLx) * dr * dr + (qR * DRr * bRr + qL * DLr * bLr) * dx * dx
                    - GLx * dr * dx * dr + GRx * dr * dx * dr - qL * GLr * dx * dx * dr
                    + qR * GRr * dx * dx * dr + dx * dx * dr * dr / dt_m)
        aE[I, J] = DRx * dr * dr * bRx
        aW[I, J] = DLx * dr * dr * bLx
        aN[I, J] = qR * DRr * dx * dx * bRr
        aS[I, J] = qL * DLr * dx * dx * bLr
        G = g["rhoe"][I, J] * (g["nu_excMeta"][I, J] + 0.5 * g["nu_exc"][I, J])
        L = g["rhoe"][I, J] * (g["nu_ionzStep"][I, J] + g["nu_excStep"][I, J] + g["nu_super"][I, J])
        b[I, J] = (rhom_old[I, J] / dt_m * dx * dx * dr * dr + (G - L) * dx * dx * dr * dr
                   + (0.0) * dr * dx * dr - (0.0) * dr * dx * dr + qL * (0.0) * dx * dx * dr
                   - qR * (Gop) * dx * dx * dr)
    x = solve(aP, aE, aW, aN, aS, b, geo["ib"], geo["jb"])
    rhom = g["rhom"]
    for (a0, a1), (c0, c1) in zip(geo["ib"], geo["jb"]):
        rhom[a0:a1 + 1, c0:c1 + 1] = x[a0:a1 + 1, c0:c1 + 1]
    for (a0, a1), (c0, c1) in list(zip(geo["ib"], geo["jb"]))[:2]:
        sl = (slice(a0, a1 + 1), slice(c0, c1 + 1))
        rhom[sl] = np.where(rhom[sl] < 0.0, np.fmax(rhom_old[sl], 0.0), rhom[sl])
    for (a0, a1), (c0, c1) in zip(geo["fxi"], geo["fxj"]):
        I, J, Im = slice(a0, a1 + 1), slice(c0, c1 + 1), slice(a0 - 1, a1)
        D = DmN / ((rhon[I, J] + rhon[Im, J]) / 2.0 + 1e-100)
        g["rhoUmx"][I, J] = -D * (rhom[I, J] - rhom[Im, J]) / dx
    for (a0, a1), (c0, c1) in zip(geo["fri"], geo["frj"]):
        I, J, Jm = slice(a0, a1 + 1), slice(c0, c1 + 1), slice(c0 - 1, c1)
        D = DmN / ((rhon[I, J] + rhon[I, Jm]) / 2.0 + 1e-100)
        g["rhoUmr"][I, J] = -D * (rhom[I, J] - rhom[I, Jm]) / dr
    for name in ("z0", "z1", "z2", "z4"):
        for i, j in _pts(C[name]):
            g["rhoUmx"][i, j] = -0.25 * rhom[i, j] * vth
            g["rhoUmx_wall"][i, j] = g["rhoUmx"][i, j]
    for name in ("z3", "z5"):
        for i, j in _pts(C[name]):
            g["rhoUmx"][i + 1, j] = 0.25 * rhom[i, j] * vth
            g["rhoUmx_wall"][i + 1, j] = g["rhoUmx"][i + 1, j]
    for name in ("x0", "x2"):
        for i, j in _pts(C[name]):
            g["rhoUmr"][i, j] = -0.25 * rhom[i, j] * vth
            g["rhoUmr_wall"][i, j] = g["rhoUmr"][i, j]
    for name in ("x1", "x4"):
        for i, j in _pts(C[name]):
            g["rhoUmr"][i, j + 1] = 0.25 * rhom[i, j] * vth
            g["rhoUmr_wall"][i, j + 1] = g["rhoUmr"][i, j + 1]
    for i, j in _pts(C["x5"]):
        rL = (r[j] + r[j - 1]) / 2.0
        rR = (r[j] + r[j + 1]) / 2.0
        g["rhoUmr"][i, j + 1] = Umr_old[i, j] * rL / rR
        g["rhoUmr_wall"][i, j + 1] = 0.0
    err_m = calc_res(rhom, rhom_old, geo["ib"], geo["jb"], 1e-100, fe)
    out = {k: g[k] for k in ("rhon", "rhom", "rhoUnx", "rhoUnr", "rhoUnx_wall", "rhoUnr_wall", "rhoUmx", "rhoUmr",
                             "rhoUmx_wall", "rhoUmr_wall")}
    out.update(rhon_old=rhon_old, rhom_old=rhom_old, error_rhon=err_n, error_rhom=err_m)
    return out


def fluid_step(st: dict, P: dict, geo: dict, see, tb: dict, solve) -> dict:
    """One time step in the order of src/main.cpp:170-251 chained from the
    restatements above: check_CFL, ion sub-step, potential, electron density and
    energy predictor-correctors, neutrals, transport coefficients.  P holds itime,
    ndt_*, flag_adp_dt, dt, CFL, gtime and the blocks ion, phi, rhoe, eps, neutral
    (with xL, x6, width_neutIn), transport; it is updated in place.  Returns the
    new state."""
    s = dict(st)
    c = check_cfl(s, dict(rmin=P["transport"]["rmin"], dr=P["transport"]["dr"], masse=P["transport"]["masse"],
                          flag_adp_dt=P["flag_adp_dt"], CFL=P["CFL"], dt=P["dt"]))
    P["dt"], P["CFL"] = c["dt"], c["CFL"]
    P["gtime"] += P["dt"]
    P["itime"] += 1
    for blk in ("ion", "phi", "rhoe", "eps", "neutral"):
        P[blk]["dt"] = P["dt"]
    P["ion"]["CFL"] = P["CFL"]
    if P["itime"] % P["ndt_i"] == 0:
        s.update({k: v for k, v in ion_step(s, P["ion"], geo, solve, solve, solve).items()
                  if not k.startswith("error")})
    s.update({k: v for k, v in solve_phi_pc(s, P["phi"], geo, see, solve).items()
              if k in ("phi", "Ex", "Er", "nUex", "nUer")})
    s.update({k: v for k, v in solve_sg_pc(s, P["rhoe"], geo, see, solve, "rhoe").items()
              if k in ("rhoe", "rhoUex", "rhoUer", "rhoUex_wall", "rhoUer_wall", "rhoe_old", "I_Anode", "Ii_Anode",
                       "Ie_Anode")})
    s.update({k: v for k, v in solve_sg_pc(s, P["eps"], geo, see, solve, "rhoeps").items()
              if k in ("rhoeps", "Gx", "Gr", "Gx_wall", "Gr_wall", "Te", "Te_old")})
    if P["itime"] % P["ndt_n"] == 0 and P["itime"] % P["ndt_m"] == 0:
        s.update({k: v for k, v in update_neutrals(s, P["neutral"], geo, solve).items() if not k.startswith("error")})
    s.update(update_transport_coef(s, tb, P["transport"], geo["flags"]))
    return s
