"""CPU restatement of the reference's microwave (frequency-domain) solve.

TEST INFRASTRUCTURE ONLY (checker and CPU baseline; the product never imports it).

Restated here:
  * the coax impedance test, EmfieldModule::solve_Microwave_impedanceTest
    (include/emfieldModule.hpp:5528-6099) on the boundary lists of
    InitialModule::makeBoundary_impedanceTest (include/initialModule.hpp:1061-1330):
    Er-only 5-point complex system, port excitation (code 7) at z=0, first-order
    open boundary (code 1) at z=L, Gauss-law walls (code 2) at r=r1 and r=r2,
    direct sparse solve (Eigen SparseLU in the reference, SuperLU here: the same
    supernodal-LU family), ghost post-processing, port V/I, forward power and the
    rescaling to Pmw;
  * the cell-centred output of OutputModule::output_phase
    (include/outputModule.hpp:81-83 for Er, :136-139 for the analytic TEM field).
Arrays follow the reference: (ni+2, nj+2) complex128, [i][j], Er at r-faces j-1/2.
"""
from __future__ import annotations

import re

import numpy as np

E0 = 1.60217662e-19
EPS0 = 8.8541878128e-12
MU0 = 1.2566370614e-6


def coax_params() -> dict:
    """Parameters of the reference calibration run (test/校正/setup.yaml)."""
    ni, nj = 194, 7
    xL, xR, rmin, rmax = 0.0, 0.0388, 0.0006, 0.002
    fmw = 4.25e9
    p = dict(ni=ni, nj=nj, xL=xL, xR=xR, rmin=rmin, rmax=rmax, fmw=fmw, Pmw=8.0, Z0=50.0,
             J1r_exc=0.212687, epsr_diele=2.083825280349, nu_eff=2.0e9, masse=9.10938356e-31)
    # iniParam (initialModule.hpp:54-84)
    p["dx"] = (xR - xL) / ni
    p["dr"] = (rmax - rmin) / nj
    p["omegam"] = 2.0 * np.pi * fmw
    p["x"] = xL + (np.arange(ni + 2) - 0.5) * p["dx"]
    p["r"] = rmin + (np.arange(nj + 2) - 0.5) * p["dr"]
    # makeBoundary_impedanceTest: r1 = rmin, r2 = rmax, Er faces i=1..ni, j=2..nj,
    # epsr = epsr_diele in the cells (initialModule.hpp:1068-1072, :1090-1093, :1320-1325)
    p["r1"], p["r2"] = rmin, rmax
    epsr = np.ones((ni + 2, nj + 2))
    epsr[1:ni + 1, 1:nj + 1] = p["epsr_diele"]
    p["epsr"] = epsr
    return p


def coax_er_system(p: dict):
    """Er coefficients of solve_Microwave_impedanceTest after the BC surgery.

    Returns dict with complex (ni+2, nj+2) arrays aP, aE, aW, aN, aS, b and the
    unknown mask (Er faces i=1..ni, j=2..nj).  Stencil convention as the
    reference: aP x_P - aE x_E - aW x_W - aN x_N - aS x_S = b.
    """
    ni, nj, dx, dr, w = p["ni"], p["nj"], p["dx"], p["dr"], p["omegam"]
    r, epsr = p["r"], p["epsr"]
    shape = (ni + 2, nj + 2)
    aP = np.zeros(shape, complex); aE = np.zeros(shape, complex); aW = np.zeros(shape, complex)
    aN = np.zeros(shape, complex); aS = np.zeros(shape, complex); b = np.zeros(shape, complex)
    mask = np.zeros(shape, bool)
    # rho = 0 in the test (emfieldModule.hpp:5531-5536): sigma = 0
    for i in range(1, ni + 1):
        for j in range(2, nj + 1):
            rC = (r[j - 1] + r[j]) / 2.0
            rR = (r[j] + r[j + 1]) / 2.0
            rL = (r[j - 2] + r[j - 1]) / 2.0
            eps_t = (epsr[i, j] + epsr[i, j - 1]) / 2.0
            aP[i, j] = (rC * (1.0 / r[j] + 1.0 / r[j - 1]) * dx * dx + 2.0 * dr * dr
                        - EPS0 * eps_t * MU0 * w * w * dx * dx * dr * dr)
            aE[i, j] = dr * dr
            aW[i, j] = dr * dr
            aN[i, j] = rR / r[j] * dx * dx
            aS[i, j] = rL / r[j - 1] * dx * dx
            mask[i, j] = True
    # left (code 7, excitation), emfieldModule.hpp:5616-5633
    for j in range(2, nj + 1):
        i = 1
        eps_t = (epsr[i, j] + epsr[i, j - 1]) / 2.0
        c0 = np.sqrt(1.0 / (EPS0 * eps_t * MU0))
        deno = complex(2.0 * c0, w * dx)
        R = complex(2.0 * c0, -w * dx)
        r_t = (r[j] + r[j - 1]) / 2.0
        Er_Fw = p["J1r_exc"] / r_t / np.log(p["r2"] / p["r1"]) * 1e3
        S = complex(0.0, 4.0 * w * dx) * Er_Fw
        aP[i, j] = aP[i, j] - aW[i, j] * R / (deno + 1e-100)
        b[i, j] = b[i, j] + aW[i, j] * S / (deno + 1e-100)
        aW[i, j] = 0.0
    # right (code 1, open), emfieldModule.hpp:5642-5657
    for j in range(2, nj + 1):
        i = ni
        eps_t = (epsr[i, j] + epsr[i, j - 1]) / 2.0
        c0 = np.sqrt(1.0 / (EPS0 * eps_t * MU0))
        deno = (2.0 * c0) ** 2 + (w * dx) ** 2
        R = complex((2.0 * c0) ** 2 - (w * dx) ** 2, -4.0 * c0 * w * dx)
        aP[i, j] = aP[i, j] - aE[i, j] * R / (deno + 1e-100)
        aE[i, j] = 0.0
    # lower (code 2, Gauss), emfieldModule.hpp:5675-5682; the SE/SW terms couple to Ex,
    # which the impedance test does not solve
    for i in range(1, ni + 1):
        j = 2
        rR = (r[j] + r[j - 1]) / 2.0
        rL = (r[j - 1] + r[j - 2]) / 2.0
        aP[i, j] = aP[i, j] - aS[i, j] * rR / rL
        aS[i, j] = 0.0
    # upper (code 2, Gauss), emfieldModule.hpp:5706-5712
    for i in range(1, ni + 1):
        j = nj
        rR = (r[j + 1] + r[j]) / 2.0
        rL = (r[j] + r[j - 1]) / 2.0
        aP[i, j] = aP[i, j] - aN[i, j] * rL / rR
        aN[i, j] = 0.0
    return dict(aP=aP, aE=aE, aW=aW, aN=aN, aS=aS, b=b, mask=mask)


def solve_c5_direct(sysd: dict) -> np.ndarray:
    """Sparse direct solve of a complex 5-point system on its unknown mask
    (couplings to non-unknowns dropped, as the Eigen assembly at
    emfieldModule.hpp:5749-5766 inserts only unknown-to-unknown entries)."""
    import scipy.sparse as sp
    import scipy.sparse.linalg as spla
    m = sysd["mask"]
    n = int(m.sum())
    idx = -np.ones(m.shape, np.int64)
    idx[m] = np.arange(n)
    ci, cj = np.nonzero(m)
    k = idx[ci, cj]
    rows = [k]
    cols = [k]
    vals = [sysd["aP"][ci, cj]]
    for name, di, dj in (("aE", 1, 0), ("aW", -1, 0), ("aN", 0, 1), ("aS", 0, -1)):
        ii, jj = ci + di, cj + dj
        ok = (ii >= 0) & (ii < m.shape[0]) & (jj >= 0) & (jj < m.shape[1])
        nb = np.full(ci.shape, -1, np.int64)
        nb[ok] = idx[ii[ok], jj[ok]]
        sel = nb >= 0
        rows.append(k[sel])
        cols.append(nb[sel])
        vals.append(-sysd[name][ci[sel], cj[sel]])
    A = sp.csc_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))), shape=(n, n))
    xk = spla.spsolve(A, sysd["b"][ci, cj])
    x = np.zeros(m.shape, complex)
    x[ci, cj] = xk
    return x


def coax_postprocess(E1r: np.ndarray, p: dict):
    """Ghost values, port V/I, forward power and rescaling to Pmw
    (emfieldModule.hpp:5788-5815, :5835-5861, :5880-5960 and :6001-6036).
    Returns (scaled E1r, scaled J1r_exc scalar, dict of port quantities)."""
    ni, nj, dx, dr, w = p["ni"], p["nj"], p["dx"], p["dr"], p["omegam"]
    r, epsr = p["r"], p["epsr"]
    E = E1r.copy()
    # left ghost (code 7)
    for j in range(2, nj + 1):
        i = 1
        eps_t = (epsr[i, j] + epsr[i, j - 1]) / 2.0
        c0 = np.sqrt(1.0 / (EPS0 * eps_t * MU0))
        deno = complex(2.0 * c0, w * dx)
        R = complex(2.0 * c0, -w * dx)
        r_t = (r[j] + r[j - 1]) / 2.0
        Er_Fw = p["J1r_exc"] / r_t / np.log(p["r2"] / p["r1"]) * 1e3
        S = complex(0.0, 4.0 * w * dx) * Er_Fw
        E[i - 1, j] = R / (deno + 1e-100) * E[i, j] + S / (deno + 1e-100)
    # lower / upper Gauss ghosts with E1x = 0
    for i in range(1, ni + 1):
        j = 2
        rR = (r[j] + r[j - 1]) / 2.0
        rL = (r[j - 1] + r[j - 2]) / 2.0
        E[i, j - 1] = rR / rL * E[i, j]
        j = nj
        rR = (r[j + 1] + r[j]) / 2.0
        rL = (r[j] + r[j - 1]) / 2.0
        E[i, j + 1] = rL / rR * E[i, j]
    # reference plane i_ref = int(0/dx + 1.5) = 1
    i = int(0.0 / dx + 1.5)
    I_ref = 0.0j
    coef = 0.0j
    n = 0
    for j in range(2, nj + 1):
        r_t = (r[j] + r[j - 1]) / 2.0
        H = (E[i, j] - E[i - 1, j]) / dx / (w * MU0) * 1j
        I_ref += 2.0 * np.pi * r_t * H
        coef += (E[i, j] + E[i - 1, j]) / 2.0 * r_t
        n += 1
    I_ref /= n
    coef /= n
    V_ref = coef * np.log(p["r2"] / p["r1"])
    Z0 = p["Z0"]
    a2 = (V_ref - Z0 * I_ref) / (2.0 * np.sqrt(2.0 * Z0))
    b2 = (V_ref + Z0 * I_ref) / (2.0 * np.sqrt(2.0 * Z0))
    P_fwd = abs(b2) ** 2
    ratio = p["Pmw"] / P_fwd
    return E * np.sqrt(ratio), p["J1r_exc"] * np.sqrt(ratio), dict(V=V_ref, I=I_ref, P_fwd=P_fwd,
                                                                   P_ref=abs(a2) ** 2, ratio=ratio)


def coax_output(Es: np.ndarray, J1r_exc: float, p: dict, n: int = 0):
    """Cell-centred Er and the analytic TEM field of phase snapshot n of 18
    (outputModule.hpp:81-83, :136-139).  Returns (Er, Er_anly) of shape (ni, nj)."""
    ni, nj, w = p["ni"], p["nj"], p["omegam"]
    r, x, epsr = p["r"], p["x"], p["epsr"]
    deg = 2.0 * np.pi / 18 * n
    Er = np.zeros((ni, nj), complex)
    An = np.zeros((ni, nj), complex)
    for i in range(1, ni + 1):
        for j in range(1, nj + 1):
            rL = (r[j - 1] + r[j]) / 2.0
            rR = (r[j + 1] + r[j]) / 2.0
            Er[i - 1, j - 1] = (rR * Es[i, j + 1] + rL * Es[i, j]) / (2.0 * r[j]) * np.exp(1j * deg)
            c0 = np.sqrt(1.0 / (EPS0 * epsr[i, j] * MU0))
            An[i - 1, j - 1] = J1r_exc / r[j] * 1e3 / np.log(p["r2"] / p["r1"]) * np.exp(1j * (-w / c0 * x[i] + deg))
    return Er, An


def er_rect_params(ni: int, nj: int, Lz: float = 10e-3, Lr: float = 5e-3, fmw: float = 2.67e10 / (2 * np.pi),
                   J1r_exc: float = 0.212687, r1: float = 0.6e-3, r2: float = 2.0e-3) -> dict:
    """Rectangle r in [0, Lr], z in [0, Lz] with the coax feed radii r1, r2."""
    dx, dr = Lz / ni, Lr / nj
    return dict(ni=ni, nj=nj, dx=dx, dr=dr, omegam=2.0 * np.pi * fmw, J1r_exc=J1r_exc, r1=r1, r2=r2,
                masse=9.10938356e-31, x=(np.arange(ni + 2) - 0.5) * dx, r=(np.arange(nj + 2) - 0.5) * dr)


def er_rect_system(ne: np.ndarray, nu: np.ndarray, epsr: np.ndarray, p: dict):
    """Er equation of solve_Microwave (emfieldModule.hpp:2350-2395) with B = 0,
    so that sigma_rr = n e^2 / (m (nu + i w)) and every Hall coupling to Ex / Ephi
    vanishes, on the rectangle with the impedance test's boundary codes:
    port excitation (code 7, :5616-5633) on the z = 0 faces with r1 <= r <= r2 and
    first-order open (code 1, :5602-5612) on the other z = 0 faces, open (code 1,
    :5642-5657) at z = L, Gauss (code 2, :5706-5712) at r = R (its coupling to Ex
    dropped: Ex is not part of this system), and Er = 0 on the axis face r = 0
    (the axis face is not an unknown).  Unknowns: Er faces i = 1..ni, j = 2..nj."""
    ni, nj, dx, dr, w = p["ni"], p["nj"], p["dx"], p["dr"], p["omegam"]
    r, me = p["r"], p["masse"]
    sh = (ni + 2, nj + 2)
    aP = np.zeros(sh, complex); aE = np.zeros(sh, complex); aW = np.zeros(sh, complex)
    aN = np.zeros(sh, complex); aS = np.zeros(sh, complex); b = np.zeros(sh, complex)
    mask = np.zeros(sh, bool)
    EPS = complex(1e-100, 1e-100)
    iwm = complex(0.0, w * MU0)
    I = slice(1, ni + 1)
    jj = np.arange(2, nj + 1)
    r_t = ((r[jj - 1] + r[jj]) / 2.0)[None, :]
    rR = ((r[jj] + r[jj + 1]) / 2.0)[None, :]
    rL = ((r[jj - 2] + r[jj - 1]) / 2.0)[None, :]
    nu_t = (nu[I, 2:nj + 1] + nu[I, 1:nj]) / 2.0
    rho_t = (ne[I, 2:nj + 1] + ne[I, 1:nj]) / 2.0
    eps_t = (epsr[I, 2:nj + 1] + epsr[I, 1:nj]) / 2.0
    coef = rho_t * E0 * E0 / (me * (nu_t + 1j * w) + EPS) / (1.0 + EPS)
    J = slice(2, nj + 1)
    aP[I, J] = (r_t * (1.0 / r[jj][None, :] + 1.0 / r[jj - 1][None, :]) * dx * dx + 2.0 * dr * dr
                - EPS0 * eps_t * MU0 * w * w * dx * dx * dr * dr + iwm * coef * dx * dx * dr * dr)
    aE[I, J] = dr * dr
    aW[I, J] = dr * dr
    aN[I, J] = rR / r[jj][None, :] * dx * dx
    aS[I, J] = rL / r[jj - 1][None, :] * dx * dx
    mask[I, J] = True
    for j in range(2, nj + 1):
        # left: port on [r1, r2], open elsewhere
        i = 1
        eps_t = (epsr[i, j] + epsr[i, j - 1]) / 2.0
        c0 = np.sqrt(1.0 / (EPS0 * eps_t * MU0))
        r_t = (r[j] + r[j - 1]) / 2.0
        if p["r1"] <= r_t <= p["r2"]:
            deno = complex(2.0 * c0, w * dx)
            R = complex(2.0 * c0, -w * dx)
            Er_Fw = p["J1r_exc"] / r_t / np.log(p["r2"] / p["r1"]) * 1e3
            S = complex(0.0, 4.0 * w * dx) * Er_Fw
            aP[i, j] -= aW[i, j] * R / (deno + 1e-100)
            b[i, j] += aW[i, j] * S / (deno + 1e-100)
        else:
            deno = (2.0 * c0) ** 2 + (w * dx) ** 2
            R = complex((2.0 * c0) ** 2 - (w * dx) ** 2, -4.0 * c0 * w * dx) / (deno + 1e-100)
            aP[i, j] -= aW[i, j] * R
        aW[i, j] = 0.0
        # right: open
        i = ni
        eps_t = (epsr[i, j] + epsr[i, j - 1]) / 2.0
        c0 = np.sqrt(1.0 / (EPS0 * eps_t * MU0))
        deno = (2.0 * c0) ** 2 + (w * dx) ** 2
        R = complex((2.0 * c0) ** 2 - (w * dx) ** 2, -4.0 * c0 * w * dx)
        aP[i, j] -= aE[i, j] * R / (deno + 1e-100)
        aE[i, j] = 0.0
    for i in range(1, ni + 1):
        j = nj
        rR = (r[j + 1] + r[j]) / 2.0
        rL = (r[j] + r[j - 1]) / 2.0
        aP[i, j] -= aN[i, j] * rL / rR
        aN[i, j] = 0.0
        aS[i, 2] = 0.0
    return dict(aP=aP, aE=aE, aW=aW, aN=aN, aS=aS, b=b, mask=mask)


# ---------------------------------------------------------------------------
# two-port feed helpers (include/cmpMat2.hpp:8-34, include/initialModule.hpp:
# 107-192 and 1689-1739), restated with numpy complex scalars
# ---------------------------------------------------------------------------
def s_to_abcd(S11, S21, S12, S22, Z0):
    """sParamToABCD (initialModule.hpp:1689-1710); ValueError where the reference throws."""
    if abs(S21) < 1.0e-14:
        raise ValueError("S21 is too small")
    den = 2.0 * S21
    return np.array([[((1 + S11) * (1 - S22) + S12 * S21) / den, Z0 * ((1 + S11) * (1 + S22) - S12 * S21) / den],
                     [1.0 / Z0 * ((1 - S11) * (1 - S22) - S12 * S21) / den,
                      ((1 - S11) * (1 + S22) + S12 * S21) / den]])


def abcd_to_s(T, Z0):
    """ABCDToSParam (initialModule.hpp:1717-1739)."""
    A, B, C, D = T[0, 0], T[0, 1], T[1, 0], T[1, 1]
    den = A + B / Z0 + C * Z0 + D
    if abs(den) < 1.0e-14:
        raise ValueError("denominator is too small")
    return ((A + B / Z0 - C * Z0 - D) / den, 2.0 / den, 2.0 * (A * D - B * C) / den, (-A + B / Z0 - C * Z0 + D) / den)


def sparam_setup(p: dict):
    """S-parameters after the stub and cable corrections (initialModule.hpp:107-192)."""
    def polar(mag, arg):
        return complex(mag * np.cos(arg / 180.0 * np.pi), mag * np.sin(arg / 180.0 * np.pi))
    S = [polar(p[f"{n}_mag"], p[f"{n}_arg_deg"]) for n in ("S11", "S21", "S12", "S22")]
    ph = p["phase_pre_deg"] / 180.0 * np.pi
    Z0 = p["Z0"]
    Tpre = np.array([[np.cos(ph), 1j * Z0 * np.sin(ph)], [1j * np.sin(ph) / Z0, np.cos(ph)]])
    Tbase = s_to_abcd(*S, Z0)
    c0 = np.sqrt(1.0 / (8.8541878128e-12 * p["epsr_diele"] * 1.2566370614e-6))
    beta = p["omegam"] / c0
    t0, t1 = np.tan(beta * p["h0_stab"]), np.tan(beta * (p["h0_stab"] + p["dh_stab"]))
    if abs(t0) < 1e-14 or abs(t1) < 1e-14:
        raise ValueError("tan(beta*l) is too small")
    dYs = (-1j / Z0 / t1) - (-1j / Z0 / t0)
    Tcorr = np.array([[1.0, 0.0], [dYs, 1.0]])
    Tstub = Tpre @ Tcorr @ np.linalg.inv(Tpre) @ Tbase
    S11, S21, S12, S22 = abcd_to_s(Tstub, Z0)
    q = np.exp(-1j * beta * p["dl_cable"])
    return (S11, S21 * q, S12 * q, S22 * q * q), beta * p["dl_cable"] / np.pi * 180.0


def energy_profile(E1x, E1r, E1p, rhoe, nu_m1, Bx, Br, p, xblocks, rblocks, cblocks):
    """Absorbed-power part of update_energy_profile (emfieldModule.hpp:7630-7790)
    on [i][j] arrays; blocks are (i0, i1, j0, j1) inclusive index boxes (a cell
    in several boxes is counted once, as a block union).  Returns J1x, J1r,
    J1p, Pabsx, Pabsr, Pabsp, Pabs (zero outside the blocks) and (Px, Pr, Pp)."""
    e0, me, w = 1.60217662e-19, p["masse"], p["omegam"]
    dx, dr = p["dx"], p["dr"]
    ni2, nj2 = rhoe.shape
    r = p["rmin"] + (np.arange(nj2) - 0.5) * dr
    EPS = 1e-100 + 1e-100j

    def mask(blocks):
        m = np.zeros((ni2, nj2), bool)
        for i0, i1, j0, j1 in blocks:
            m[i0:i1 + 1, j0:j1 + 1] = True
        return m

    def sig(nu, rho, bx, br):
        den = me * (nu + 1j * w) + EPS
        hx, hr = e0 * bx / den, e0 * br / den
        coef = rho * e0 * e0 / den / (1.0 + hx * hx + hr * hr + EPS)
        return coef, hx, hr

    out = {k: np.zeros((ni2, nj2), complex) for k in ("J1x", "J1r", "J1p")}
    out.update({k: np.zeros((ni2, nj2)) for k in ("Pabsx", "Pabsr", "Pabsp", "Pabs")})
    P = [0.0, 0.0, 0.0]
    mx, mr, mc = mask(xblocks), mask(rblocks), mask(cblocks)
    for i, j in zip(*np.nonzero(mx)):
        rL, rR = (r[j] + r[j - 1]) / 2, (r[j] + r[j + 1]) / 2
        c, hx, hr = sig((nu_m1[i, j] + nu_m1[i - 1, j]) / 2, (rhoe[i, j] + rhoe[i - 1, j]) / 2,
                        (Bx[i, j] + Bx[i - 1, j]) / 2, (Br[i, j] + Br[i - 1, j]) / 2)
        Ex = E1x[i, j]
        Er = (rL * (E1r[i, j] + E1r[i - 1, j]) + rR * (E1r[i, j + 1] + E1r[i - 1, j + 1])) / (4 * r[j])
        Ep = (E1p[i, j] + E1p[i - 1, j]) / 2
        J = c * hx * hr * Er + c * hr * Ep + c * (1 + hx * hx) * Ex
        out["J1x"][i, j] = J
        out["Pabsx"][i, j] = 0.5 * (J * np.conj(Ex)).real
        P[0] += out["Pabsx"][i, j] * dx * dr * 2 * np.pi * r[j]
    for i, j in zip(*np.nonzero(mr)):
        rt = (r[j - 1] + r[j]) / 2
        c, hx, hr = sig((nu_m1[i, j] + nu_m1[i, j - 1]) / 2, (rhoe[i, j] + rhoe[i, j - 1]) / 2,
                        (r[j] * Bx[i, j] + r[j - 1] * Bx[i, j - 1]) / (2 * rt),
                        (r[j] * Br[i, j] + r[j - 1] * Br[i, j - 1]) / (2 * rt))
        Ex = (r[j] * (E1x[i, j] + E1x[i + 1, j]) + r[j - 1] * (E1x[i, j - 1] + E1x[i + 1, j - 1])) / (4 * rt)
        Er = E1r[i, j]
        Ep = (r[j] * E1p[i, j] + r[j - 1] * E1p[i, j - 1]) / (2 * rt)
        J = c * (1 + hr * hr) * Er + c * (-hx) * Ep + c * hx * hr * Ex
        out["J1r"][i, j] = J
        out["Pabsr"][i, j] = 0.5 * (J * np.conj(Er)).real
        P[1] += out["Pabsr"][i, j] * dx * dr * 2 * np.pi * rt
    for i, j in zip(*np.nonzero(mc)):
        qL = (r[j - 1] + r[j]) / 2 / (r[j] + 1e-100)
        qR = (r[j + 1] + r[j]) / 2 / (r[j] + 1e-100)
        c, hx, hr = sig(nu_m1[i, j], rhoe[i, j], Bx[i, j], Br[i, j])
        Ex = (E1x[i, j] + E1x[i + 1, j]) / 2
        Er = (qR * E1r[i, j + 1] + qL * E1r[i, j]) / 2
        Ep = E1p[i, j]
        J = c * hx * Er + c * Ep + c * (-hr) * Ex
        out["J1p"][i, j] = J
        out["Pabsp"][i, j] = 0.5 * (J * np.conj(Ep)).real
        P[2] += out["Pabsp"][i, j] * dx * dr * 2 * np.pi * r[j]
    for i, j in zip(*np.nonzero(mc)):
        out["Pabs"][i, j] = ((out["Pabsx"][i, j] + out["Pabsx"][i + 1, j]) / 2
                             + (out["Pabsr"][i, j] + out["Pabsr"][i, j + 1]) / 2 + out["Pabsp"][i, j])
    return out, tuple(P)


# ---------------------------------------------------------------------------
# magnetised 3-component system of EmfieldModule::solve_Microwave
# (include/emfieldModule.hpp:2249-2998) on the rectangle r in [0, R], z in [0, L]
# ---------------------------------------------------------------------------
MAG_X = ("P", "E", "W", "N", "S", "NE", "SE", "NW", "SW", "EE", "WW")   # Ex rows: Er at NE..SW, Ephi at EE, WW
MAG_R = ("P", "E", "W", "N", "S", "NE", "SE", "NW", "SW", "NN", "SS")   # Er rows: Ex at NE..SW, Ephi at NN, SS
MAG_P = ("P", "E", "W", "N", "S", "EE", "WW", "NN", "SS")               # Ephi rows: Ex at EE, WW, Er at NN, SS


def mag_masks(ni: int, nj: int):
    """Unknowns of the rectangle: Ex x-faces i = 2..ni (the z = 0 and z = L faces
    are eliminated by the Gauss law), j = 1..nj; Er r-faces i = 1..ni, j = 2..nj
    (the axis face is not an unknown, the r = R face is eliminated by the Gauss
    law); Ephi cells i = 1..ni, j = 1..nj."""
    mx = np.zeros((ni + 2, nj + 2), bool); mx[2:ni + 1, 1:nj + 1] = True
    mr = np.zeros((ni + 2, nj + 2), bool); mr[1:ni + 1, 2:nj + 1] = True
    mp = np.zeros((ni + 2, nj + 2), bool); mp[1:ni + 1, 1:nj + 1] = True
    return mx, mr, mp


def _sigma_terms(rho, nu, bx, br, w, me):
    """coef and the Hall factors of the magnetised cold-plasma conductivity
    (emfieldModule.hpp:2312-2318), with the reference's EPS = 1e-100 (1 + i) guards."""
    EPS = complex(1e-100, 1e-100)
    nu_c = nu + 1j * w
    hx = E0 * bx / (me * nu_c + EPS)
    hr = E0 * br / (me * nu_c + EPS)
    mag2 = hx * hx + hr * hr
    coef = rho * E0 * E0 / (me * nu_c + EPS) / (1.0 + mag2 + EPS)
    return coef, hx, hr


def _mag_interior(ne, nu, Bx, Br, epsr, p: dict, masks):
    """Interior coefficients of the three field equations on their unknowns
    (emfieldModule.hpp:2300-2453), before any boundary surgery."""
    ni, nj, dx, dr, w, me = p["ni"], p["nj"], p["dx"], p["dr"], p["omegam"], p["masse"]
    r = p["r"]
    sh = (ni + 2, nj + 2)
    iwm = complex(0.0, w * MU0)
    D = dx * dx * dr * dr
    X = {k: np.zeros(sh, complex) for k in MAG_X}
    Rr = {k: np.zeros(sh, complex) for k in MAG_R}
    Pp = {k: np.zeros(sh, complex) for k in MAG_P}
    bx = np.zeros(sh, complex); br = np.zeros(sh, complex); bp = np.zeros(sh, complex)
    mx, mr, mp = masks
    # --- Ex on x-faces (i between cells i-1 and i) ---
    I, J = np.nonzero(mx)
    qL = (r[J - 1] + r[J]) / 2.0 / (r[J] + 1e-100)
    qR = (r[J + 1] + r[J]) / 2.0 / (r[J] + 1e-100)
    coef, hx, hr = _sigma_terms((ne[I, J] + ne[I - 1, J]) / 2.0, (nu[I, J] + nu[I - 1, J]) / 2.0,
                                (Bx[I, J] + Bx[I - 1, J]) / 2.0, (Br[I, J] + Br[I - 1, J]) / 2.0, w, me)
    eps_t = (epsr[I, J] + epsr[I - 1, J]) / 2.0
    s_xr, s_xp, s_xx = coef * (hx * hr), coef * hr, coef * (1.0 + hx * hx)
    X["P"][I, J] = 2.0 * dx * dx + 2.0 * dr * dr - EPS0 * eps_t * MU0 * w * w * D + iwm * s_xx * D
    X["E"][I, J] = dr * dr; X["W"][I, J] = dr * dr
    X["N"][I, J] = qR * dx * dx; X["S"][I, J] = qL * dx * dx
    X["EE"][I, J] = -iwm * s_xp * 0.5 * D; X["WW"][I, J] = -iwm * s_xp * 0.5 * D
    X["NE"][I, J] = -iwm * s_xr * 0.25 * qR * D; X["NW"][I, J] = -iwm * s_xr * 0.25 * qR * D
    X["SE"][I, J] = -iwm * s_xr * 0.25 * qL * D; X["SW"][I, J] = -iwm * s_xr * 0.25 * qL * D
    # --- Er on r-faces (j between cells j-1 and j) ---
    I, J = np.nonzero(mr)
    r_t = (r[J - 1] + r[J]) / 2.0
    rR = (r[J] + r[J + 1]) / 2.0
    rL = (r[J - 2] + r[J - 1]) / 2.0
    coef, hx, hr = _sigma_terms((ne[I, J] + ne[I, J - 1]) / 2.0, (nu[I, J] + nu[I, J - 1]) / 2.0,
                                (r[J] * Bx[I, J] + r[J - 1] * Bx[I, J - 1]) / (2.0 * r_t),
                                (r[J] * Br[I, J] + r[J - 1] * Br[I, J - 1]) / (2.0 * r_t), w, me)
    eps_t = (epsr[I, J] + epsr[I, J - 1]) / 2.0
    s_rr, s_rp, s_rx = coef * (1.0 + hr * hr), coef * (-hx), coef * (hx * hr)
    Rr["P"][I, J] = (r_t * (1.0 / r[J] + 1.0 / r[J - 1]) * dx * dx + 2.0 * dr * dr
                     - EPS0 * eps_t * MU0 * w * w * D + iwm * s_rr * D)
    Rr["E"][I, J] = dr * dr; Rr["W"][I, J] = dr * dr
    Rr["N"][I, J] = rR / r[J] * dx * dx; Rr["S"][I, J] = rL / r[J - 1] * dx * dx
    Rr["NN"][I, J] = -iwm * s_rp * 0.5 * r[J] / r_t * D
    Rr["SS"][I, J] = -iwm * s_rp * 0.5 * r[J - 1] / r_t * D
    Rr["NE"][I, J] = -iwm * s_rx * 0.25 * r[J] / r_t * D; Rr["NW"][I, J] = -iwm * s_rx * 0.25 * r[J] / r_t * D
    Rr["SE"][I, J] = -iwm * s_rx * 0.25 * r[J - 1] / r_t * D; Rr["SW"][I, J] = -iwm * s_rx * 0.25 * r[J - 1] / r_t * D
    # --- Ephi on cells ---
    I, J = np.nonzero(mp)
    qL = (r[J - 1] + r[J]) / 2.0 / (r[J] + 1e-100)
    qR = (r[J + 1] + r[J]) / 2.0 / (r[J] + 1e-100)
    coef, hx, hr = _sigma_terms(ne[I, J], nu[I, J], Bx[I, J], Br[I, J], w, me)
    s_pr, s_pp, s_px = coef * hx, coef, coef * (-hr)
    Pp["P"][I, J] = (2.0 * dx * dx + 2.0 * dr * dr + D / (r[J] * r[J])
                     - EPS0 * epsr[I, J] * MU0 * w * w * D + iwm * s_pp * D)
    Pp["E"][I, J] = dr * dr; Pp["W"][I, J] = dr * dr
    Pp["N"][I, J] = qR * dx * dx; Pp["S"][I, J] = qL * dx * dx
    Pp["EE"][I, J] = -iwm * s_px * 0.5 * D; Pp["WW"][I, J] = -iwm * s_px * 0.5 * D
    Pp["NN"][I, J] = -iwm * s_pr * 0.5 * qR * D; Pp["SS"][I, J] = -iwm * s_pr * 0.5 * qL * D

    return X, Rr, Pp, (bx, br, bp)


def mag_rect_system(ne, nu, Bx, Br, epsr, p: dict):
    """Coefficients of the three field equations after the boundary surgery.

    Interior: Ex (emfieldModule.hpp:2300-2348), Er (:2352-2411), Ephi
    (:2414-2453), stencil convention aP x_P - sum a_k x_k = b.  Boundary codes of
    the rectangle (the reference's own codes): Ex Gauss (code 2, :2464-2471 and
    :2497-2504) at z = 0 and z = L, conductor (code 0, :2536-2538) at r = R; Er
    port excitation (code 7, :2606-2621) on the z = 0 faces with r1 <= r <= r2
    and open (code 1, :2579-2588) on the others, open (code 1, :2630-2645) at
    z = L, Gauss (code 2, :2687-2694) at r = R; Ephi open (code 1, :2720-2729) at
    z = 0, conductor (code 0, :2737-2739 and :2755-2757) at z = L and r = R.  On
    the axis the r-weights of the Ex and Ephi south couplings vanish and the Er
    axis face is not an unknown, so no code is needed there.

    Returns {"x": {name: array}, "r": {...}, "p": {...}, "b": (bx, br, bp), masks}
    with complex (ni+2, nj+2) arrays in the reference's [i][j] order."""
    ni, nj, dx, dr, w = p["ni"], p["nj"], p["dx"], p["dr"], p["omegam"]
    r = p["r"]
    masks = mag_masks(ni, nj)
    X, Rr, Pp, (bx, br, bp) = _mag_interior(ne, nu, Bx, Br, epsr, p, masks)

    def open_R(eps_t):
        c0 = np.sqrt(1.0 / (EPS0 * eps_t * MU0))
        deno = (2.0 * c0) ** 2 + (w * dx) ** 2
        return complex((2.0 * c0) ** 2 - (w * dx) ** 2, -4.0 * c0 * w * dx) / (deno + 1e-100)

    for j in range(1, nj + 1):
        qL = (r[j - 1] + r[j]) / 2.0 / (r[j] + 1e-100)
        qR = (r[j + 1] + r[j]) / 2.0 / (r[j] + 1e-100)
        # Ex, z = 0 (first unknown face i = 2): Gauss
        i = 2
        a = X["W"][i, j]
        X["P"][i, j] -= a
        X["NW"][i, j] += a * dx / dr * qR
        X["SW"][i, j] -= a * dx / dr * qL
        X["W"][i, j] = 0.0
        # Ex, z = L (last unknown face i = ni): Gauss
        i = ni
        a = X["E"][i, j]
        X["P"][i, j] -= a
        X["NE"][i, j] -= a * dx / dr * qR
        X["SE"][i, j] += a * dx / dr * qL
        X["E"][i, j] = 0.0
        # Ephi, z = 0: open; z = L: conductor
        i = 1
        Pp["P"][i, j] -= Pp["W"][i, j] * open_R(epsr[i, j])
        Pp["W"][i, j] = 0.0
        i = ni
        Pp["P"][i, j] += Pp["E"][i, j]
        Pp["E"][i, j] = 0.0
    for j in range(2, nj + 1):
        # Er, z = 0: port excitation on [r1, r2], open elsewhere
        i = 1
        eps_t = (epsr[i, j] + epsr[i, j - 1]) / 2.0
        r_t = (r[j] + r[j - 1]) / 2.0
        if p["r1"] <= r_t <= p["r2"]:
            c0 = np.sqrt(1.0 / (EPS0 * eps_t * MU0))
            deno = complex(2.0 * c0, w * dx)
            Rq = complex(2.0 * c0, -w * dx)
            Er_Fw = p["J1r_exc"] / r_t / np.log(p["r2"] / p["r1"]) * 1e3
            S = complex(0.0, 4.0 * w * dx) * Er_Fw
            Rr["P"][i, j] -= Rr["W"][i, j] * Rq / (deno + 1e-100)
            br[i, j] += Rr["W"][i, j] * S / (deno + 1e-100)
        else:
            Rr["P"][i, j] -= Rr["W"][i, j] * open_R(eps_t)
        Rr["W"][i, j] = 0.0
        # Er, z = L: open
        i = ni
        eps_t = (epsr[i, j] + epsr[i, j - 1]) / 2.0
        Rr["P"][i, j] -= Rr["E"][i, j] * open_R(eps_t)
        Rr["E"][i, j] = 0.0
    for i in range(1, ni + 1):
        j = nj
        rR = (r[j + 1] + r[j]) / 2.0
        rL = (r[j] + r[j - 1]) / 2.0
        # Er, r = R: Gauss
        a = Rr["N"][i, j]
        Rr["P"][i, j] -= a * rL / rR
        Rr["NE"][i, j] -= a * dr / dx * r[j] / rR
        Rr["NW"][i, j] += a * dr / dx * r[j] / rR
        Rr["N"][i, j] = 0.0
        # Ex (i >= 2) and Ephi, r = R: conductor
        if i >= 2:
            X["P"][i, j] += r[j] / r[j + 1] * X["N"][i, j]
            X["N"][i, j] = 0.0
        Pp["P"][i, j] += r[j] / r[j + 1] * Pp["N"][i, j]
        Pp["N"][i, j] = 0.0
    return dict(x=X, r=Rr, p=Pp, b=(bx, br, bp), masks=masks)


# neighbour offsets (di, dj, target component) of each coupling
_NB_X = {"E": (1, 0, 0), "W": (-1, 0, 0), "N": (0, 1, 0), "S": (0, -1, 0),
         "NE": (0, 1, 1), "SE": (0, 0, 1), "NW": (-1, 1, 1), "SW": (-1, 0, 1), "EE": (0, 0, 2), "WW": (-1, 0, 2)}
_NB_R = {"E": (1, 0, 1), "W": (-1, 0, 1), "N": (0, 1, 1), "S": (0, -1, 1),
         "NE": (1, 0, 0), "SE": (1, -1, 0), "NW": (0, 0, 0), "SW": (0, -1, 0), "NN": (0, 0, 2), "SS": (0, -1, 2)}
_NB_P = {"E": (1, 0, 2), "W": (-1, 0, 2), "N": (0, 1, 2), "S": (0, -1, 2),
         "EE": (1, 0, 0), "WW": (0, 0, 0), "NN": (0, 1, 1), "SS": (0, 0, 1)}


def mag_rect_matrix(sysd: dict):
    """Sparse matrix of the three equations (unknown order: Ex, Er, Ephi, each
    row-major over (i, j) as the reference numbers them, :2790-2820), inserting
    only unknown-to-unknown couplings (:2822-2990).  Returns (A csr, b, keys)."""
    import scipy.sparse as sp
    masks = sysd["masks"]
    sh = masks[0].shape
    kmap = []
    off = 0
    for m in masks:
        k = -np.ones(sh, np.int64)
        k[m] = off + np.arange(int(m.sum()))
        kmap.append(k)
        off += int(m.sum())
    rows, cols, vals = [], [], []
    for comp, (coefs, nb) in enumerate(((sysd["x"], _NB_X), (sysd["r"], _NB_R), (sysd["p"], _NB_P))):
        I, J = np.nonzero(masks[comp])
        krow = kmap[comp][I, J]
        rows.append(krow); cols.append(krow); vals.append(coefs["P"][I, J])
        for name, (di, dj, tc) in nb.items():
            kc = kmap[tc][I + di, J + dj]
            ok = kc >= 0
            rows.append(krow[ok]); cols.append(kc[ok]); vals.append(-coefs[name][I, J][ok])
    A = sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))), shape=(off, off))
    b = np.concatenate([sysd["b"][c][masks[c]] for c in range(3)])
    return A, b, kmap


def mag_rect_solve(sysd: dict):
    """Direct sparse solve (SuperLU; the reference factorises with Eigen
    SparseLU, :2995-2998).  Returns Ex, Er, Ephi as (ni+2, nj+2) complex arrays."""
    import scipy.sparse.linalg as spl
    A, b, _ = mag_rect_matrix(sysd)
    x = spl.splu(A.tocsc()).solve(b)
    return mag_unpack(sysd, x)


def mag_unpack(sysd: dict, x):
    masks = sysd["masks"]
    out, off = [], 0
    for m in masks:
        f = np.zeros(m.shape, complex)
        n = int(m.sum())
        f[m] = x[off:off + n]
        out.append(f)
        off += n
    return tuple(out)


def mag_pack(sysd: dict, fields):
    return np.concatenate([fields[c][sysd["masks"][c]] for c in range(3)])


# ---------------------------------------------------------------------------
# the magnetised system on the reference's cathode geometry: six blocks per
# field (initialModule.hpp:219-345; block 5 is the coax feed) and the boundary
# lists of InitialModule::makeBoundary (initialModule.hpp:420-1055), read from
# the segment table tests/golden/mw_lists_cathode.json
# ---------------------------------------------------------------------------
def cathode_mw_params(ni: int = 194, nj: int = 70, xR: float = 0.0388, rmax: float = 0.014,
                      omegam: float = 2.67e10, J1r_exc: float = 0.212687) -> dict:
    """Grid and microwave parameters of the cathode geometry; r1, r2 as
    makeBoundary sets them (initialModule.hpp:217-218); rmin = 0."""
    dx, dr = xR / ni, rmax / nj
    return dict(ni=ni, nj=nj, dx=dx, dr=dr, xR=xR, rmax=rmax, omegam=omegam, J1r_exc=J1r_exc, r1=0.6e-3,
                r2=2.0e-3, masse=9.10938356e-31, x=(np.arange(ni + 2) - 0.5) * dx, r=(np.arange(nj + 2) - 0.5) * dr)


def cathode_mw_blocks(p: dict):
    """(cells, x-faces, r-faces): each a pair (i_bl, j_bl) of 6 blocks
    (initialModule.hpp:219-345 with the feed block 5)."""
    dx, dr, xR, rmax = p["dx"], p["dr"], p["xR"], p["rmax"]
    x1, x2, x3, x4, x5, x6 = 0.0, 5.6e-3 + 7.8e-3, 10.0e-3 + 7.8e-3, 15.0e-3 + 7.8e-3, 20.0e-3 + 7.8e-3, 7.8e-3
    r1, r2, r3, r4, r5 = 0.6e-3, 2.0e-3, 4.0e-3, 9.0e-3, 2.0e-3
    lo = lambda v, d, k: int(v / d + 0.5) + k
    hi = lambda v, d, k: int(v / d - 0.5) + k
    ci = [[lo(x6, dx, 1), hi(x2, dx, 1)], [lo(x2, dx, 1), hi(x4, dx, 1)], [lo(x2, dx, 1), hi(x3, dx, 1)],
          [lo(x3, dx, 1), hi(x5, dx, 1)], [lo(x5, dx, 1), hi(xR, dx, 1)], [lo(x1, dx, 1), hi(x2, dx, 1)]]
    cj = [[lo(r3, dr, 1), hi(r4, dr, 1)], [lo(r5, dr, 1), hi(r4, dr, 1)], [lo(r1, dr, 1), hi(r5, dr, 1)],
          [lo(0.0, dr, 1), hi(r5, dr, 1)], [lo(0.0, dr, 1), hi(rmax, dr, 1)], [lo(r1, dr, 1), hi(r2, dr, 1)]]
    xi = [[lo(x6, dx, 2), hi(x2, dx, 2)], [lo(x2, dx, 2), hi(x4, dx, 1)], [lo(x2, dx, 2), hi(x3, dx, 2)],
          [lo(x3, dx, 2), hi(x5, dx, 2)], [lo(x5, dx, 2), hi(xR, dx, 1)], [lo(x1, dx, 2), hi(x2, dx, 2)]]
    xj = cj
    ri = ci
    rj = [[lo(r3, dr, 2), hi(r4, dr, 1)], [lo(r5, dr, 1), hi(r4, dr, 1)], [lo(r1, dr, 2), hi(r5, dr, 1)],
          [lo(0.0, dr, 2), hi(r5, dr, 1)], [lo(0.0, dr, 2), hi(rmax, dr, 1)], [lo(r1, dr, 2), hi(r2, dr, 1)]]
    a = lambda v: np.array(v, np.int32)
    return (a(ci), a(cj)), (a(xi), a(xj)), (a(ri), a(rj))


def block_mask(ni: int, nj: int, ib, jb) -> np.ndarray:
    m = np.zeros((ni + 2, nj + 2), bool)
    for (a, b), (c, d) in zip(ib, jb):
        m[a:b + 1, c:d + 1] = True
    return m


def cathode_mw_lists(cells, table: dict) -> dict:
    """The 12 boundary lists {(field, side): [(i, j, code), ...]} in the
    reference's order, evaluated from the segment table on the cell blocks."""
    blocks = {"ic": cells[0], "jc": cells[1]}
    form = re.compile(r"([ij]c)\[(\d)\]\[([01])\]([+-]\d+)?")

    def ev(e: str) -> int:  # the table's one form: ic[b][k] or jc[b][k], plus or minus a constant
        m = form.fullmatch(e)
        if not m:
            raise ValueError(f"unexpected bound expression: {e}")
        return int(blocks[m.group(1)][int(m.group(2))][int(m.group(3))]) + int(m.group(4) or 0)

    out = {(f, sd): [] for f in "xrp" for sd in "WESN"}
    for sg in table["segments"]:
        key = (sg["field"], sg["side"])
        if sg["kind"] == "point":
            out[key].append((ev(sg["i"]), ev(sg["j"]), sg["code"]))
        else:
            fix = ev(sg["fix"])
            for v in range(ev(sg["lo"]), ev(sg["hi"]) + 1):
                out[key].append((fix, v, sg["code"]) if sg["var"] == "j" else (v, fix, sg["code"]))
    return out


def mag_system_lists(ne, nu, Bx, Br, epsr, p: dict, masks, lists: dict, jflc00: int):
    """The three field equations on the given unknowns with the boundary surgery
    of solve_Microwave applied list by list in the reference's order (Ex, Er,
    Ephi; sides W, E, S, N; emfieldModule.hpp:2456-2784).  jflc00 is
    gc.j_flc_bl[0][0], which the Er code 3 on the south side compares with r
    (a radius against an index: the reference's special case at :2672)."""
    dx, dr, w = p["dx"], p["dr"], p["omegam"]
    r, J1 = p["r"], p["J1r_exc"]
    X, Rr, Pp, (bx, br, bp) = _mag_interior(ne, nu, Bx, Br, epsr, p, masks)

    def c0_of(e):
        return np.sqrt(1.0 / (EPS0 * e * MU0))

    def open_x(e):  # code 1 along z (:2579-2588, :2720-2729), normalised
        c0 = c0_of(e)
        deno = (2.0 * c0) ** 2 + (w * dx) ** 2
        return complex((2.0 * c0) ** 2 - (w * dx) ** 2, -4.0 * c0 * w * dx) / (deno + 1e-100)

    def open_r(e, j):  # code 1 along r (:2553-2566, :2771-2782)
        c0 = c0_of(e)
        rt = (r[j + 1] + r[j]) / 2.0
        qL, qR = r[j] / (rt + 1e-100), r[j + 1] / (rt + 1e-100)
        deno = (2.0 * c0 * np.sqrt(qR)) ** 2 + (w * dr * qR) ** 2
        R = complex((2.0 * c0) ** 2 * np.sqrt(qL * qR) - (w * dr) ** 2 * qL * qR,
                    -2.0 * c0 * w * dr * (qL * np.sqrt(qR) + qR * np.sqrt(qL)))
        return R / (deno + 1e-100)

    for i, j, c in lists[("x", "W")]:  # :2458-2489
        qL = (r[j - 1] + r[j]) / 2.0 / (r[j] + 1e-100); qR = (r[j + 1] + r[j]) / 2.0 / (r[j] + 1e-100)
        a = X["W"][i, j]
        if c == 0:
            X["W"][i, j] = 0.0
        elif c == 2:
            X["P"][i, j] -= a; X["NW"][i, j] += a * dx / dr * qR; X["SW"][i, j] -= a * dx / dr * qL; X["W"][i, j] = 0.0
        elif c == 3:
            deno = 1.0 + dx / dr * qL
            X["P"][i, j] -= a / deno; X["NW"][i, j] += a * (dx / dr * qR) / deno; X["W"][i, j] = 0.0
        elif c == 4:
            deno = 1.0 + dx / dr * qR
            X["P"][i, j] -= a / deno; X["SW"][i, j] -= a * (dx / dr * qL) / deno; X["W"][i, j] = 0.0
    for i, j, c in lists[("x", "E")]:  # :2491-2514
        qL = (r[j - 1] + r[j]) / 2.0 / (r[j] + 1e-100); qR = (r[j + 1] + r[j]) / 2.0 / (r[j] + 1e-100)
        a = X["E"][i, j]
        if c == 0:
            X["E"][i, j] = 0.0
        elif c == 2:
            X["P"][i, j] -= a; X["NE"][i, j] -= a * dx / dr * qR; X["SE"][i, j] += a * dx / dr * qL; X["E"][i, j] = 0.0
        elif c == 4:
            deno = 1.0 + dx / dr * qR
            X["P"][i, j] -= a / deno; X["SE"][i, j] += a * (dx / dr * qL) / deno; X["E"][i, j] = 0.0
    for i, j, c in lists[("x", "S")]:  # :2516-2531
        a = X["S"][i, j]
        if c == 0:
            X["P"][i, j] += r[j] / r[j - 1] * a; X["S"][i, j] = 0.0
        elif c == 6:
            rR, rL = (r[j + 1] + r[j]) / 2.0, (r[j] + r[j - 1]) / 2.0
            X["P"][i, j] -= a * (dr / dx * r[j] / rL); X["W"][i, j] += a * (-dr / dx * r[j] / rL)
            X["NW"][i, j] += a * (rR / rL); X["S"][i, j] = 0.0
    for i, j, c in lists[("x", "N")]:  # :2533-2571
        a = X["N"][i, j]
        rR, rL = (r[j + 1] + r[j]) / 2.0, (r[j] + r[j - 1]) / 2.0
        if c == 0:
            X["P"][i, j] += r[j] / r[j + 1] * a; X["N"][i, j] = 0.0
        elif c == 1:
            X["P"][i, j] -= a * open_r((epsr[i, j] + epsr[i - 1, j]) / 2.0, j); X["N"][i, j] = 0.0
        elif c == 5:
            X["P"][i, j] -= a * (dr / dx * r[j] / rR); X["E"][i, j] += a * (-dr / dx * r[j] / rR)
            X["SE"][i, j] += a * (rL / rR); X["N"][i, j] = 0.0
        elif c == 6:
            X["P"][i, j] -= a * (dr / dx * r[j] / rR); X["W"][i, j] += a * (-dr / dx * r[j] / rR)
            X["SW"][i, j] += a * (-rL / rR); X["N"][i, j] = 0.0
    for i, j, c in lists[("r", "W")]:  # :2574-2622
        a = Rr["W"][i, j]
        eps_t = (epsr[i, j] + epsr[i, j - 1]) / 2.0
        if c == 0:
            Rr["P"][i, j] += a; Rr["W"][i, j] = 0.0
        elif c == 1:
            Rr["P"][i, j] -= a * open_x(eps_t); Rr["W"][i, j] = 0.0
        elif c == 5:
            rR, rL = (r[j + 1] + r[j]) / 2.0, (r[j] + r[j - 1]) / 2.0
            Rr["P"][i, j] -= a * (dx / dr * rL / r[j]); Rr["N"][i, j] += a * (-dx / dr * rR / r[j])
            Rr["NE"][i, j] += a * (-1.0); Rr["W"][i, j] = 0.0
        elif c == 6:
            rR, rL = (r[j] + r[j - 1]) / 2.0, (r[j - 1] + r[j - 2]) / 2.0
            Rr["P"][i, j] -= a * (dx / dr * rR / r[j - 1]); Rr["S"][i, j] += a * (-dx / dr * rL / r[j - 1])
            Rr["SE"][i, j] += a * 1.0; Rr["W"][i, j] = 0.0
        elif c == 7:
            c0 = c0_of(eps_t)
            deno, Rq = complex(2.0 * c0, w * dx), complex(2.0 * c0, -w * dx)
            rt = (r[j] + r[j - 1]) / 2.0
            S = complex(0.0, 4.0 * w * dx) * (J1 / rt / np.log(p["r2"] / p["r1"]) * 1e3)
            Rr["P"][i, j] -= a * Rq / (deno + 1e-100); br[i, j] += a * S / (deno + 1e-100); Rr["W"][i, j] = 0.0
    for i, j, c in lists[("r", "E")]:  # :2624-2656
        a = Rr["E"][i, j]
        eps_t = (epsr[i, j] + epsr[i, j - 1]) / 2.0
        if c == 0:
            Rr["P"][i, j] += a; Rr["E"][i, j] = 0.0
        elif c == 1:
            c0 = c0_of(eps_t)
            deno = (2.0 * c0) ** 2 + (w * dx) ** 2
            R = complex((2.0 * c0) ** 2 - (w * dx) ** 2, -4.0 * c0 * w * dx)
            Rr["P"][i, j] -= a * R / (deno + 1e-100); Rr["E"][i, j] = 0.0
        elif c == 5:
            rR, rL = (r[j + 1] + r[j]) / 2.0, (r[j] + r[j - 1]) / 2.0
            Rr["P"][i, j] -= a * (dx / dr * rL / r[j]); Rr["N"][i, j] += a * (-dx / dr * rR / r[j])
            Rr["NW"][i, j] += a * 1.0; Rr["E"][i, j] = 0.0
    for i, j, c in lists[("r", "S")]:  # :2658-2681
        a = Rr["S"][i, j]
        rR, rL = (r[j] + r[j - 1]) / 2.0, (r[j - 1] + r[j - 2]) / 2.0
        if c == 2:
            Rr["P"][i, j] -= a * rR / rL; Rr["SE"][i, j] += a * dr / dx * r[j - 1] / rL
            Rr["SW"][i, j] -= a * dr / dx * r[j - 1] / rL; Rr["S"][i, j] = 0.0
        elif c == 3:
            deno = dr / dx * r[j - 1] / rL
            if r[j] < jflc00:
                deno = 1.0
            Rr["P"][i, j] -= a * rR / rL / deno; Rr["NE"][i, j] += a * dr / dx * r[j - 1] / rL / deno
            Rr["S"][i, j] = 0.0
    for i, j, c in lists[("r", "N")]:  # :2683-2711
        a = Rr["N"][i, j]
        rR, rL = (r[j + 1] + r[j]) / 2.0, (r[j] + r[j - 1]) / 2.0
        if c == 2:
            Rr["P"][i, j] -= a * rL / rR; Rr["NE"][i, j] -= a * dr / dx * r[j] / rR
            Rr["NW"][i, j] += a * dr / dx * r[j] / rR; Rr["N"][i, j] = 0.0
        elif c == 3:
            deno = dr / dx * r[j] / rR
            Rr["P"][i, j] -= a * rL / rR / deno; Rr["SE"][i, j] -= a * dr / dx * r[j] / rR / deno; Rr["N"][i, j] = 0.0
        elif c == 4:
            deno = dr / dx * r[j] / rR
            Rr["P"][i, j] -= a * rL / rR / deno; Rr["SW"][i, j] += a * dr / dx * r[j] / rR / deno; Rr["N"][i, j] = 0.0
    for i, j, c in lists[("p", "W")]:  # :2713-2730
        a = Pp["W"][i, j]
        if c == 0:
            Pp["P"][i, j] += a; Pp["W"][i, j] = 0.0
        elif c == 1:
            Pp["P"][i, j] -= a * open_x(epsr[i, j]); Pp["W"][i, j] = 0.0
    for i, j, c in lists[("p", "E")]:  # :2731-2739
        if c == 0:
            Pp["P"][i, j] += Pp["E"][i, j]; Pp["E"][i, j] = 0.0
    for i, j, c in lists[("p", "S")]:  # :2741-2749
        if c == 0:
            Pp["P"][i, j] += r[j] / r[j - 1] * Pp["S"][i, j]; Pp["S"][i, j] = 0.0
    for i, j, c in lists[("p", "N")]:  # :2751-2784
        a = Pp["N"][i, j]
        if c == 0:
            Pp["P"][i, j] += r[j] / r[j + 1] * a; Pp["N"][i, j] = 0.0
        elif c == 1:
            Pp["P"][i, j] -= a * open_r(epsr[i, j], j); Pp["N"][i, j] = 0.0
    return dict(x=X, r=Rr, p=Pp, b=(bx, br, bp), masks=masks)


def rect_mw_lists(ni: int, nj: int, p: dict) -> dict:
    """The rectangle's boundary rules (those of mag_rect_system) as the
    reference's 12 lists: Ex Gauss (2) at z = 0, L and conductor (0) at r = R;
    Er port (7) on the z = 0 faces with r1 <= r <= r2, open (1) on the other
    z = 0 faces and at z = L, Gauss (2) at r = R; Ephi open (1) at z = 0,
    conductor (0) at z = L and r = R."""
    r = p["r"]
    L = {(f, sd): [] for f in "xrp" for sd in "WESN"}
    for j in range(1, nj + 1):
        L[("x", "W")].append((2, j, 2))
        L[("x", "E")].append((ni, j, 2))
        L[("p", "W")].append((1, j, 1))
        L[("p", "E")].append((ni, j, 0))
    for j in range(2, nj + 1):
        rt = (r[j] + r[j - 1]) / 2.0
        L[("r", "W")].append((1, j, 7 if p["r1"] <= rt <= p["r2"] else 1))
        L[("r", "E")].append((ni, j, 1))
    for i in range(1, ni + 1):
        L[("r", "N")].append((i, nj, 2))
        if i >= 2:
            L[("x", "N")].append((i, nj, 0))
        L[("p", "N")].append((i, nj, 0))
    return L


# which ghost each (list, code) writes: (di, dj) from the entry, per field/side
_GHOST = {("x", "W"): ((-1, 0), (0, 2, 3, 4)), ("x", "E"): ((1, 0), (0, 2, 4)), ("x", "S"): ((0, -1), (0,)),
          ("x", "N"): ((0, 1), (0, 1)), ("r", "W"): ((-1, 0), (0, 1, 7)), ("r", "E"): ((1, 0), (0, 1)),
          ("r", "S"): ((0, -1), (2, 3)), ("r", "N"): ((0, 1), (2, 3, 4)), ("p", "W"): ((-1, 0), (0, 1)),
          ("p", "E"): ((1, 0), tuple(range(8))), ("p", "S"): ((0, -1), tuple(range(8))),
          ("p", "N"): ((0, 1), (0, 1))}


def ghost_targets(lists: dict):
    """{field: set of (i, j)} the ghost pass writes."""
    out = {f: set() for f in "xrp"}
    for (f, sd), ent in lists.items():
        (di, dj), codes = _GHOST[(f, sd)]
        for i, j, c in ent:
            if c in codes:
                out[f].add((i + di, j + dj))
    return out


def mag_ghosts(E, Er_dc, epsr, p: dict, lists: dict, jflc00: int):
    """The boundary post-processing of solve_Microwave
    (emfieldModule.hpp:3026-3260): ghost values of E1x, E1r, E1p written from
    the solution list by list in the reference's order.  E = (Ex, Er, Ep) full
    (ni+2, nj+2) complex arrays (solution on the unknowns, earlier ghosts
    elsewhere); returns new arrays.  Er_dc is the real field gr.Er, which the
    Er east code 1 reads (:3162), dividing by its deno twice, as there."""
    Ex, Er, Ep = (np.array(e, dtype=complex) for e in E)
    dx, dr, w, r = p["dx"], p["dr"], p["omegam"], p["r"]

    def c0_of(e):
        return np.sqrt(1.0 / (EPS0 * e * MU0))

    def open_x(e):
        c0 = c0_of(e)
        deno = (2.0 * c0) ** 2 + (w * dx) ** 2
        return complex((2.0 * c0) ** 2 - (w * dx) ** 2, -4.0 * c0 * w * dx) / (deno + 1e-100)

    def open_r(e, j):
        c0 = c0_of(e)
        rt = (r[j + 1] + r[j]) / 2.0
        qL, qR = r[j] / (rt + 1e-100), r[j + 1] / (rt + 1e-100)
        deno = (2.0 * c0 * np.sqrt(qR)) ** 2 + (w * dr * qR) ** 2
        R = complex((2.0 * c0) ** 2 * np.sqrt(qL * qR) - (w * dr) ** 2 * qL * qR,
                    -2.0 * c0 * w * dr * (qL * np.sqrt(qR) + qR * np.sqrt(qL)))
        return R / (deno + 1e-100)

    for i, j, c in lists[("x", "W")]:  # :3028-3053
        qL = (r[j - 1] + r[j]) / 2.0 / (r[j] + 1e-100); qR = (r[j + 1] + r[j]) / 2.0 / (r[j] + 1e-100)
        if c == 0:
            Ex[i - 1, j] = 0.0
        elif c == 2:
            Ex[i - 1, j] = Ex[i, j] + dx / dr * (qR * Er[i - 1, j + 1] - qL * Er[i - 1, j])
        elif c == 3:
            deno = 1.0 + dx / dr * qL
            Ex[i - 1, j] = Ex[i, j] / deno + dx / dr * (qR * Er[i - 1, j + 1]) / deno
        elif c == 4:
            deno = 1.0 + dx / dr * qR
            Ex[i - 1, j] = Ex[i, j] / deno - dx / dr * (qL * Er[i - 1, j]) / deno
    for i, j, c in lists[("x", "E")]:  # :3054-3073
        qL = (r[j - 1] + r[j]) / 2.0 / (r[j] + 1e-100); qR = (r[j + 1] + r[j]) / 2.0 / (r[j] + 1e-100)
        if c == 0:
            Ex[i + 1, j] = 0.0
        elif c == 2:
            Ex[i + 1, j] = Ex[i, j] - dx / dr * (qR * Er[i, j + 1] - qL * Er[i, j])
        elif c == 4:
            deno = 1.0 + dx / dr * qR
            Ex[i + 1, j] = Ex[i, j] / deno + dx / dr * qL * Er[i, j] / deno
    for i, j, c in lists[("x", "S")]:  # :3074-3083
        if c == 0:
            Ex[i, j - 1] = -r[j] / r[j - 1] * Ex[i, j]
    for i, j, c in lists[("x", "N")]:  # :3084-3107
        if c == 0:
            Ex[i, j + 1] = -r[j] / r[j + 1] * Ex[i, j]
        elif c == 1:
            Ex[i, j + 1] = open_r((epsr[i, j] + epsr[i - 1, j]) / 2.0, j) * Ex[i, j]
    for i, j, c in lists[("r", "W")]:  # :3109-3143
        eps_t = (epsr[i, j] + epsr[i, j - 1]) / 2.0
        if c == 0:
            Er[i - 1, j] = -Er[i, j]
        elif c == 1:
            Er[i - 1, j] = open_x(eps_t) * Er[i, j]
        elif c == 7:
            c0 = c0_of(eps_t)
            deno, Rq = complex(2.0 * c0, w * dx), complex(2.0 * c0, -w * dx)
            rt = (r[j] + r[j - 1]) / 2.0
            S = complex(0.0, 4.0 * w * dx) * (p["J1r_exc"] / rt / np.log(p["r2"] / p["r1"]) * 1e3)
            Er[i - 1, j] = Rq / (deno + 1e-100) * Er[i, j] + S / (deno + 1e-100)
    for i, j, c in lists[("r", "E")]:  # :3144-3166
        if c == 0:
            Er[i + 1, j] = -Er[i, j]
        elif c == 1:
            eps_t = (epsr[i, j] + epsr[i, j - 1]) / 2.0
            c0 = c0_of(eps_t)
            deno = (2.0 * c0) ** 2 + (w * dx) ** 2
            R = complex((2.0 * c0) ** 2 - (w * dx) ** 2, -4.0 * c0 * w * dx) / (deno + 1e-100)
            Er[i + 1, j] = R / (deno + 1e-100) * Er_dc[i, j]
    for i, j, c in lists[("r", "S")]:  # :3167-3187
        rR, rL = (r[j] + r[j - 1]) / 2.0, (r[j - 1] + r[j - 2]) / 2.0
        if c == 2:
            Er[i, j - 1] = rR / rL * Er[i, j] + dr / dx * r[j - 1] / rL * (Ex[i + 1, j - 1] - Ex[i, j - 1])
        elif c == 3:
            deno = dr / dx * r[j - 1] / rL
            if r[j] < jflc00:
                deno = 1.0
            Er[i, j - 1] = rR / rL * Er[i, j] / deno + dr / dx * r[j - 1] / rL * (Ex[i + 1, j - 1]) / deno
    for i, j, c in lists[("r", "N")]:  # :3188-3212
        rR, rL = (r[j + 1] + r[j]) / 2.0, (r[j] + r[j - 1]) / 2.0
        if c == 2:
            Er[i, j + 1] = rL / rR * Er[i, j] - dr / dx * r[j] / rR * (Ex[i + 1, j] - Ex[i, j])
        elif c == 3:
            deno = dr / dx * r[j] / rR
            Er[i, j + 1] = rL / rR * Er[i, j] / deno - dr / dx * r[j] / rR * (Ex[i + 1, j]) / deno
        elif c == 4:
            deno = dr / dx * r[j] / rR
            Er[i, j + 1] = rL / rR * Er[i, j] / deno + dr / dx * r[j] / rR * (Ex[i, j]) / deno
    for i, j, c in lists[("p", "W")]:  # :3213-3229
        if c == 0:
            Ep[i - 1, j] = -Ep[i, j]
        elif c == 1:
            Ep[i - 1, j] = open_x(epsr[i, j]) * Ep[i, j]
    for i, j, c in lists[("p", "E")]:  # :3230-3236, every code
        Ep[i + 1, j] = -Ep[i, j]
    for i, j, c in lists[("p", "S")]:  # :3237-3243, every code
        Ep[i, j - 1] = -r[j] / r[j - 1] * Ep[i, j]
    for i, j, c in lists[("p", "N")]:  # :3244-3264
        if c == 0:
            Ep[i, j + 1] = -r[j] / r[j + 1] * Ep[i, j]
        elif c == 1:
            Ep[i, j + 1] = open_r(epsr[i, j], j) * Ep[i, j]
    return Ex, Er, Ep


def mw_loss_rR(j, i0, i1, E1x, E1r, E1p, r, dx, dr, w):
    """mWLoss_at_boundary_rR (emfieldModule.hpp:8631-8664): the Poynting flux
    through the upper faces of row j, columns i0..i1."""
    P = 0.0
    iwm = complex(0.0, 1.0 / (w * MU0))
    for i in range(i0, i1 + 1):
        rt = (r[j] + r[j + 1]) / 2.0
        dRdx_L = (E1r[i, j + 1] - E1r[i - 1, j + 1]) / dx
        dXdr_L = (E1x[i, j + 1] - E1x[i, j]) / dr
        dRdx_R = (E1r[i + 1, j + 1] - E1r[i, j + 1]) / dx
        dXdr_R = (E1x[i + 1, j + 1] - E1x[i + 1, j]) / dr
        H1p = (iwm * (dRdx_R - dXdr_R) + iwm * (dRdx_L - dXdr_L)) / 2.0
        H1x = iwm * ((r[j + 1] * E1p[i, j + 1] - r[j] * E1p[i, j]) / (rt * dr))
        Ep = (r[j + 1] * E1p[i, j + 1] + r[j] * E1p[i, j]) / (2.0 * rt)
        Ex_L = (r[j + 1] * E1x[i, j + 1] + r[j] * E1x[i, j]) / (2.0 * rt)
        Ex_R = (r[j + 1] * E1x[i + 1, j + 1] + r[j] * E1x[i + 1, j]) / (2.0 * rt)
        Ex = (Ex_R + Ex_L) / 2.0
        S = 0.5 * (Ep * np.conj(H1x) - Ex * np.conj(H1p)).real
        P += 2.0 * np.pi * rt * S * dx
    return P


def mw_port_rescale(E1x, E1r, E1p, J, Jexc, Pabs, power_sum, p: dict):
    """The port / reflection / rescale part of update_energy_profile
    (emfieldModule.hpp:7792-8105).  p: dx, dr, rmin, omegam, r1, r2, Z0, Pmw,
    S11, S21, S12, S22 (complex), flag_mwRef, i_ref, j_out, i_out0, i_out1,
    jf0, jf1.  Returns (planes, result): planes = dict of the rescaled arrays
    (E1x, E1r, E1p, J1x, J1r, J1p, the excitation planes, Pabs), result = the
    reported quantities after the reference's rescaling."""
    dx, dr, w = p["dx"], p["dr"], p["omegam"]
    nj2 = E1x.shape[1]
    r = p["rmin"] + (np.arange(nj2) - 0.5) * dr
    out = dict(E1x=E1x.copy(), E1r=E1r.copy(), E1p=E1p.copy(), J1x=J[0].copy(), J1r=J[1].copy(), J1p=J[2].copy(),
               Pabs=Pabs.copy())
    for k, v in zip(("J1x_exc", "J1r_exc", "J1p_exc"), Jexc or (None,) * 3):
        if v is not None:
            out[k] = v.copy()
    if not p["flag_mwRef"]:  # :8073-8095
        ratio = p["Pmw"] / power_sum
        out["Pabs"] = out["Pabs"] * ratio
        return out, dict(ratio=ratio, pabs_factor=ratio, field_factor=1.0, J1r_exc_factor=np.sqrt(ratio),
                         power_sum=power_sum)
    P_out = mw_loss_rR(p["j_out"], p["i_out0"], p["i_out1"], E1x, E1r, E1p, r, dx, dr, w)  # :7848-7849
    i = p["i_ref"]
    I = 0.0j
    V = 0.0j
    n = 0
    for j in range(p["jf0"], p["jf1"] + 1):  # :7866-7920
        rt = (r[j] + r[j - 1]) / 2.0
        H = (E1r[i, j] - E1r[i - 1, j]) / dx / (w * MU0) * 1j
        I = I + 2.0 * np.pi * rt * H
        V = V + (E1r[i, j] + E1r[i - 1, j]) / 2.0 * rt
        n += 1
    I_ref = I / n
    V_ref = V / n * np.log(p["r2"] / p["r1"])
    Z0 = p["Z0"]
    a2 = (V_ref - Z0 * I_ref) / (2.0 * np.sqrt(2.0 * Z0))  # :7930-7935
    b2 = (V_ref + Z0 * I_ref) / (2.0 * np.sqrt(2.0 * Z0))
    P_fwd, P_ref = abs(b2) ** 2, abs(a2) ** 2
    P_err = P_fwd - P_ref - power_sum - P_out
    a1 = (b2 - p["S22"] * a2) / p["S21"]
    b1 = p["S11"] * a1 + p["S12"] * a2
    P_fwd_all, P_ref_all = abs(a1) ** 2, abs(b1) ** 2
    ratio = p["Pmw"] / P_fwd_all  # :7988
    ratio_eff = ratio * (power_sum + P_err) / power_sum
    out["Pabs"] = out["Pabs"] * ratio_eff  # :7993-8015
    for k in ("E1x", "E1r", "E1p", "J1x", "J1r", "J1p", "J1x_exc", "J1r_exc", "J1p_exc"):
        if k in out:
            out[k] = out[k] * np.sqrt(ratio_eff)
    Gp, Ga = a2 / b2, b1 / a1
    res = dict(P_out=P_out * ratio, P_fwd=P_fwd * ratio, P_ref=P_ref * ratio, P_fwd_all=P_fwd_all * ratio,
               P_ref_all=P_ref_all * ratio, P_err=P_err * ratio, power_sum=(power_sum + P_err) * ratio,
               ratio=ratio, pabs_factor=ratio_eff, field_factor=np.sqrt(ratio_eff), J1r_exc_factor=np.sqrt(ratio),
               I_ref=I_ref, V_ref=V_ref, Gamma_p=Gp, Zp=Z0 * (1.0 + Gp) / (1.0 - Gp), Gamma_all=Ga,
               Zall=Z0 * (1.0 + Ga) / (1.0 - Ga))
    return out, res


def divergence(E1x, E1r, E1p, J1x, J1r, J1p, p: dict, mask):
    """output_phase's representative field and divE, divJ, div(E+J) columns
    (outputModule.hpp:43-105), loop by loop; mask = gc.jdgBnd_Ep (the six cell
    blocks).  Returns (divE, divJ, divEJ) as (ni+2, nj+2) arrays and Emag_rep."""
    ni, nj = E1x.shape[0] - 2, E1x.shape[1] - 2
    dx, dr, w = p["dx"], p["dr"], p["omegam"]
    r = p.get("rmin", 0.0) + (np.arange(nj + 2) - 0.5) * dr
    tot, n = 0.0, 0
    for i in range(1, ni + 1):
        for j in range(1, nj + 1):
            rL = (r[j - 1] + r[j]) / 2.0
            rR = (r[j + 1] + r[j]) / 2.0
            ex = (E1x[i, j] + E1x[i + 1, j]) / 2.0
            er = (rR * E1r[i, j + 1] + rL * E1r[i, j]) / (2.0 * r[j])
            tot += abs(ex) ** 2 + abs(er) ** 2 + abs(E1p[i, j]) ** 2
            n += 1
    rep = np.sqrt(tot / n)
    out = [np.zeros(E1x.shape, complex) for _ in range(3)]
    for i in range(1, ni + 1):
        for j in range(1, nj + 1):
            if not mask[i, j]:
                continue
            rL = (r[j - 1] + r[j]) / 2.0
            rR = (r[j + 1] + r[j]) / 2.0
            dE = (rR * E1r[i, j + 1] - rL * E1r[i, j]) / (dr * r[j]) + (E1x[i + 1, j] - E1x[i, j]) / dx
            dJ = (rR * J1r[i, j + 1] - rL * J1r[i, j]) / (dr * r[j]) + (J1x[i + 1, j] - J1x[i, j]) / dx
            divE = dE * (dx / rep)
            divJ = dJ * (dx / (rep * w * EPS0))
            out[0][i, j] = divE
            out[1][i, j] = divJ
            out[2][i, j] = (divJ + 1j * w * EPS0 * divE) * (dx / (rep * w * EPS0))
    return out[0], out[1], out[2], rep

