"""Seeded synthetic inputs in the reference's shapes.

The reference ships no benchmark data; these generators build the inputs of
the measured workloads from fixed seeds, in the reference's array convention
((ni+2) x (nj+2) float64 arrays indexed [i][j], i = axial z, j = radial r,
cell centres x_i = xL + (i-0.5) dx, r_j = rmin + (j-0.5) dr as in
initialModule.hpp:77-84).

``poisson_slab`` is the isolated 512x1024 r-z potential system: the
reference's 5-point Poisson stencil (fluidModule.hpp:2693-2703: x faces
weighted dr^2, r faces weighted q dx^2 with q = r_face / r_cell) with a
face permittivity taking the place of the dielectric-relaxation factor,
Dirichlet electrodes by ghost reflection (fluidModule.hpp:2156-2240: ghost
= -phi at 0 V, ghost = 2 V - phi at the biased electrode) and the axis
handled by q = 0 at r = 0.
"""
from __future__ import annotations

import numpy as np

E0 = 1.60217662e-19  # constants.hpp:6
EPS0 = 8.8541878128e-12  # constants.hpp:7
MU0 = 1.2566370614e-6  # constants.hpp:8
BOLTZ = 1.380649e-23  # constants.hpp:5


def grid(ni: int, nj: int, Lz: float = 10e-3, Lr: float = 5e-3):
    dx = Lz / ni
    dr = Lr / nj
    x = (np.arange(ni + 2) - 0.5) * dx
    r = (np.arange(nj + 2) - 0.5) * dr
    return dx, dr, x, r


def poisson_slab(ni: int = 1024, nj: int = 512, seed: int = 1, V_bias: float = 20.0,
                 epsr_slab: float = 3.8, slab=(2e-3, 3e-3)) -> dict:
    """Isolated potential system on the 10 mm (z) x 5 mm (r) rectangle.

    Permittivity eps0, except epsr_slab*eps0 for slab[0] <= z <= slab[1];
    face values are harmonic means of the two cells.  Space charge
    rho = e (n_i - n_e) with n_e log-uniform in [1e15, 1e18] m^-3 and
    n_i = n_e (1 + 0.01 N(0,1)), both drawn from default_rng(seed) in that
    order, each as an (ni, nj) interior array.
    Boundaries: z = 0 at 0 V, z = L at V_bias, r = R at 0 V (ghost
    reflection), r = 0 axis (q = 0).  Returns the reference's solver inputs
    aP, aE, aW, aN, aS, b (shape (ni+2, nj+2)) plus the one-block table.
    """
    dx, dr, x, r = grid(ni, nj)
    rng = np.random.default_rng(seed)
    ne = np.zeros((ni + 2, nj + 2))
    nion = np.zeros((ni + 2, nj + 2))
    ne[1:-1, 1:-1] = 10.0 ** rng.uniform(15.0, 18.0, size=(ni, nj))
    nion[1:-1, 1:-1] = ne[1:-1, 1:-1] * (1.0 + 0.01 * rng.standard_normal(size=(ni, nj)))
    eps = np.full((ni + 2, nj + 2), EPS0)
    in_slab = (x >= slab[0]) & (x <= slab[1])
    eps[in_slab, :] = epsr_slab * EPS0

    def hm(a, b):
        return 2.0 * a * b / (a + b)

    I = slice(1, ni + 1)
    J = slice(1, nj + 1)
    rc = r[J][None, :]
    rR = 0.5 * (r[1:nj + 1] + r[2:nj + 2])[None, :]
    rL = 0.5 * (r[1:nj + 1] + r[0:nj])[None, :]
    qR = rR / rc
    qL = rL / rc
    eRx = hm(eps[I, J], eps[2:ni + 2, J])
    eLx = hm(eps[I, J], eps[0:ni, J])
    eRr = hm(eps[I, J], eps[I, 2:nj + 2])
    eLr = hm(eps[I, J], eps[I, 0:nj])

    shape = (ni + 2, nj + 2)
    aE = np.zeros(shape); aW = np.zeros(shape); aN = np.zeros(shape); aS = np.zeros(shape)
    aP = np.zeros(shape); b = np.zeros(shape)
    aE[I, J] = eRx * dr * dr
    aW[I, J] = eLx * dr * dr
    aN[I, J] = qR * eRr * dx * dx
    aS[I, J] = qL * eLr * dx * dx
    aP[I, J] = aE[I, J] + aW[I, J] + aN[I, J] + aS[I, J]
    b[I, J] = E0 * (nion[I, J] - ne[I, J]) * dx * dx * dr * dr

    # z = 0 electrode (0 V): ghost = -phi
    aP[1, J] += aW[1, J]
    aW[1, J] = 0.0
    # z = L electrode (V_bias): ghost = 2 V - phi
    aP[ni, J] += aE[ni, J]
    b[ni, J] += 2.0 * V_bias * aE[ni, J]
    aE[ni, J] = 0.0
    # r = R wall (0 V): ghost = -phi
    aP[I, nj] += aN[I, nj]
    aN[I, nj] = 0.0
    # r = 0 axis: qL = 0 already makes aS vanish at j = 1
    aS[I, 1] = 0.0

    return dict(ni=ni, nj=nj, dx=dx, dr=dr,
                i_bl=np.array([[1, ni]], dtype=np.int32), j_bl=np.array([[1, nj]], dtype=np.int32),
                aP=aP, aE=aE, aW=aW, aN=aN, aS=aS, b=b)


def random_mmatrix(ni: int, nj: int, seed: int = 0, diag_extra: float = 0.0, blocks=None,
                   aniso: float = 1.0, jump: float = 1.0) -> dict:
    """Random variable-coefficient 5-point M-matrix system for solver tests.

    Face conductances are log-uniform over [1, jump] (both directions share
    each face, so the operator is symmetric), the x faces are scaled by
    ``aniso``, and ``diag_extra`` adds a time-derivative-like diagonal term.
    Couplings across the outer boundary are folded as Dirichlet walls
    (aP += a_nb, a_nb = 0).  ``blocks`` defaults to one block covering the
    interior.
    """
    rng = np.random.default_rng(seed)
    shape = (ni + 2, nj + 2)
    cx = np.exp(rng.uniform(0.0, np.log(jump), size=(ni + 1, nj))) * aniso  # x faces i-1/2 .. ni+1/2
    cr = np.exp(rng.uniform(0.0, np.log(jump), size=(ni, nj + 1)))  # r faces
    aE = np.zeros(shape); aW = np.zeros(shape); aN = np.zeros(shape); aS = np.zeros(shape)
    aW[1:-1, 1:-1] = cx[:-1, :]
    aE[1:-1, 1:-1] = cx[1:, :]
    aS[1:-1, 1:-1] = cr[:, :-1]
    aN[1:-1, 1:-1] = cr[:, 1:]
    aP = np.zeros(shape)
    aP[1:-1, 1:-1] = aE[1:-1, 1:-1] + aW[1:-1, 1:-1] + aN[1:-1, 1:-1] + aS[1:-1, 1:-1] + diag_extra
    b = np.zeros(shape)
    b[1:-1, 1:-1] = rng.standard_normal(size=(ni, nj))
    if blocks is None:
        i_bl = np.array([[1, ni]], dtype=np.int32)
        j_bl = np.array([[1, nj]], dtype=np.int32)
    else:
        i_bl = np.asarray(blocks[0], dtype=np.int32)
        j_bl = np.asarray(blocks[1], dtype=np.int32)
    return dict(ni=ni, nj=nj, i_bl=i_bl, j_bl=j_bl, aP=aP, aE=aE, aW=aW, aN=aN, aS=aS, b=b)


def mw_er_rect(ni: int = 1024, nj: int = 512, seed: int = 2, omegam: float = 2.67e10) -> dict:
    """Isolated microwave Er system on the 10 mm (z) x 5 mm (r) rectangle.

    Cold-plasma medium: n_e log-uniform in [1e15, 1e18] m^-3 and the collision
    frequency nu log-uniform in [1e8, 1e10] s^-1, drawn from default_rng(seed) in
    that order as (ni+2, nj+2) cell arrays; epsr = 1; w = 2.67e10 rad/s; port
    radii of the cathode's coax feed r1 = 0.6 mm, r2 = 2.0 mm.  The Er unknowns are
    the r-faces i = 1..ni, j = 2..nj (block i_bl = [1, ni], j_bl = [2, nj]).
    """
    rng = np.random.default_rng(seed)
    ne = 10.0 ** rng.uniform(15.0, 18.0, size=(ni + 2, nj + 2))
    nu = 10.0 ** rng.uniform(8.0, 10.0, size=(ni + 2, nj + 2))
    epsr = np.ones((ni + 2, nj + 2))
    dx, dr, x, r = grid(ni, nj)
    params = dict(dx=dx, dr=dr, rmin=0.0, omegam=omegam, J1r_exc=0.212687, r1=0.6e-3, r2=2.0e-3,
                  masse=9.10938356e-31)
    return dict(ni=ni, nj=nj, ne=ne, nu=nu, epsr=epsr, params=params,
                i_bl=np.array([[1, ni]], dtype=np.int32), j_bl=np.array([[2, nj]], dtype=np.int32))


def mw3_rect(ni: int = 1024, nj: int = 512, seed: int = 2, omegam: float = 2.67e10, bmax: float = 0.05) -> dict:
    """Magnetised microwave system on the 10 mm (z) x 5 mm (r) rectangle.

    n_e, nu and epsr as mw_er_rect (same generator and draws), plus the field of
    a magnet near the port: Bx = bmax exp(-((z - 2 mm) / 3 mm)^2) and
    Br = -(r / 2) dBx/dz (divergence-free to first order in r), on the cell
    centres.  bmax = 0.05 T puts the electron cyclotron frequency at a third of
    w = 2.67e10 rad/s.
    """
    w = mw_er_rect(ni, nj, seed=seed, omegam=omegam)
    dx, dr, x, r = grid(ni, nj)
    z0, wz = 2.0e-3, 3.0e-3
    X, R = np.meshgrid(x, r, indexing="ij")
    g = np.exp(-((X - z0) / wz) ** 2)
    w["Bx"] = bmax * g
    w["Br"] = -(R / 2.0) * bmax * g * (-2.0 * (X - z0) / wz ** 2)
    return w


MASSE = 9.10938356e-31               # params.hpp:34
MASSI_XE = 131.293e-3 / 6.02214076e23  # params.hpp:35


def plasma_state(ni: int, nj: int, seed: int = 3, dr: float | None = None) -> dict:
    """Seeded fluid state in the reference's field names and shapes.

    Cell fields (ni+2, nj+2): rhoe log-uniform in [1e15, 1e19] m^-3, rhoi =
    rhoe (1 + 0.01 N(0,1)), rhon log-uniform in [1e20, 1e22], rhom = 1e-3 rhon,
    Te uniform in [0.5, 20] eV (in K) with 1 % of the cells in [150, 250] eV
    (past the end of the rate tables), Bx, Br N(0, 0.05) T, nu_ano log-uniform
    in [1e6, 1e8] s^-1, nu_ano_IAT = 0, Uip N(0, 100) m/s; face fields Uix, Uir
    N(0, 100) m/s with 10 % of the faces N(0, 3000), rhoUex, rhoUer = rhoe N(0, 1e5).
    Transport parameters: the xenon discharge of params.hpp:34-83 (Ti = 300 K,
    nu_eff = 1e9 s^-1) with the Bohm and Sagdeev terms switched on.
    """
    rng = np.random.default_rng(seed)
    sh = (ni + 2, nj + 2)
    f = {}
    f["rhoe"] = 10.0 ** rng.uniform(15.0, 19.0, sh)
    f["rhoi"] = f["rhoe"] * (1.0 + 0.01 * rng.standard_normal(sh))
    f["rhon"] = 10.0 ** rng.uniform(20.0, 22.0, sh)
    f["rhom"] = 1e-3 * f["rhon"]
    te_ev = rng.uniform(0.5, 20.0, sh)
    hot = rng.random(sh) < 0.01
    te_ev[hot] = rng.uniform(150.0, 250.0, hot.sum())
    f["Te"] = te_ev * E0 / BOLTZ
    f["Bx"] = 0.05 * rng.standard_normal(sh)
    f["Br"] = 0.05 * rng.standard_normal(sh)
    f["nu_ano"] = 10.0 ** rng.uniform(6.0, 8.0, sh)
    f["nu_ano_IAT"] = np.zeros(sh)
    f["Uip"] = 100.0 * rng.standard_normal(sh)
    for k in ("Uix", "Uir"):
        u = 100.0 * rng.standard_normal(sh)
        fast = rng.random(sh) < 0.1
        u[fast] = 3000.0 * rng.standard_normal(fast.sum())
        f[k] = u
    f["rhoUex"] = f["rhoe"] * 1e5 * rng.standard_normal(sh)
    f["rhoUer"] = f["rhoe"] * 1e5 * rng.standard_normal(sh)
    prm = dict(masse=MASSE, massi=MASSI_XE, Ti=300.0, nu_eff=1e9, flag_Bohm=1, flag_Sagdeev=1,
               dr=dr if dr is not None else 5e-3 / nj, rmin=0.0)
    return dict(fields=f, prm=prm)


def pc_state(ni: int, nj: int, seed: int = 4, Lz: float = 10e-3, Lr: float = 5e-3) -> dict:
    """Seeded state of the potential predictor-corrector in the reference's names.

    rhoe = 1e17 P x lognormal(0, 0.1) + 1e14 m^-3 with the profile
    P = exp(-((z - Lz/2)^2 + r^2) / (2 (Lr/5)^2)); rhoi, rhoe_old = rhoe (1 + 0.01 N(0,1));
    Te = (1 + 4 P)(1 + 0.01 N(0,1)) eV (in K); phi = 20 z / Lz + 0.01 N(0,1) V with
    Ex, Er its face differences (+ 1 % noise); nUex, nUer = rhoe 1e3 N(0,1);
    Uix, Uir N(0, 1000) m/s; rhoUmx, rhoUmr 1e19 N(0,1);
    rate_ionize = rhoe 1e5 U(0,1); mobility tensor of B ~ N(0, 0.05) T and a
    momentum frequency log-uniform in [1e8, 1e10] s^-1 (fluidModule.hpp:5957-5973).
    Physics parameters: dt 1e-10 s, V_bias 20 V, SEE coefficients 0.08 (params.hpp:62-63),
    the inner solve of the shipped setup (SMG, 30 iterations, 1e-10) and 2 PC iterations
    with calcRes mode 3 (input/setup.yaml)."""
    rng = np.random.default_rng(seed)
    sh = (ni + 2, nj + 2)
    dx, dr = Lz / ni, Lr / nj
    z = (np.arange(ni + 2) - 0.5) * dx
    r = (np.arange(nj + 2) - 0.5) * dr
    sig = Lr / 5.0
    prof = np.exp(-(((z[:, None] - Lz / 2) ** 2) + r[None, :] ** 2) / (2 * sig * sig))
    f = {}
    f["rhoe"] = 1e17 * prof * np.exp(0.1 * rng.standard_normal(sh)) + 1e14
    f["rhoi"] = f["rhoe"] * (1.0 + 0.01 * rng.standard_normal(sh))
    f["rhoe_old"] = f["rhoe"] * (1.0 + 0.01 * rng.standard_normal(sh))
    f["Te"] = (1.0 + 4.0 * prof) * (1.0 + 0.01 * rng.standard_normal(sh)) * E0 / BOLTZ
    phi = 20.0 * z[:, None] / Lz + 0.01 * rng.standard_normal(sh)
    f["phi"] = phi
    Ex = np.zeros(sh)
    Er = np.zeros(sh)
    Ex[1:, :] = -(phi[1:, :] - phi[:-1, :]) / dx
    Er[:, 1:] = -(phi[:, 1:] - phi[:, :-1]) / dr
    f["Ex"] = Ex * (1.0 + 0.01 * rng.standard_normal(sh))
    f["Er"] = Er * (1.0 + 0.01 * rng.standard_normal(sh))
    f["nUex"] = f["rhoe"] * 1e3 * rng.standard_normal(sh)
    f["nUer"] = f["rhoe"] * 1e3 * rng.standard_normal(sh)
    f["Uix"] = 1000.0 * rng.standard_normal(sh)
    f["Uir"] = 1000.0 * rng.standard_normal(sh)
    f["rhoUmx"] = 1e19 * rng.standard_normal(sh)
    f["rhoUmr"] = 1e19 * rng.standard_normal(sh)
    f["rate_ionize"] = f["rhoe"] * 1e5 * rng.random(sh)
    Bx = 0.05 * rng.standard_normal(sh)
    Br = 0.05 * rng.standard_normal(sh)
    nu_m = 10.0 ** rng.uniform(8.0, 10.0, sh)
    mu_para = E0 / (MASSE * nu_m + 1e-100)
    Om = E0 * np.sqrt(Bx * Bx + Br * Br) / (MASSE * nu_m + 1e-100)
    Omx = E0 * Bx / (MASSE * nu_m + 1e-100)
    Omr = E0 * Br / (MASSE * nu_m + 1e-100)
    deno = 1.0 + Om * Om
    f["mu_para"] = mu_para
    f["mu_xx"] = mu_para * (1.0 + Omx * Omx) / deno
    f["mu_rr"] = mu_para * (1.0 + Omr * Omr) / deno
    f["mu_xr"] = mu_para * (Omx * Omr) / deno
    f["mu_perp"] = mu_para / deno
    prm = dict(dt=1e-10, dx=dx, dr=dr, rmin=0.0, V_bias=20.0, masse=MASSE, coefIISEE_ts=0.08,
               coefMISEE_ts=0.08, error_cnv_HES_phi=1e-21, error_cnv_SOR_phi=1e-10, maxITR_HES_phi=2,
               maxITR_SOR_phi=30, flag_error=3, flag_iter_phi=1, precision=1)
    return dict(fields=f, prm=prm)


def sg_state(ni: int, nj: int, seed: int = 6, Lz: float = 10e-3, Lr: float = 5e-3) -> dict:
    """pc_state extended with the arrays of the electron density and energy sweeps:
    rhoeps = 3/2 rhoe k Te, Gx, Gr = rhoeps 1e3 N(0,1), rhoUex, rhoUer = rhoe 1e3 N(0,1),
    rhoUix_wall = rhoi 1e3 N(0,1), Pabs U(0, 1e8) W/m^3, rate_eloss U(0, 8e-10) J/s,
    zero wall-flux arrays.  Parameters: the electron sweeps of input/setup.yaml
    (SMG, 30 iterations, 1e-10; 2 PC iterations; calcRes mode 3), Te_emitSEE 2.5 eV,
    ratioEngy_EISEE_rd 0.5 (params.hpp:64-65), dt 1e-10 s."""
    st = pc_state(ni, nj, seed=seed, Lz=Lz, Lr=Lr)
    f = st["fields"]
    rng = np.random.default_rng(seed + 1000)
    sh = f["rhoe"].shape
    f["rhoeps"] = 1.5 * f["rhoe"] * BOLTZ * f["Te"]
    f["Gx"] = f["rhoeps"] * 1e3 * rng.standard_normal(sh)
    f["Gr"] = f["rhoeps"] * 1e3 * rng.standard_normal(sh)
    f["rhoUex"] = f["rhoe"] * 1e3 * rng.standard_normal(sh)
    f["rhoUer"] = f["rhoe"] * 1e3 * rng.standard_normal(sh)
    f["rhoUix_wall"] = f["rhoi"] * 1e3 * rng.standard_normal(sh)
    f["Pabs"] = rng.uniform(0.0, 1e8, sh)
    f["rate_eloss"] = rng.uniform(0.0, 8e-10, sh)
    for k in ("rhoUex_wall", "rhoUer_wall", "Gx_wall", "Gr_wall"):
        f[k] = np.zeros(sh)
    p = st["prm"]
    prm = dict(dt=p["dt"], dx=p["dx"], dr=p["dr"], rmin=p["rmin"], masse=MASSE, coefIISEE_ts=0.08,
               coefMISEE_ts=0.08, Te_emitSEE_eV=2.5, ratioEngy_EISEE_rd=0.5, error_cnv_HES=1e-21,
               error_cnv_SOR=1e-10, maxITR_HES=2, maxITR_SOR=30, flag_error=3, flag_iter=1, precision=1)
    return dict(fields=f, prm=prm)


def ion_state(ni: int, nj: int, seed: int = 7, Lz: float = 10e-3, Lr: float = 5e-3) -> dict:
    """pc_state extended with the ion arrays: Uix, Uir N(0, 300) m/s, Uip N(0, 100) m/s,
    nui_m log-uniform in [1e4, 1e6] s^-1, zero ion fluxes.  Parameters of the shipped
    setup (input/setup.yaml): Ti 300 K, Te_rep 0.1 eV, SMG 30 iterations to 1e-10,
    ndt_i 1, calcRes mode 3, CFL 1; dt 1e-10 s, rmax = Lr."""
    st = pc_state(ni, nj, seed=seed, Lz=Lz, Lr=Lr)
    f = st["fields"]
    rng = np.random.default_rng(seed + 2000)
    sh = f["rhoe"].shape
    f["Uix"] = 300.0 * rng.standard_normal(sh)
    f["Uir"] = 300.0 * rng.standard_normal(sh)
    f["Uip"] = 100.0 * rng.standard_normal(sh)
    f["nui_m"] = 10.0 ** rng.uniform(4.0, 6.0, sh)
    f["Bx"] = 0.05 * rng.standard_normal(sh)
    f["Br"] = 0.05 * rng.standard_normal(sh)
    for k in ("rhoUix", "rhoUir", "rhoUix_wall", "rhoUir_wall"):
        f[k] = np.zeros(sh)
    p = st["prm"]
    prm = dict(dt=p["dt"], dx=p["dx"], dr=p["dr"], rmin=0.0, rmax=Lr, massi=MASSI_XE, Ti=300.0, V_bias=20.0,
               Te_rep_eV=0.1, CFL=1.0, error_cnv_SOR=1e-10, ndt_i=1, maxITR_SOR=30, flag_iter=1, precision=1,
               flag_error=3)
    return dict(fields=f, prm=prm)


def neutral_state(ni: int, nj: int, seed: int = 8, Lz: float = 10e-3, Lr: float = 5e-3) -> dict:
    """Seeded state of the neutral sweeps: rhon = 1e21 (1 + 0.1 U(0,1)) m^-3, rhom =
    1e17 lognormal(0, 0.2), face fluxes N(0, 1e19), ion and metastable wall fluxes
    N(0, 1e18), rhoe = 1e17 lognormal(0, 0.3), collision frequencies log-uniform in
    [1e5, 1e7] s^-1.  Parameters: Tn 300 K, Xe radius 216 pm, DmN 5.2e19 (input/setup.yaml),
    the inlet flux of 0.069 mg/s through 2 pi r4 x 5.5 mm (initialModule.hpp:234-237),
    the inner solve of the potential (SMG, 30 iterations, 1e-10), dt 1e-10 s."""
    rng = np.random.default_rng(seed)
    sh = (ni + 2, nj + 2)
    f = {}
    f["rhon"] = 1e21 * (1.0 + 0.1 * rng.random(sh))
    f["rhom"] = 1e17 * np.exp(0.2 * rng.standard_normal(sh))
    for k in ("rhoUnx", "rhoUnr", "rhoUmx", "rhoUmr"):
        f[k] = 1e19 * rng.standard_normal(sh)
    for k in ("rhoUix_wall", "rhoUir_wall", "rhoUmx_wall", "rhoUmr_wall"):
        f[k] = 1e18 * rng.standard_normal(sh)
    for k in ("rhoUnx_wall", "rhoUnr_wall"):
        f[k] = np.zeros(sh)
    f["rhoe"] = 1e17 * np.exp(0.3 * rng.standard_normal(sh))
    for k in ("nu_excStep", "nu_super", "nu_excMeta", "nu_exc", "nu_ionz", "nu_ionzStep"):
        f[k] = 10.0 ** rng.uniform(5.0, 7.0, sh)
    fn_In = 0.069e-6 / MASSI_XE / (2.0 * np.pi * 9.0e-3 * 5.5e-3)
    prm = dict(dt=1e-10, dx=Lz / ni, dr=Lr / nj, rmin=0.0, fn_In=fn_In, Tn=300.0, ri=216.0e-12, massi=MASSI_XE,
               DmN=5.2e19, error_cnv_SOR=1e-10, ndt_n=1, ndt_m=1, maxITR_SOR=30, flag_iter=1, precision=1,
               flag_error=3)
    return dict(fields=f, prm=prm)


RATE_TABLES = ("nu_elas_N", "nu_exc_N", "nu_excReso_N", "nu_excMeta_N", "nu_ionz_N", "nu_ionzStep_N",
               "nu_excStep_N", "nu_super_N", "rate_eloss_n_N", "rate_eloss_m_N", "nui_m_N")


def synthetic_rate_tables(n_e: int = 1801, n_i: int = 39, d_eps_eV: float = 0.1, d_ei_eV: float = 0.001):
    """Rate tables of the synthetic xenon discharge on the reference's uniform
    mean-energy grid (inputModule.hpp:1413-1655; Te = 2/3 mean energy): ionisation
    k = 1e-13 Te^0.5 exp(-12.13/Te) m^3/s with its 12.13 eV loss, elastic 2e-13 m^3/s,
    ion momentum transfer 5.2e-16 m^3/s.  Returns (tables, dTe [K], dEi [J])."""
    eps = np.arange(n_e) * d_eps_eV
    Te = 2.0 / 3.0 * eps
    kion = np.zeros(n_e)
    pos = Te > 0
    kion[pos] = 1e-13 * np.sqrt(Te[pos]) * np.exp(-12.13 / Te[pos])
    tb = {k: np.zeros(n_e) for k in RATE_TABLES if k != "nui_m_N"}
    tb["nu_elas_N"] = np.full(n_e, 2e-13)
    tb["nu_ionz_N"] = kion
    tb["rate_eloss_n_N"] = kion * 12.13 * E0
    tb["nui_m_N"] = np.full(n_i, 5.2e-16)
    return tb, d_eps_eV * 2.0 / 3.0 * E0 / BOLTZ, d_ei_eV * E0


def discharge_state(ni: int, nj: int, Lz: float = 10e-3, Lr: float = 5e-3, seed: int = 0) -> dict:
    """Initial state of the synthetic xenon discharge on the r-z rectangle: ne = ni =
    1e17 exp(-((z - Lz/2)^2 + r^2) / (2 (1 mm)^2)) x lognormal(0, 0.1) from
    default_rng(seed), floor 1e12 m^-3; neutrals 1e20 m^-3; Te 5 eV;
    cusp field Bz = 0.25 T cos(pi z/Lz) e^(-r/2 mm), Br = 0.25 T sin(pi z/Lz) e^(-r/2 mm)
    sampled on the (ni+1) x (nj+1) cell corners and averaged to the cells; zero
    potential, fields, fluxes and velocities."""
    rng = np.random.default_rng(seed)
    sh = (ni + 2, nj + 2)
    dx, dr = Lz / ni, Lr / nj
    z = (np.arange(ni + 2) - 0.5) * dx
    r = (np.arange(nj + 2) - 0.5) * dr
    sig = 1e-3
    ne = 1e17 * np.exp(-(((z[:, None] - Lz / 2) ** 2) + r[None, :] ** 2) / (2 * sig * sig))
    ne = np.maximum(ne * np.exp(0.1 * rng.standard_normal(sh)), 1e12)
    zn = np.arange(ni + 1) * dx
    rn = np.arange(nj + 1) * dr
    Bz_n = 0.25 * np.cos(np.pi * zn[:, None] / Lz) * np.exp(-rn[None, :] / 2e-3)
    Br_n = 0.25 * np.sin(np.pi * zn[:, None] / Lz) * np.exp(-rn[None, :] / 2e-3)
    Bx = np.zeros(sh)
    Br = np.zeros(sh)
    Bx[1:-1, 1:-1] = (Bz_n[:-1, :-1] + Bz_n[1:, :-1] + Bz_n[:-1, 1:] + Bz_n[1:, 1:]) / 4.0
    Br[1:-1, 1:-1] = (Br_n[:-1, :-1] + Br_n[1:, :-1] + Br_n[:-1, 1:] + Br_n[1:, 1:]) / 4.0
    Te = np.full(sh, 5.0 * E0 / BOLTZ)
    f = dict(rhoe=ne.copy(), rhoi=ne.copy(), rhon=np.full(sh, 1e20), rhom=np.zeros(sh), Te=Te, Bx=Bx, Br=Br,
             rhoeps=1.5 * ne * BOLTZ * Te)
    return dict(fields=f, dx=dx, dr=dr)


def discharge_params(geo: dict, dr: float, rmax: float) -> dict:
    """Parameter blocks of one predictor-corrector time step of the synthetic
    discharge with the solver settings of input/setup.yaml (SMG, 30 iterations,
    1e-10 relative residual; 2 PC iterations; calcRes mode 3), dt 1e-10 s, bias 20 V,
    Ti 0.05 eV, ion-induced SEE yield 0.05 and no electron-induced SEE, neutral inlet
    flux of 0.069 mg/s through 2 pi r4 x 5.5 mm (initialModule.hpp:234-237)."""
    dx = geo["dx"]
    tb, dTe, dEi = synthetic_rate_tables()
    Ti = 0.05 * E0 / BOLTZ
    solve = dict(error_cnv_SOR=1e-10, maxITR_SOR=30, flag_iter=1, precision=1)
    p = dict(
        itime=0, ndt_i=1, ndt_n=1, ndt_m=1, flag_adp_dt=0, dt=1e-10, CFL=1.0, gtime=0.0,
        pos_boxes=list(geo.get("pos_boxes", [])),
        ion=dict(dt=1e-10, dx=dx, dr=dr, rmin=0.0, rmax=rmax, massi=MASSI_XE, Ti=Ti, V_bias=20.0, Te_rep_eV=0.1,
                 CFL=1.0, ndt_i=1, flag_error=3, **solve),
        phi=dict(dt=1e-10, dx=dx, dr=dr, rmin=0.0, V_bias=20.0, masse=MASSE, coefIISEE_ts=0.05, coefMISEE_ts=0.05,
                 dTe_SEE=0.5 * E0 / BOLTZ, error_cnv_HES_phi=1e-21, error_cnv_SOR_phi=1e-10, maxITR_HES_phi=2,
                 maxITR_SOR_phi=30, flag_error=3, flag_iter_phi=1, precision=1),
        rhoe=dict(dt=1e-10, dx=dx, dr=dr, rmin=0.0, masse=MASSE, coefIISEE_ts=0.05, coefMISEE_ts=0.05,
                  dTe_SEE=0.5 * E0 / BOLTZ, Te_emitSEE_eV=2.5, ratioEngy_EISEE_rd=0.5, error_cnv_HES=1e-21,
                  maxITR_HES=2, flag_error=3, **solve),
        neutral=dict(dt=1e-10, dx=dx, dr=dr, rmin=0.0, fn_In=0.069e-6 / MASSI_XE / (2.0 * np.pi * 9.0e-3 * 5.5e-3),
                     Tn=300.0, ri=216.0e-12, massi=MASSI_XE, DmN=5.2e19, ndt_n=1, ndt_m=1, flag_error=3,
                     do_rhon=1, do_rhom=1, **solve),
        transport=dict(masse=MASSE, massi=MASSI_XE, Ti=Ti, nu_eff=1e9, dTe=dTe, dEi=dEi, dr=dr, rmin=0.0,
                       flag_Bohm=0, flag_Sagdeev=0))
    p["eps"] = dict(p["rhoe"])
    return dict(params=p, tables=tb, see=dict(coefEISEE_eb_table=np.zeros(201), coefEISEE_rd_table=np.zeros(201),
                                               coefEISEE_ts_table=np.zeros(201)))


def mw3_cathode(ni: int = 194, nj: int = 70, seed: int = 2, omegam: float = 2.67e10, bmax: float = 0.05,
                xR: float = 0.0388, rmax: float = 0.014) -> dict:
    """Magnetised microwave system on the cathode geometry (38.8 mm x 14 mm,
    six blocks per field with the coax feed).

    n_e log-uniform in [1e15, 1e18] m^-3 and nu log-uniform in [1e8, 1e10] s^-1,
    drawn from default_rng(seed) in that order as (ni+2, nj+2) cell arrays;
    epsr = 1; a magnet field Bx = bmax exp(-((z - 20 mm) / 8 mm)^2) with
    Br = -(r / 2) dBx/dz on the cell centres."""
    rng = np.random.default_rng(seed)
    ne = 10.0 ** rng.uniform(15.0, 18.0, size=(ni + 2, nj + 2))
    nu = 10.0 ** rng.uniform(8.0, 10.0, size=(ni + 2, nj + 2))
    epsr = np.ones((ni + 2, nj + 2))
    dx, dr, x, r = grid(ni, nj, xR, rmax)
    z0, wz = 20.0e-3, 8.0e-3
    X, R = np.meshgrid(x, r, indexing="ij")
    g = np.exp(-((X - z0) / wz) ** 2)
    params = dict(dx=dx, dr=dr, rmin=0.0, omegam=omegam, J1r_exc=0.212687, r1=0.6e-3, r2=2.0e-3,
                  masse=9.10938356e-31)
    return dict(ni=ni, nj=nj, ne=ne, nu=nu, epsr=epsr, Bx=bmax * g, Br=-(R / 2.0) * bmax * g * (-2.0 * (X - z0) / wz ** 2),
                params=params, xR=xR, rmax=rmax)
