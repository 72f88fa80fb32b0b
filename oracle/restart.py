"""Restart files of the reference: writer and reader restated.

TEST INFRASTRUCTURE ONLY (the checker of the device writer and reader).

write(): the restart<nOut>.csv of OutputModule::output (outputModule.hpp:429-470).
read():  InputModule::input_restart_data (inputModule.hpp:667-1157) on the
cathode geometry: the registered variables, then its post-processing loop by
loop over the named wall segments.
"""
from __future__ import annotations

import numpy as np

BOLTZ = 1.380649e-23
E0 = 1.60217662e-19

# outputModule.hpp:436, the field columns between r and zero
COLUMNS = ("rhoi", "rhoi_old", "Uix", "Uix_old", "Uir", "Uir_old", "Uip", "Uip_old", "rhoe", "rhoe_old", "rhoUex",
           "rhoUex_old", "rhoUer", "rhoUer_old", "Te", "Te_old", "Gx", "Gx_old", "Gr", "Gr_old", "phi", "phi_old",
           "rhom", "rhom_old", "rhoUmx", "rhoUmr", "rate_ionize", "scx", "scr", "nUex", "nUex_old", "nUer",
           "nUer_old", "rhon", "rhon_old", "rhoUnx", "rhoUnr", "rhoeps", "rhoeps_old", "rhoUix_wall", "rhoUir_wall",
           "rhoUex_wall", "rhoUer_wall", "rhoUmx_wall", "rhoUmr_wall", "rhoUnx_wall", "rhoUnr_wall", "Gx_wall",
           "Gr_wall")
# inputModule.hpp:755-812, the reader's registry (the wall fluxes are not read back)
REGISTRY = COLUMNS[:39]


def _trunc(v):
    return 0.0 if abs(v) < 1e-100 else v


def write(fields: dict, x, r) -> str:
    """The file text; fields are (ni+2, nj+2) arrays [i][j] (missing ones are zero)."""
    ni2, nj2 = len(x), len(r)
    cols = [np.asarray(fields.get(k, np.zeros((ni2, nj2)))) for k in COLUMNS]
    out = ["i,j,x,r," + ",".join(COLUMNS) + ",zero"]
    for i in range(ni2):
        for j in range(nj2):
            vals = []
            for k, a in zip(COLUMNS, cols):
                v = _trunc(float(a[i, j]))
                if k in ("Te", "Te_old"):
                    v = v * BOLTZ / E0
                vals.append("%.17e" % v)
            out.append("%d,%d,%.17e,%.17e," % (i, j, x[i], r[j]) + ",".join(vals) + ",%.17e" % 0.0)
    return "\n".join(out) + "\n"


def read(text: str, state: dict, geo: dict, x, r, dx: float, dr: float, V_bias: float) -> dict:
    """Read a restart text into a copy of ``state`` and apply the reader's
    post-processing on the cathode geometry ``geo`` (oracle.fluid.cathode_geometry:
    blocks ib/jb, x-face blocks fxi/fxj, r-face blocks fri/frj)."""
    lines = text.split("\n")
    head = [h.strip() for h in lines[0].split(",")]
    col = {h: k for k, h in enumerate(head)}
    for need in ("i", "j", "x", "r"):
        if need not in col:
            raise ValueError(f"required column is missing: {need}")
    ni2, nj2 = len(x), len(r)
    s = {k: np.array(v, dtype=np.float64, copy=True) for k, v in state.items()}
    for k in REGISTRY + ("Ex", "Er"):
        s.setdefault(k, np.zeros((ni2, nj2)))
    found = np.zeros((ni2, nj2), bool)
    for L in lines[1:]:
        if not L:
            continue
        f = L.split(",")
        i, j = int(f[col["i"]]), int(f[col["j"]])
        if not (0 <= i < ni2 and 0 <= j < nj2):
            raise ValueError("index out of range")
        if found[i, j]:
            raise ValueError("duplicated cell")
        found[i, j] = True
        xv, rv = float(f[col["x"]]), float(f[col["r"]])
        for a, b in ((x[i], xv), (r[j], rv)):
            if abs(a - b) > 1e-12 + 1e-10 * max(1.0, abs(a), abs(b)):
                raise ValueError("grid coordinate is inconsistent")
        for k in REGISTRY:
            if k in col:
                v = float(f[col[k]])
                if k in ("Te", "Te_old"):
                    v = v * E0 / BOLTZ
                s[k][i, j] = v
    if not found.all():
        raise ValueError("missing cell")
    ib, jb = geo["ib"], geo["jb"]
    phi, Ex, Er = s["phi"], s["Ex"], s["Er"]
    # rhoe masked to the fluid cells (inputModule.hpp:1003-1008)
    fluid_cells = np.zeros((ni2, nj2), bool)
    for (a, b), (c, e) in zip(ib, jb):
        fluid_cells[a:b + 1, c:e + 1] = True
    s["rhoe"] = s["rhoe"] * fluid_cells
    # Ex on the x-face blocks (:1010-1018)
    for (a, b), (c, e) in zip(geo["fxi"], geo["fxj"]):
        for i in range(a, b + 1):
            for j in range(c, e + 1):
                Ex[i, j] = -(phi[i, j] - phi[i - 1, j]) / dx
    # left walls z0, z1, z2, z4 (phi = 0), right walls z3 (0), z5 (V_bias) (:1020-1058)
    for j in range(jb[0][0], jb[0][1] + 1):
        i = ib[0][0]; phi[i - 1, j] = -phi[i, j]; Ex[i, j] = -(phi[i, j] - phi[i - 1, j]) / dx
    for j in range(jb[2][0], jb[0][0]):
        i = ib[2][0]; phi[i - 1, j] = -phi[i, j]; Ex[i, j] = -(phi[i, j] - phi[i - 1, j]) / dx
    for j in range(jb[3][0], jb[2][0]):
        i = ib[3][0]; phi[i - 1, j] = -phi[i, j]; Ex[i, j] = -(phi[i, j] - phi[i - 1, j]) / dx
    for j in range(jb[1][0], jb[4][1] + 1):
        i = ib[4][0]; phi[i - 1, j] = -phi[i, j]; Ex[i, j] = -(phi[i, j] - phi[i - 1, j]) / dx
    for j in range(jb[1][0], jb[1][1] + 1):
        i = ib[1][1]; phi[i + 1, j] = -phi[i, j]; Ex[i + 1, j] = -(phi[i + 1, j] - phi[i, j]) / dx
    for j in range(jb[4][0], jb[4][1] + 1):
        i = ib[4][1]; phi[i + 1, j] = 2.0 * V_bias - phi[i, j]; Ex[i + 1, j] = -(phi[i + 1, j] - phi[i, j]) / dx
    # Er on the r-face blocks (:1060-1068)
    for (a, b), (c, e) in zip(geo["fri"], geo["frj"]):
        for i in range(a, b + 1):
            for j in range(c, e + 1):
                Er[i, j] = -(phi[i, j] - phi[i, j - 1]) / dr
    # lower walls x0, x2; axis x6; upper walls x1, x4; open x5 (:1070-1118)
    for i in range(ib[0][0], ib[0][1] + 1):
        j = jb[0][0]; phi[i, j - 1] = -phi[i, j]; Er[i, j] = -(phi[i, j] - phi[i, j - 1]) / dr
    for i in range(ib[2][0], ib[2][1] + 1):
        j = jb[2][0]; phi[i, j - 1] = -phi[i, j]; Er[i, j] = -(phi[i, j] - phi[i, j - 1]) / dr
    for i in range(ib[3][0], ib[4][1] + 1):
        Er[i, jb[3][0]] = 0.0
    for i in range(ib[0][0], ib[1][1] + 1):
        j = jb[0][1]; phi[i, j + 1] = -phi[i, j]; Er[i, j + 1] = -(phi[i, j + 1] - phi[i, j]) / dr
    for i in range(ib[1][1] + 1, ib[3][1] + 1):
        j = jb[3][1]; phi[i, j + 1] = -phi[i, j]; Er[i, j + 1] = -(phi[i, j + 1] - phi[i, j]) / dr
    for i in range(ib[4][0], ib[4][1] + 1):
        j = jb[4][1]; phi[i, j + 1] = phi[i, j]; Er[i, j + 1] = -(phi[i, j + 1] - phi[i, j]) / dr
    return s
