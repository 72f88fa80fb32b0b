"""Helpers that set up the reference's own FluidModule (oracle/_ref/libref.so, built
from the unmodified reference headers) with the inputs the other tests give the
oracle and the device path: the same fields, the same parameters under the
reference's Params names, the same tables, on the reference's cathode geometry
as its InitialModule::makeBoundary builds it."""
from __future__ import annotations

import numpy as np

# the package's per-sweep settings use generic names; Params has one set per equation
GENERIC = ("error_cnv_SOR", "maxITR_SOR", "flag_iter", "error_cnv_HES", "maxITR_HES")
SUFFIX = {"ion": ("_Ui", "_rhoi"), "rhoe": ("_rhoe",), "eps": ("_rhoeps",),
          # update_rhon / update_rhom take the potential's solver settings (fluidModule.hpp:5129-5131, :5574-5576)
          "neutral": ()}


def expand(prm: dict, block: str | None) -> dict:
    out = {}
    for k, v in prm.items():
        if k in GENERIC:
            for s in SUFFIX.get(block, ()):
                out[k + s] = v
        else:
            out[k] = v
    return out


def case(ni=194, nj=70, xR=0.0388, rmax=0.014, width_neutIn=0.0055, dropin=False):
    """A reference case on the cathode geometry at ni x nj (makeBoundary run); with
    dropin=True its linear solves run on the GPU through include/cathode_solver.hpp."""
    from oracle import ref
    c = ref.RefCase(ni, nj, dropin=dropin)
    for k, v in dict(xR=xR, rmax=rmax, width_neutIn=width_neutIn).items():
        assert c.set_param(k, v), k
    c.make_boundary()
    return c


def put(c, prm: dict, block: str | None = None) -> None:
    """Scalar parameters of one sweep's dict (keys outside Params are ignored: precision, do_rhon, ...)."""
    c.set_params({k: v for k, v in expand(prm, block).items()
                  if isinstance(v, (int, float, np.integer, np.floating)) and not isinstance(v, bool)})


def put_see(c, see) -> None:
    eb, rd, ts = see[:3]
    c.set_table("coefEISEE_eb_table", eb)
    c.set_table("coefEISEE_rd_table", rd)
    c.set_table("coefEISEE_ts_table", ts)


def put_step(c, st: dict, cfg: dict) -> None:
    """Fields, parameter blocks and tables of a whole-step test (workloads.discharge_params)."""
    P = cfg["params"]
    put(c, P["transport"])
    put(c, P["neutral"], "neutral")
    put(c, P["ion"], "ion")
    put(c, P["phi"])
    put(c, P["rhoe"], "rhoe")
    put(c, P["eps"], "eps")
    for k in ("itime", "ndt_i", "ndt_n", "ndt_m", "flag_adp_dt", "dt", "CFL", "gtime"):
        assert c.set_param(k, P[k]), k
    c.set_param("flag_PC", 1)
    c.set_param("flag_inertia", 0)
    c.set_fields(st)
    for k, v in cfg["tables"].items():
        c.set_table(k, v)
    for k, v in cfg["see"].items():
        c.set_table(k, v)


def emag(Ex, Er, r):
    """Cell-centred |E| of the face fields as the reference's result output forms it
    (outputModule.hpp:310-311)."""
    Exc = (Ex[:-1, :] + Ex[1:, :]) / 2.0
    rL = (r[1:-1] + r[:-2]) / 2.0
    rR = (r[1:-1] + r[2:]) / 2.0
    Erc = (rL[None, :] * Er[:, 1:-1] + rR[None, :] * Er[:, 2:]) / (2.0 * r[None, 1:-1])
    out = np.zeros_like(Ex)
    out[:-1, 1:-1] = np.sqrt(Exc[:, 1:-1] ** 2 + Erc[:-1, :] ** 2)
    return out


def rel_l2(a, b, mask) -> float:
    """||a - b||_2 / ||b||_2 over the cells where mask is set."""
    d = (a - b)[mask]
    n = np.linalg.norm(b[mask])
    return float(np.linalg.norm(d) / (n if n > 0 else 1.0))


def fluid_mask(c) -> np.ndarray:
    """The reference's fluid cells (gc.jdgBnd_flc: blocks 0..4, initialModule.hpp:347-353)."""
    return c.int_field("jdgBnd_flc") == 1
