"""CPU checks of the oracle's magnetised 3-component microwave system
(oracle/microwave.py: mag_rect_system, restating solve_Microwave,
include/emfieldModule.hpp:2249-2998).  No reference fixture exercises the
magnetised system, so these pin the restatement by properties."""
import numpy as np
import pytest


def _case(ni=40, nj=16, bmax=0.05, seed=2):
    from importlib import import_module
    wl = import_module("02_cathode-08_modulerev_b200.workloads")
    from oracle import microwave as mw
    w = wl.mw3_rect(ni, nj, seed=seed, bmax=bmax)
    p = mw.er_rect_params(ni, nj)
    return w, p, mw


def test_b0_decouples_ephi():
    """With B = 0 every Hall coupling vanishes: the Ephi equation has no source
    and no coupling, so Ephi = 0, while Ex and Er stay coupled only through the
    boundary Gauss-law eliminations."""
    w, p, mw = _case()
    s = mw.mag_rect_system(w["ne"], w["nu"], 0 * w["Bx"], 0 * w["Br"], w["epsr"], p)
    for k in ("EE", "WW", "NE", "SE", "NW", "SW"):
        interior = s["x"][k][3:-3, 2:-2]
        assert np.all(interior == 0), k
    Ex, Er, Ep = mw.mag_rect_solve(s)
    assert np.max(np.abs(Ep)) == 0.0
    assert np.max(np.abs(Er)) > 0.0


def test_direct_solution_residual_and_masks():
    w, p, mw = _case()
    s = mw.mag_rect_system(w["ne"], w["nu"], w["Bx"], w["Br"], w["epsr"], p)
    A, b, kmap = mw.mag_rect_matrix(s)
    n = sum(int(m.sum()) for m in s["masks"])
    assert A.shape == (n, n)
    # at most 11 entries per row (the reference reserves 11 per row, :2825)
    assert np.max(np.diff(A.indptr)) <= 11
    E = mw.mag_rect_solve(s)
    x = mw.mag_pack(s, E)
    assert np.linalg.norm(A @ x - b) / np.linalg.norm(b) < 1e-12
    for f, m in zip(E, s["masks"]):
        assert np.all(f[~m] == 0)


def test_hall_couplings_scale_with_field():
    """The Er-Ephi couplings are linear in the Hall factor at weak field."""
    w, p, mw = _case(bmax=1e-4)
    s1 = mw.mag_rect_system(w["ne"], w["nu"], w["Bx"], w["Br"], w["epsr"], p)
    s2 = mw.mag_rect_system(w["ne"], w["nu"], 2 * w["Bx"], 2 * w["Br"], w["epsr"], p)
    a1, a2 = s1["r"]["NN"][2:-2, 3:-2], s2["r"]["NN"][2:-2, 3:-2]
    # second-order terms are of relative size (hall factor)^2 ~ 4e-7 here
    assert np.max(np.abs(a2 - 2 * a1)) <= 1e-5 * np.max(np.abs(a2))
