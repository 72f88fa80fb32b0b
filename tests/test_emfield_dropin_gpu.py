"""The header-only drop-in for the reference's microwave update
(include/cathode_emfield.hpp: EmfieldModule::solve_Microwave and
update_energy_profile, emfieldModule.hpp:74, :79) compiled against the
reference's own Params / GridCenter / GridInterfaceX / GridInterfaceR /
MicrowaveBC types and run on boundary lists made by the reference's own
InitialModule::makeBoundary (oracle/_ref/libref_dropin.so), on the cathode at
194 x 70: the fields after the solve and ghost pass, then the absorbed power,
currents and the port rescale (flag_mwRef = 1), against the oracle's direct
solve and its restatement of the energy profile and port part."""
import numpy as np
import pytest

import refpin

pytestmark = pytest.mark.gpu
NI, NJ = 194, 70


@pytest.fixture(scope="module")
def ref():
    from oracle import ref as R
    if not R.available(dropin=True):
        pytest.skip("oracle/_ref/libref_dropin.so not built (it is built from the reference sources)")
    return R


def _rel(a, b):
    return float(np.abs(a - b).max() / (np.abs(b).max() + 1e-300))


def _lists(c):
    return {(f, s): [tuple(int(v) for v in row) for row in c.mw_list(f"Bnd{s}{f}")] for f in "xrp" for s in "WESN"}


def test_microwave_update_through_the_dropin(pkg, cuda_device, ref):
    from oracle import microwave as omw
    w = pkg.workloads.mw3_cathode(NI, NJ, seed=2, bmax=0.05)
    c = refpin.case(NI, NJ, dropin=True)
    c.set_param("omegam", w["params"]["omegam"])
    for k in ("dx", "dr", "omegam", "J1r_exc", "r1", "r2", "masse"):
        assert c.param(k) == pytest.approx(w["params"][k], rel=1e-15), k
    for k, v in (("rhoe", "ne"), ("nu_m1", "nu"), ("Bx", "Bx"), ("Br", "Br"), ("epsr", "epsr")):
        c.set_field(k, w[v])
    rng = np.random.default_rng(7)
    shp = (NI + 2, NJ + 2)
    er_dc = rng.standard_normal(shp)
    c.set_field("Er", er_dc)
    start = [rng.standard_normal(shp) + 1j * rng.standard_normal(shp) for _ in range(3)]   # earlier ghosts
    for k, v in zip(("E1x", "E1r", "E1p"), start):
        c.set_cfield(k, v)
    st = c.microwave("solve_Microwave", tol=1e-12, maxit=2000)
    assert st["converged"] == 1, st
    got = [c.cfield(k) for k in ("E1x", "E1r", "E1p")]

    p = omw.cathode_mw_params(NI, NJ)
    cells, xf, rf = omw.cathode_mw_blocks(p)
    for which, (a, b) in (("flc", cells), ("flx", xf), ("flr", rf)):     # the reference's blocks
        i_bl, j_bl = c.blocks(which, 6)
        assert np.array_equal(a, i_bl) and np.array_equal(b, j_bl), which
    lists = _lists(c)
    jflc = int(cells[1][0][0])
    masks = (omw.block_mask(NI, NJ, *xf), omw.block_mask(NI, NJ, *rf), omw.block_mask(NI, NJ, *cells))
    sysd = omw.mag_system_lists(w["ne"], w["nu"], w["Bx"], w["Br"], w["epsr"], p, masks, lists, jflc)
    E_ref = omw.mag_rect_solve(sysd)
    want = omw.mag_ghosts([np.where(masks[k], E_ref[k], start[k]) for k in range(3)], er_dc, w["epsr"], p, lists,
                          jflc)
    for k in range(3):
        assert _rel(got[k], want[k]) < 1e-8, (k, _rel(got[k], want[k]))

    # update_energy_profile with the port part: currents and absorbed power from zero planes,
    # a random excitation current, S-parameters of a lossy feed
    for k in ("J1x", "J1r", "J1p", "J1x_exc", "J1p_exc"):
        c.set_cfield(k, np.zeros(shp, complex))
    jexc = 1e3 * (rng.standard_normal(shp) + 1j * rng.standard_normal(shp))
    c.set_cfield("J1r_exc", jexc)
    for k in ("Pabs", "Pabsx", "Pabsr", "Pabsp"):
        c.set_field(k, np.zeros(shp))
    S = dict(S11=0.1 + 0.05j, S21=0.9 - 0.2j, S12=0.9 - 0.2j, S22=-0.05 + 0.1j)
    c.set_sparams(*S.values())
    for k, v in (("flag_mwRef", 1), ("Z0", 50.0), ("Pmw", 8.0)):
        c.set_param(k, v)
    J1r_exc0 = c.param("J1r_exc")
    c.microwave("update_energy_profile")

    box = lambda I, J: [(int(I[b][0]), int(I[b][1]), int(J[b][0]), int(J[b][1])) for b in range(6)]
    prof, P = omw.energy_profile(*got, w["ne"], w["nu"], w["Bx"], w["Br"], dict(p, rmin=0.0), box(*xf), box(*rf),
                                 box(*cells))
    prm = dict(dx=p["dx"], dr=p["dr"], rmin=0.0, omegam=p["omegam"], r1=p["r1"], r2=p["r2"], Z0=50.0, Pmw=8.0,
               flag_mwRef=1, i_ref=1, j_out=int(cells[1][4][1]) - 1, i_out0=int(cells[0][4][0]),
               i_out1=int(cells[0][4][1]), jf0=int(rf[1][5][0]), jf1=int(rf[1][5][1]), **S)
    planes, res = omw.mw_port_rescale(*got, [prof["J1x"], prof["J1r"], prof["J1p"]], [None, jexc, None],
                                      prof["Pabs"], sum(P), prm)
    for k in ("E1x", "E1r", "E1p", "J1x", "J1r", "J1p", "J1r_exc"):
        assert _rel(c.cfield(k), planes[k]) < 1e-8, (k, _rel(c.cfield(k), planes[k]))
    assert _rel(c.field("Pabs"), planes["Pabs"]) < 1e-8
    assert c.param("J1r_exc") == pytest.approx(J1r_exc0 * res["J1r_exc_factor"], rel=1e-8)


def test_explicit_variant_through_the_dropin(pkg, cuda_device, ref):
    """EmfieldModule::solve_Microwave_explicit (emfieldModule.hpp:3328-4400): J = sigma E
    of the present field on the right-hand side of the vacuum + epsr operator, the
    same lists, solve and ghost pass; against the oracle's system with the plasma
    conductivity removed and that J added to b."""
    from oracle import microwave as omw
    w = pkg.workloads.mw3_cathode(NI, NJ, seed=3, bmax=0.05)
    c = refpin.case(NI, NJ, dropin=True)
    c.set_param("omegam", w["params"]["omegam"])
    for k, v in (("rhoe", "ne"), ("nu_m1", "nu"), ("Bx", "Bx"), ("Br", "Br"), ("epsr", "epsr")):
        c.set_field(k, w[v])
    rng = np.random.default_rng(11)
    shp = (NI + 2, NJ + 2)
    c.set_field("Er", np.zeros(shp))
    prev = [1e2 * (rng.standard_normal(shp) + 1j * rng.standard_normal(shp)) for _ in range(3)]
    for k, v in zip(("E1x", "E1r", "E1p"), prev):
        c.set_cfield(k, v)
    for k in ("J1x", "J1r", "J1p"):
        c.set_cfield(k, np.zeros(shp, complex))
    st = c.microwave("solve_Microwave_explicit", tol=1e-12, maxit=2000)
    assert st["converged"] == 1, st
    got = [c.cfield(k) for k in ("E1x", "E1r", "E1p")]
    gotJ = [c.cfield(k) for k in ("J1x", "J1r", "J1p")]

    p = omw.cathode_mw_params(NI, NJ)
    cells, xf, rf = omw.cathode_mw_blocks(p)
    box = lambda I, J: [(int(I[b][0]), int(I[b][1]), int(J[b][0]), int(J[b][1])) for b in range(6)]
    prof, _ = omw.energy_profile(*prev, w["ne"], w["nu"], w["Bx"], w["Br"], dict(p, rmin=0.0), box(*xf), box(*rf),
                                 box(*cells))
    J = [prof["J1x"], prof["J1r"], prof["J1p"]]
    for k in range(3):
        assert _rel(gotJ[k], J[k]) < 1e-12, k
    lists = _lists(c)
    jflc = int(cells[1][0][0])
    masks = (omw.block_mask(NI, NJ, *xf), omw.block_mask(NI, NJ, *rf), omw.block_mask(NI, NJ, *cells))
    sysd = omw.mag_system_lists(np.zeros(shp), w["nu"], w["Bx"], w["Br"], w["epsr"], p, masks, lists, jflc)
    g2 = p["dx"] ** 2 * p["dr"] ** 2
    for k in range(3):
        sysd["b"][k][masks[k]] += (-1j * p["omegam"] * omw.MU0 * g2) * J[k][masks[k]]
    E_ref = omw.mag_rect_solve(sysd)
    want = omw.mag_ghosts([np.where(masks[k], E_ref[k], prev[k]) for k in range(3)], np.zeros(shp), w["epsr"], p,
                          lists, jflc)
    for k in range(3):
        assert _rel(got[k], want[k]) < 1e-8, (k, _rel(got[k], want[k]))
