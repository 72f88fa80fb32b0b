"""The CPU restatement (oracle/fluid.py) and the package's geometry tables pinned to
the reference itself: its FluidModule and InitialModule compiled from the
unmodified headers (fluidModule.hpp, initialModule.hpp and what they include)
into oracle/_ref/libref.so, with the HYPRE solves replaced by the exact solve
that SMG converges to (oracle/refshim/solverFuncs.hpp).

Every sweep runs on the reference's cathode geometry (makeBoundary at 194 x 70)
from the same seeded inputs on both sides.  The bar is the arithmetic itself:
the ion, neutral and transport paths agree to the last bits; the potential and
electron sweeps to rounding, where the Scharfetter-Gummel weights and the wall
fluxes take exp() from numpy on one side and from the C library on the other."""
import os

import numpy as np
import pytest

import refpin

HERE = os.path.dirname(os.path.abspath(__file__))
SIZES = [(194, 70), (97, 35), (388, 140), (776, 280)]


@pytest.fixture(scope="module")
def ref():
    from oracle import ref as R
    R.build()
    if not R.available():
        pytest.skip("oracle/_ref/libref.so not built: the reference sources are needed to build it")
    return R


def _see():
    z = np.load(os.path.join(HERE, "golden", "see_tables.npz"))
    return (z["coefEISEE_eb_table"], z["coefEISEE_rd_table"], z["coefEISEE_ts_table"], float(z["dTe_SEE"]))


def _solver(ni, nj, capture=None):
    import oracle

    def solve(aP, aE, aW, aN, aS, b, ib, jb):
        if capture is not None:
            capture.append(dict(aP=aP.copy(), aE=aE.copy(), aW=aW.copy(), aN=aN.copy(), aS=aS.copy(), b=b.copy()))
        return oracle.direct_solve(dict(ni=ni, nj=nj, i_bl=ib, j_bl=jb, aP=aP, aE=aE, aW=aW, aN=aN, aS=aS, b=b))
    return solve


def _maxrel(a, b):
    return float(np.abs(a - b).max() / (np.abs(b).max() + 1e-300))


@pytest.mark.parametrize("ni,nj", SIZES)
def test_blocks_match_makeBoundary(ref, pkg, ni, nj):
    """Cell, x-face and r-face blocks of the oracle's and the package's cathode
    geometry equal the ones InitialModule::makeBoundary computes."""
    from oracle import fluid
    c = refpin.case(ni, nj)
    for geo in (fluid.cathode_geometry(ni, nj), pkg.fluid.cathode_geometry(ni, nj)):
        for which, (ki, kj) in dict(flc=("ib", "jb"), flx=("fxi", "fxj"), flr=("fri", "frj")).items():
            i_bl, j_bl = c.blocks(which, 5)
            np.testing.assert_array_equal(np.asarray(geo[ki]), i_bl, err_msg=which)
            np.testing.assert_array_equal(np.asarray(geo[kj]), j_bl, err_msg=which)
    # fluid cells = union of blocks 0..4, and every flagged cell is one (and only those)
    geo = pkg.fluid.cathode_geometry(ni, nj)
    np.testing.assert_array_equal(geo["flags"] != 0, c.int_field("jdgBnd_flc") == 1)


@pytest.mark.parametrize("ni,nj", SIZES)
def test_microwave_lists_match_makeBoundary(ref, pkg, ni, nj):
    """The 12 MicrowaveBC lists the package builds from its segment table
    (data/mw_lists_cathode.json) equal makeBoundary's at every resolution, entry
    for entry and in order."""
    c = refpin.case(ni, nj)
    mw = pkg.fluid.cathode_microwave(ni, nj)
    names = {"x": "x", "r": "r", "p": "p"}
    for (field, side), entries in mw["lists"].items():
        got = np.asarray(entries, np.int64).reshape(-1, 3)
        want = c.mw_list(f"Bnd{side}{names[field]}").astype(np.int64)
        np.testing.assert_array_equal(got, want, err_msg=f"{field}{side}")
    # the microwave blocks (six per field) are the reference's too
    (xi, xj), (ri, rj), (ci, cj) = mw["blocks"]
    for (a, b), which in (((xi, xj), "flx"), ((ri, rj), "flr"), ((ci, cj), "flc")):
        i_bl, j_bl = c.blocks(which, 6)
        np.testing.assert_array_equal(np.asarray(a), i_bl, err_msg=which)
        np.testing.assert_array_equal(np.asarray(b), j_bl, err_msg=which)


def test_phi_pc_matches_reference(ref, pkg):
    """solve_phi_couple_wdTe_wSEE_PC (fluidModule.hpp:2080-3075): both PC iterations'
    assembled systems and the updated phi, E and electron fluxes."""
    from oracle import fluid
    geo = fluid.cathode_geometry()
    ni, nj = geo["ni"], geo["nj"]
    st = pkg.workloads.pc_state(ni, nj, seed=22, Lz=0.0388, Lr=0.014)
    see = _see()
    f, prm = st["fields"], dict(st["prm"], dTe_SEE=see[3])
    cap = []
    o = fluid.solve_phi_pc(f, prm, geo, see, _solver(ni, nj, cap))
    c = refpin.case(ni, nj)
    refpin.put(c, prm)
    c.set_fields(f)
    refpin.put_see(c, see)
    ref.capture(True)
    c.call("solve_phi_couple_wdTe_wSEE_PC")
    sysr = ref.captured_planes(ni, nj)
    ref.capture(False)
    assert len(sysr) == len(cap) == 2
    blk = geo["flags"] != 0
    for a, b in zip(cap, sysr):
        for k in ("aP", "aE", "aW", "aN", "aS", "b"):
            assert _maxrel(a[k][blk], b[k][blk]) < 1e-14, k
    for k in ("phi", "Ex", "Er", "nUex", "nUer"):
        assert _maxrel(o[k], c.field(k)) < 1e-13, k
    for k in ("error_phi", "error_nUex", "error_nUer"):
        assert o[k] == pytest.approx(c.param(k), rel=1e-12), k


@pytest.mark.parametrize("species", ["rhoe", "rhoeps"])
def test_sg_pc_matches_reference(ref, pkg, species):
    """solve_rhoe_wdTe_wSEE_PC (:3082-3970) and solve_Te_wdTe_wSEE_PC (:4006-4957):
    Scharfetter-Gummel assembly of both PC iterations, the updated density /
    energy, fluxes, wall fluxes (the energy sweep leaves Gr_wall of the x2 wall
    as it was), Te recovery, calcRes errors and the anode currents."""
    from oracle import fluid
    geo = fluid.cathode_geometry()
    ni, nj = geo["ni"], geo["nj"]
    st = pkg.workloads.sg_state(ni, nj, seed=31, Lz=0.0388, Lr=0.014)
    see = _see()
    f, prm = st["fields"], dict(st["prm"], dTe_SEE=see[3])
    # a nonzero previous wall flux, so that a wall the sweep does not record shows
    f["Gr_wall"] = f["rhoeps"] * 1e2
    cap = []
    o = fluid.solve_sg_pc(f, prm, geo, see, _solver(ni, nj, cap), species)
    c = refpin.case(ni, nj)
    refpin.put(c, prm, "rhoe" if species == "rhoe" else "eps")
    c.set_fields(f)
    refpin.put_see(c, see)
    ref.capture(True)
    c.call("solve_rhoe_wdTe_wSEE_PC" if species == "rhoe" else "solve_Te_wdTe_wSEE_PC")
    sysr = ref.captured_planes(ni, nj)
    ref.capture(False)
    assert len(sysr) == len(cap) == 2
    blk = geo["flags"] != 0
    for a, b in zip(cap, sysr):
        for k in ("aP", "aE", "aW", "aN", "aS", "b"):
            assert _maxrel(a[k][blk], b[k][blk]) < 1e-11, (k, _maxrel(a[k][blk], b[k][blk]))
    if species == "rhoe":
        outs = ("rhoe", "rhoUex", "rhoUer", "rhoUex_wall", "rhoUer_wall")
        errs = ("error_rhoe", "error_rhoUex", "error_rhoUer", "I_Anode", "Ii_Anode", "Ie_Anode")
    else:
        outs = ("rhoeps", "Gx", "Gr", "Gx_wall", "Gr_wall", "Te")
        errs = ("error_rhoeps", "error_Gx", "error_Gr")
    for k in outs:
        assert _maxrel(o[k], c.field(k)) < 1e-11, (k, _maxrel(o[k], c.field(k)))
    for k in errs:
        assert o[k] == pytest.approx(c.param(k), rel=1e-11), k


@pytest.mark.parametrize("flag_error", [3, 0])
def test_ion_step_matches_reference(ref, pkg, flag_error):
    """solve_Uix_tmp, solve_Uir_tmp, solve_Uip_tmp, solve_rhoi_constTe and
    correct_Ui_constTe (:123-2072) in the order of src/main.cpp:191-197."""
    from oracle import fluid
    geo = fluid.cathode_geometry()
    ni, nj = geo["ni"], geo["nj"]
    st = pkg.workloads.ion_state(ni, nj, seed=41, Lz=0.0388, Lr=0.014)
    f, prm = st["fields"], dict(st["prm"], flag_error=flag_error)
    s = _solver(ni, nj)
    o = fluid.ion_step(f, prm, geo, s, s, s)
    c = refpin.case(ni, nj)
    refpin.put(c, prm, "ion")
    c.set_fields(f)
    for m in ("solve_Uix_tmp", "solve_Uir_tmp", "solve_Uip_tmp", "solve_rhoi_constTe", "correct_Ui_constTe"):
        c.call(m)
    for k in ("Uix", "Uir", "Uip", "rhoi", "rhoUix", "rhoUir", "rhoUix_wall", "rhoUir_wall", "Uix_old", "rhoi_old"):
        assert _maxrel(o[k], c.field(k)) < 1e-14, (k, _maxrel(o[k], c.field(k)))
    for k in ("error_rhoi", "error_Uix", "error_Uir", "error_Uip"):
        assert o[k] == pytest.approx(c.param(k), rel=1e-13), k


def test_neutrals_match_reference(ref, pkg):
    """update_rhon (:4963-5410) and update_rhom (:5416-5792) with the gas inlet."""
    from oracle import fluid
    geo = fluid.cathode_geometry()
    pg = pkg.fluid.cathode_geometry()
    ni, nj = geo["ni"], geo["nj"]
    st = pkg.workloads.neutral_state(ni, nj, seed=51, Lz=0.0388, Lr=0.014)
    f = st["fields"]
    prm = dict(st["prm"], xL=pg["xL"], x6=pg["x6"], width_neutIn=pg["width_neutIn"])
    o = fluid.update_neutrals(f, prm, geo, _solver(ni, nj))
    c = refpin.case(ni, nj)
    refpin.put(c, prm, "neutral")
    c.set_fields(f)
    c.call("update_rhon")
    c.call("update_rhom")
    for k in ("rhon", "rhom", "rhoUnx", "rhoUnr", "rhoUnx_wall", "rhoUnr_wall", "rhoUmx", "rhoUmr", "rhoUmx_wall",
              "rhoUmr_wall", "rhon_old", "rhom_old"):
        assert _maxrel(o[k], c.field(k)) < 1e-14, (k, _maxrel(o[k], c.field(k)))
    for k in ("error_rhon", "error_rhom"):
        assert o[k] == pytest.approx(c.param(k), rel=1e-13), k


def test_transport_matches_reference(ref, pkg):
    """update_transport_coef (:5799-5976) on the reference's rate tables: the
    ionisation source, collision frequencies (Bohm and Sagdeev terms on) and the
    mobility tensor."""
    from oracle import fluid
    geo = fluid.cathode_geometry()
    ni, nj = geo["ni"], geo["nj"]
    z = np.load(os.path.join(HERE, "golden", "rate_tables.npz"))
    tb = {k: z[k] for k in z.files if k not in ("dTe", "dEi")}
    st = pkg.workloads.plasma_state(ni, nj, seed=11, dr=0.014 / nj)
    f, prm = st["fields"], dict(st["prm"], dTe=float(z["dTe"]), dEi=float(z["dEi"]))
    o = fluid.update_transport_coef(f, tb, prm, geo["flags"])
    c = refpin.case(ni, nj)
    refpin.put(c, prm)
    c.set_fields(f)
    for k, v in tb.items():
        c.set_table(k, v)
    c.call("update_transport_coef")
    for k in ("nu_ano_IAT", "Mache", "nu_elas", "nu_exc", "nu_excReso", "nu_excMeta", "nu_ionz", "nu_ionzStep",
              "nu_excStep", "nu_super", "nu_m", "nu_m1", "rate_ionize", "nui_m", "rate_eloss", "delossdeps", "mu_para",
              "mu_xx", "mu_rr", "mu_xr", "mu_perp", "mu_min"):
        assert _maxrel(o[k], c.field(k)) < 1e-14, (k, _maxrel(o[k], c.field(k)))


def test_check_cfl_matches_reference(ref, pkg):
    """check_CFL (:57-115): the CFL number of a fixed dt and the adaptive dt."""
    from oracle import fluid
    ni, nj = 194, 70
    st = pkg.workloads.plasma_state(ni, nj, seed=12, dr=0.014 / nj)
    f = st["fields"]
    for k in ("mu_para", "mu_perp"):
        f[k] = 10.0 ** np.random.default_rng(5).uniform(0.0, 3.0, f["rhoe"].shape)
    for adp in (0, 1):
        prm = dict(rmin=0.0, dr=0.014 / nj, masse=st["prm"]["masse"], flag_adp_dt=adp, CFL=2.0, dt=1e-10)
        o = fluid.check_cfl(f, prm)
        c = refpin.case(ni, nj)
        refpin.put(c, prm)
        c.set_fields(f)
        c.call("check_CFL")
        assert o["CFL"] == pytest.approx(c.param("CFL"), rel=1e-14), adp
        assert o["dt"] == pytest.approx(c.param("dt"), rel=1e-14), adp


def test_steps_match_reference(ref, pkg):
    """20 whole time steps (src/main.cpp:172-251 without the microwave update) of
    the synthetic discharge on the cathode: the oracle's chained restatement
    against the reference's own loop body.  rel-L2 over the fluid cells of phi,
    ne, ni, Te and the cell-centred |E| of the result output within 1e-8."""
    import test_fluid_step_gpu as T
    nstep = 20
    geo, ogeo, st, cfg = T.setup(pkg, "cathode")
    so, Po = T.oracle_run(geo, ogeo, st, cfg, nstep)
    c = refpin.case(geo["ni"], geo["nj"], width_neutIn=geo["width_neutIn"])
    refpin.put_step(c, st, cfg)
    c.call("update_transport_coef")
    for _ in range(nstep):
        c.call("step")
    assert c.param("itime") == Po["itime"] == nstep
    assert c.param("CFL") == pytest.approx(Po["CFL"], rel=1e-12)
    m = refpin.fluid_mask(c)
    r = c.table("r")
    for k in ("phi", "rhoe", "rhoi", "Te"):
        assert refpin.rel_l2(so[k], c.field(k), m) < 1e-8, (k, refpin.rel_l2(so[k], c.field(k), m))
    e_o = refpin.emag(so["Ex"], so["Er"], r)
    e_r = refpin.emag(c.field("Ex"), c.field("Er"), r)
    assert refpin.rel_l2(e_o, e_r, m) < 1e-8
    for k in ("rhon", "rhom", "rhoeps", "Uix", "Uir", "Uip"):
        assert refpin.rel_l2(so[k], c.field(k), m) < 1e-7, k
