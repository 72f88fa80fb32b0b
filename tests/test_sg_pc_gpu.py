"""GPU Scharfetter-Gummel predictor-correctors of the electron density
(solve_rhoe_wdTe_wSEE_PC, fluidModule.hpp:3082-3970) and energy
(solve_Te_wdTe_wSEE_PC, fluidModule.hpp:4006-4957) against the oracle's
block-by-block restatement, on the reference's cathode blocks and the rectangle."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
COMMON = ("Te", "mu_para", "mu_perp", "mu_rr", "mu_xr", "mu_xx", "Ex", "Er", "rhoi", "Uix", "Uir", "rhoUmx",
          "rhoUmr")
RHOE_IN = COMMON + ("rhoe", "rhoUex", "rhoUer", "rhoUex_wall", "rhoUer_wall", "rate_ionize", "rhoUix_wall")
EPS_IN = COMMON + ("rhoeps", "Gx", "Gr", "Gx_wall", "Gr_wall", "rhoe", "rhoe_old", "rhoUex", "rhoUer", "Pabs",
                   "rate_eloss")


def _geo(kind):
    from oracle import fluid
    if kind == "cathode":
        return fluid.cathode_geometry(), 0.0388, 0.014
    return fluid.rectangle_geometry(96, 64), 10e-3, 5e-3


def _setup(pkg, geo, seed, Lz, Lr, species, **over):
    st = pkg.workloads.sg_state(geo["ni"], geo["nj"], seed=seed, Lz=Lz, Lr=Lr)
    f, prm = st["fields"], dict(st["prm"])
    z = np.load(os.path.join(HERE, "golden", "see_tables.npz"))
    prm["dTe_SEE"] = float(z["dTe_SEE"])
    prm.update(over)
    g = pkg.Grid(geo["ni"], geo["nj"], geo["ib"], geo["jb"])
    fs = pkg.Fields(g)
    for k in (EPS_IN if species == "rhoeps" else RHOE_IN):
        fs.upload(k, f[k])
    fs.set_flags(geo["flags"])
    fs.set_ghost_rules(geo["ghosts"])
    fs.set_energy_keep_walls(geo.get("energy_keep_walls", []))
    for k in ("coefEISEE_eb_table", "coefEISEE_rd_table", "coefEISEE_ts_table"):
        fs.set_table(k, z[k])
    see = (z["coefEISEE_eb_table"], z["coefEISEE_rd_table"], z["coefEISEE_ts_table"], float(z["dTe_SEE"]))
    return f, prm, g, fs, see


def _oracle(f, prm, geo, see, species, capture=None):
    import oracle
    from oracle import fluid

    def solve(aP, aE, aW, aN, aS, b, ib, jb):
        if capture is not None:
            capture.append(dict(aP=aP.copy(), aE=aE.copy(), aW=aW.copy(), aN=aN.copy(), aS=aS.copy(), b=b.copy()))
        return oracle.direct_solve(dict(ni=geo["ni"], nj=geo["nj"], i_bl=ib, j_bl=jb, aP=aP, aE=aE, aW=aW, aN=aN,
                                        aS=aS, b=b))

    return fluid.solve_sg_pc(f, prm, geo, see, solve, species)


def _rel(a, b):
    return np.abs(a - b).max() / (np.abs(b).max() + 1e-300)


def _run(fs, species, prm):
    return fs.solve_Te_pc(prm) if species == "rhoeps" else fs.solve_rhoe_pc(prm)


@pytest.mark.parametrize("species", ["rhoe", "rhoeps"])
@pytest.mark.parametrize("kind", ["cathode", "rectangle"])
def test_sg_assembly_matches_oracle(pkg, orc, cuda_device, kind, species):
    geo, Lz, Lr = _geo(kind)
    f, prm, g, fs, see = _setup(pkg, geo, 31, Lz, Lr, species, maxITR_HES=1, precision=0, error_cnv_SOR=1e-13,
                                maxITR_SOR=200)
    cap = []
    _oracle(f, prm, geo, see, species, cap)
    _run(fs, species, prm)
    blk = geo["flags"] != 0
    scale = np.abs(cap[0]["aP"][blk]).max()
    for k in ("aP", "aE", "aW", "aN", "aS"):
        got = fs.download("pc_" + k)
        assert np.abs(got[blk] - cap[0][k][blk]).max() / scale < 1e-13, k
    got = fs.download("pc_b")
    assert _rel(got[blk], cap[0]["b"][blk]) < 1e-12
    fs.close()
    g.close()


@pytest.mark.parametrize("species", ["rhoe", "rhoeps"])
@pytest.mark.parametrize("kind", ["cathode", "rectangle"])
def test_sg_two_iterations_fp64(pkg, orc, cuda_device, kind, species):
    geo, Lz, Lr = _geo(kind)
    f, prm, g, fs, see = _setup(pkg, geo, 32, Lz, Lr, species, precision=0, error_cnv_SOR=1e-13, maxITR_SOR=200)
    ref = _oracle(f, prm, geo, see, species)
    res = _run(fs, species, prm)
    assert res["ncount"] == 2 and res["solver_rc"] == 0, res
    outs = ("rhoeps", "Gx", "Gr", "Gx_wall", "Gr_wall", "Te", "Te_old") if species == "rhoeps" else \
        ("rhoe", "rhoUex", "rhoUer", "rhoUex_wall", "rhoUer_wall", "rhoe_old")
    for k in outs:
        got = fs.download(k)
        assert _rel(got, ref[k]) < 1e-9, (k, _rel(got, ref[k]))
    names = ("rhoeps", "Gx", "Gr") if species == "rhoeps" else ("rhoe", "rhoUex", "rhoUer")
    for e, k in zip(res["errors"], names):
        assert e == pytest.approx(ref["error_" + k], rel=1e-6), k
    np.testing.assert_allclose(res["error_iter"], ref["errors_last"], rtol=1e-5)
    if species == "rhoe":
        for k in ("Ii_Anode", "Ie_Anode", "I_Anode"):
            assert res[k] == pytest.approx(ref[k], rel=1e-9, abs=1e-30), k
    fs.close()
    g.close()


def test_sg_mixed_precision_setup_tolerance(pkg, orc, cuda_device):
    """The shipped electron-sweep settings (SMG, 30 iterations, 1e-10) in mixed precision."""
    from oracle import fluid
    geo = fluid.rectangle_geometry(256, 128)
    for species in ("rhoe", "rhoeps"):
        f, prm, g, fs, see = _setup(pkg, geo, 33, 10e-3, 5e-3, species)
        ref = _oracle(f, prm, geo, see, species)
        res = _run(fs, species, prm)
        assert res["solver"]["converged"] == 1, (species, res["solver"], res["error_iter"])
        k = "rhoeps" if species == "rhoeps" else "rhoe"
        assert _rel(fs.download(k), ref[k]) < 1e-8, k
        fs.close()
        g.close()
