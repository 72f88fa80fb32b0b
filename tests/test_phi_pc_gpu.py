"""GPU potential predictor-corrector (FluidModule::solve_phi_couple_wdTe_wSEE_PC,
fluidModule.hpp:2080-3075) against the oracle's block-by-block restatement, on
the reference's cathode blocks and on the r-z rectangle, with the reference's
SEE yields (tests/golden/see_tables.npz)."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
INPUTS = ("phi", "Ex", "Er", "nUex", "nUer", "rhoe", "rhoe_old", "rhoi", "Te", "mu_para", "mu_perp", "mu_rr",
          "mu_xr", "mu_xx", "rate_ionize", "Uix", "Uir", "rhoUmx", "rhoUmr")
OUTPUTS = ("phi", "Ex", "Er", "nUex", "nUer")


def _see():
    z = np.load(os.path.join(HERE, "golden", "see_tables.npz"))
    return z


def _setup(pkg, geo, seed, Lz, Lr, **over):
    st = pkg.workloads.pc_state(geo["ni"], geo["nj"], seed=seed, Lz=Lz, Lr=Lr)
    f, prm = st["fields"], dict(st["prm"])
    z = _see()
    prm["dTe_SEE"] = float(z["dTe_SEE"])
    prm.update(over)
    g = pkg.Grid(geo["ni"], geo["nj"], geo["ib"], geo["jb"])
    fs = pkg.Fields(g)
    for k in INPUTS:
        fs.upload(k, f[k])
    fs.set_flags(geo["flags"])
    for k in ("coefEISEE_eb_table", "coefEISEE_rd_table", "coefEISEE_ts_table"):
        fs.set_table(k, z[k])
    see = (z["coefEISEE_eb_table"], z["coefEISEE_rd_table"], z["coefEISEE_ts_table"], float(z["dTe_SEE"]))
    return f, prm, g, fs, see


def _oracle(f, prm, geo, see, capture=None):
    import oracle
    from oracle import fluid

    def solve(aP, aE, aW, aN, aS, b, ib, jb):
        if capture is not None:
            capture.append(dict(aP=aP.copy(), aE=aE.copy(), aW=aW.copy(), aN=aN.copy(), aS=aS.copy(), b=b.copy()))
        sysd = dict(ni=geo["ni"], nj=geo["nj"], i_bl=ib, j_bl=jb, aP=aP, aE=aE, aW=aW, aN=aN, aS=aS, b=b)
        return oracle.direct_solve(sysd)

    return fluid.solve_phi_pc(f, prm, geo, see, solve)


def _geo(kind):
    from oracle import fluid
    if kind == "cathode":
        return fluid.cathode_geometry(), 0.0388, 0.014
    return fluid.rectangle_geometry(96, 64), 10e-3, 5e-3


def _rel(a, b):
    return np.abs(a - b).max() / (np.abs(b).max() + 1e-300)


@pytest.mark.parametrize("kind", ["cathode", "rectangle"])
def test_phi_pc_assembly_matches_oracle(pkg, orc, cuda_device, kind):
    geo, Lz, Lr = _geo(kind)
    f, prm, g, fs, see = _setup(pkg, geo, 21, Lz, Lr, maxITR_HES_phi=1, precision=0, error_cnv_SOR_phi=1e-13,
                                maxITR_SOR_phi=200)
    cap = []
    _oracle(f, prm, geo, see, cap)
    fs.solve_phi_pc(prm)
    names = dict(aP="pc_aP", aE="pc_aE", aW="pc_aW", aN="pc_aN", aS="pc_aS", b="pc_b")
    blk = geo["flags"] != 0
    for k, n in names.items():
        got = fs.download(n)
        ref = cap[0][k]
        assert _rel(got[blk], ref[blk]) < 1e-13, (k, _rel(got[blk], ref[blk]))
    fs.close()
    g.close()


@pytest.mark.parametrize("kind", ["cathode", "rectangle"])
def test_phi_pc_two_iterations_fp64(pkg, orc, cuda_device, kind):
    geo, Lz, Lr = _geo(kind)
    f, prm, g, fs, see = _setup(pkg, geo, 22, Lz, Lr, precision=0, error_cnv_SOR_phi=1e-13, maxITR_SOR_phi=200)
    ref = _oracle(f, prm, geo, see)
    res = fs.solve_phi_pc(prm)
    assert res["ncount"] == 2 and res["solver_rc"] == 0, res
    for k in OUTPUTS:
        got = fs.download(k)
        assert _rel(got, ref[k]) < 1e-9, (k, _rel(got, ref[k]))
    for k in ("error_phi", "error_nUex", "error_nUer"):
        assert res[k] == pytest.approx(ref[k], rel=1e-6), k
    np.testing.assert_allclose(res["error_iter"], ref["errors_last"], rtol=1e-5)
    fs.close()
    g.close()


def test_phi_pc_mixed_precision_setup_tolerance(pkg, orc, cuda_device):
    """The shipped inner-solve setting (SMG, 30 iterations, 1e-10) in mixed precision."""
    from oracle import fluid
    geo = fluid.rectangle_geometry(256, 128)
    f, prm, g, fs, see = _setup(pkg, geo, 23, 10e-3, 5e-3)
    ref = _oracle(f, prm, geo, see)
    res = fs.solve_phi_pc(prm)
    assert res["solver"]["converged"] == 1, res
    for k in OUTPUTS:
        assert _rel(fs.download(k), ref[k]) < 1e-7, k
    fs.close()
    g.close()


def test_phi_pc_sor_inner_solve(pkg, orc, cuda_device):
    """flag_iter_phi = 0 selects the SOR replacement (alpha 1.9)."""
    from oracle import fluid
    geo = fluid.rectangle_geometry(40, 24)
    f, prm, g, fs, see = _setup(pkg, geo, 24, 10e-3, 5e-3, flag_iter_phi=0, maxITR_SOR_phi=20000,
                                error_cnv_SOR_phi=1e-13)
    ref = _oracle(f, prm, geo, see)
    fs.solve_phi_pc(prm)
    for k in OUTPUTS:
        assert _rel(fs.download(k), ref[k]) < 1e-8, k
    fs.close()
    g.close()
