"""CPU checks of the fluid-side oracle and host helpers: the rate-table fixture
parsed from the reference's BOLSIG+ files, the table lookups of miniFuncs.hpp
and the side flags of the cathode's fluid blocks."""
import os

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))


def _tables():
    z = np.load(os.path.join(HERE, "golden", "rate_tables.npz"))
    return {k: z[k] for k in z.files if k not in ("dTe", "dEi")}, float(z["dTe"]), float(z["dEi"])


def test_rate_table_fixture_matches_reference_rows():
    from oracle import fluid
    tb, dTe, dEi = _tables()
    assert set(tb) == set(fluid.TABLES)
    # first data rows of input/rateCoef_e.csv and rateCoef_i.csv (0 eV): elastic 5.21e-14
    # plus one superelastic column of 1.13e-15, ion elastic 5.20e-16
    assert tb["nu_elas_N"][0] == pytest.approx(5.21e-14, rel=1e-12)
    assert tb["nu_super_N"][0] == pytest.approx(1.13e-15, rel=1e-12)
    assert tb["nui_m_N"][0] == pytest.approx(5.20e-16, rel=1e-12)
    assert tb["nu_elas_N"].shape == (1801,) and tb["nui_m_N"].shape == (39,)
    # steps: 0.1 eV mean energy -> 2/3 * 0.1 eV in K; 0.001 eV drift energy in J
    assert dTe == pytest.approx(0.1 * 2.0 / 3.0 * fluid.E0 / fluid.BOLTZ, rel=1e-12)
    assert dEi == pytest.approx(0.001 * fluid.E0, rel=1e-9)
    # ground-state energy losses dominate the metastable ones at high energy
    assert tb["rate_eloss_n_N"][-1] > tb["rate_eloss_m_N"][-1] > 0


def test_bolsig_parser_on_small_text():
    from oracle import fluid
    te = ("Type,Elastic,Excitation,Ionization,Ionization_step,Other\n"
          "Energy(eV),0,10,20,5,-2\n"
          "0,1,0,0,0,3\n0.5,2,4,6,8,10\n1.0,1,1,1,1,1\n")
    ti = "Type,Elastic,Elastic\nDrift_energy(eV),0,0\n0,1,2\n0.01,3,4\n"
    tb, dTe, dEi = fluid.bolsig_tables(te, ti)
    e = fluid.E0
    assert np.allclose(tb["nu_elas_N"], [1, 2, 1]) and np.allclose(tb["nu_exc_N"], [0, 4, 1])
    assert np.allclose(tb["nu_ionz_N"], [0, 6, 1]) and np.allclose(tb["nu_ionzStep_N"], [0, 8, 1])
    assert np.allclose(tb["nu_super_N"], [3, 10, 1])
    assert np.allclose(tb["rate_eloss_n_N"], np.array([0, 4 * 10 + 6 * 20, 10 + 20]) * e)
    assert np.allclose(tb["rate_eloss_m_N"], np.array([3 * -2, 8 * 5 + 10 * -2, 5 - 2]) * e)
    assert np.allclose(tb["nui_m_N"], [3, 7])
    assert dTe == pytest.approx(0.5 * 2 / 3 * e / fluid.BOLTZ) and dEi == pytest.approx(0.01 * e)


def test_lookups_match_scalar_restatement():
    """Vectorised lookups against a per-value loop of miniFuncs.hpp:35-91."""
    from oracle import fluid
    tb, dTe, dEi = _tables()
    v, n = tb["nu_ionz_N"], tb["nu_ionz_N"].size
    rng = np.random.default_rng(0)
    Te = np.concatenate([rng.uniform(0, (n + 5) * dTe, 500), np.arange(0, n + 2) * dTe])
    f = fluid.func_Te(v, Te, dTe)
    d = fluid.func_dTe(v, Te, dTe)
    for t, a, b in zip(Te, f, d):
        iL = int(t / dTe)
        iR = iL + 1
        ref = (v[iR] - v[iL]) / (dTe + 1e-100) * (t - iL * dTe) + v[iL] if iR < n - 1 else v[n - 1]
        assert a == ref
        if iR >= n - 1:
            iL, iR = n - 2, n - 1
        assert b == (v[iR] - v[iL]) / (iR * dTe - iL * dTe + 1e-100)
    vi, m = tb["nui_m_N"], tb["nui_m_N"].size
    mi = 131.293e-3 / 6.02214076e23
    Ei = rng.uniform(0, 3 * m * dEi, 300)
    g = fluid.func_Ei(vi, Ei, dEi, mi)
    for t, a in zip(Ei, g):
        iL = int(t / dEi)
        if iL + 1 < m - 1:
            ref = (vi[iL + 1] - vi[iL]) / (dEi + 1e-100) * (t - iL * dEi) + vi[iL]
        else:
            ref = vi[m - 1] / np.sqrt((m - 1) * dEi / mi) * np.sqrt(t / mi)
        assert a == pytest.approx(ref, rel=1e-15)


def test_cathode_flags_host_helper_matches_oracle(pkg):
    from oracle import fluid
    ib, jb = fluid.cathode_blocks()
    assert ib.tolist() == [[40, 67], [68, 114], [68, 89], [90, 139], [140, 194]]
    assert jb.tolist() == [[21, 45], [11, 45], [4, 10], [1, 10], [1, 70]]
    a = fluid.cathode_flags(194, 70, ib, jb)
    b = pkg.fluid.cathode_flags(194, 70, *pkg.fluid.cathode_blocks())
    assert (a == b).all()
    # the axis and the anode (last column) are the only boundaries of block 4's corner cell
    assert a[194, 1] == fluid.F_BLX | fluid.F_BLR_WALL | fluid.F_BRR_WALL | fluid.F_BRR_OPEN | fluid.F_BRX_BIAS
    assert (a[0, :] == 0).all() and (a[:, 0] == 0).all() and (a[:, -1] == 0).all()
    assert (pkg.fluid.rectangle_flags(12, 9) == fluid.rectangle_flags(12, 9)).all()


def test_transport_oracle_limits():
    """Size-independent properties of the transport update: B = 0 makes the
    tensor isotropic, nu_m = nu_elas + Bohm + Sagdeev terms, and cells off the
    fluid blocks keep their anomalous frequency."""
    from oracle import fluid
    import importlib
    import __graft_entry__
    wl = importlib.import_module(__graft_entry__.load_package().__name__ + ".workloads")
    st = wl.plasma_state(10, 8, seed=5)
    f, prm = st["fields"], dict(st["prm"])
    f["Bx"][:] = 0.0
    f["Br"][:] = 0.0
    tb, dTe, dEi = _tables()
    prm.update(dTe=dTe, dEi=dEi)
    fl = fluid.rectangle_flags(10, 8)
    fl[3, 3] = 0
    out = fluid.update_transport_coef(f, tb, prm, fl)
    assert np.allclose(out["mu_xx"], out["mu_para"], rtol=1e-15)
    assert np.allclose(out["mu_rr"], out["mu_para"], rtol=1e-15)
    assert np.all(out["mu_xr"] == 0)
    assert np.allclose(out["nu_m"], out["nu_elas"] + f["nu_ano"] + out["nu_ano_IAT"], rtol=1e-14)
    assert out["nu_ano_IAT"][3, 3] == 0.0 and out["nu_ano_IAT"][4, 4] > 0.0


@pytest.mark.parametrize("kind", ["cathode", "rectangle"])
def test_pc_geometry_flags_match_reference_blocks(kind):
    """The side-flag rules the device kernels use (interior face = both cells in
    the fluid, wall face = cleared bit) select exactly the reference's face
    blocks and wall segments."""
    from oracle import fluid
    geo = fluid.cathode_geometry() if kind == "cathode" else fluid.rectangle_geometry(30, 20)
    fl = geo["flags"]
    F = fl != 0
    ix = np.zeros_like(F); ix[1:, :] = F[1:, :] & F[:-1, :]
    ir = np.zeros_like(F); ir[:, 1:] = F[:, 1:] & F[:, :-1]
    bx = np.zeros_like(F); br = np.zeros_like(F)
    for (a, b), (c, e) in zip(geo["fxi"], geo["fxj"]):
        assert not bx[a:b + 1, c:e + 1].any()
        bx[a:b + 1, c:e + 1] = True
    for (a, b), (c, e) in zip(geo["fri"], geo["frj"]):
        assert not br[a:b + 1, c:e + 1].any()
        br[a:b + 1, c:e + 1] = True
    assert (ix == bx).all() and (ir == br).all()
    seg = {k: np.zeros_like(F) for k in ("L", "R", "RB", "D", "U", "O")}
    for k, i0, i1, j0, j1 in geo["segs"]:
        seg[k][i0:i1 + 1, j0:j1 + 1] = True
    cleared = lambda bit: F & ((fl & bit) == 0)
    assert (cleared(fluid.F_BLX) == seg["L"]).all()
    assert (cleared(fluid.F_BRX) == (seg["R"] | seg["RB"])).all()
    assert (((fl & fluid.F_BRX_BIAS) != 0) == seg["RB"]).all()
    assert (cleared(fluid.F_BLR_WALL) == seg["D"]).all()
    assert (cleared(fluid.F_BRR_WALL) == seg["U"]).all()
    assert (cleared(fluid.F_BRR_OPEN) == seg["O"]).all()
    # every wall ghost lies outside the fluid
    assert not (F[:-1, :] & seg["L"][1:, :]).any() and not (F[1:, :] & (seg["R"] | seg["RB"])[:-1, :]).any()
    assert not (F[:, :-1] & seg["D"][:, 1:]).any() and not (F[:, 1:] & (seg["U"] | seg["O"])[:, :-1]).any()


def test_phi_pc_oracle_properties(orc):
    """Rectangle PC step in the oracle: the wall ghosts keep their Dirichlet
    relations, the interior fields are the potential's differences, and the
    assembled Poisson system is solved."""
    from oracle import fluid
    import importlib
    import __graft_entry__
    wl = importlib.import_module(__graft_entry__.load_package().__name__ + ".workloads")
    geo = fluid.rectangle_geometry(24, 16)
    st = wl.pc_state(24, 16, seed=7)
    z = np.load(os.path.join(HERE, "golden", "see_tables.npz"))
    see = (z["coefEISEE_eb_table"], z["coefEISEE_rd_table"], z["coefEISEE_ts_table"], float(z["dTe_SEE"]))
    prm = dict(st["prm"], dTe_SEE=float(z["dTe_SEE"]))
    res = []

    def solve(aP, aE, aW, aN, aS, b, ib, jb):
        s = dict(ni=24, nj=16, i_bl=ib, j_bl=jb, aP=aP, aE=aE, aW=aW, aN=aN, aS=aS, b=b)
        x = orc.direct_solve(s)
        res.append(orc.residual(s, x)[1] / orc.residual(s, np.zeros_like(x))[1])
        return x

    out = fluid.solve_phi_pc(st["fields"], prm, geo, see, solve)
    phi = out["phi"]
    assert out["ncount"] == 2 and max(res) < 1e-12
    np.testing.assert_allclose(phi[0, 1:17], -phi[1, 1:17], rtol=1e-12)
    np.testing.assert_allclose(phi[25, 1:17], 2 * 20.0 - phi[24, 1:17], rtol=1e-12)
    np.testing.assert_allclose(phi[1:25, 17], -phi[1:25, 16], rtol=1e-12)
    np.testing.assert_allclose(out["Ex"][2:25, 1:17], -(phi[2:25, 1:17] - phi[1:24, 1:17]) / prm["dx"], rtol=1e-12)
    np.testing.assert_allclose(out["Er"][1:25, 2:17], -(phi[1:25, 2:17] - phi[1:25, 1:16]) / prm["dr"], rtol=1e-12)


@pytest.mark.parametrize("species", ["rhoe", "rhoeps"])
def test_sg_oracle_properties(orc, species):
    """Electron sweeps in the oracle: the assembled increment systems are solved,
    the density stays positive, Te follows rhoeps and the ghost rules hold."""
    from oracle import fluid
    import importlib
    import __graft_entry__
    wl = importlib.import_module(__graft_entry__.load_package().__name__ + ".workloads")
    geo = fluid.rectangle_geometry(24, 16)
    st = wl.sg_state(24, 16, seed=8)
    z = np.load(os.path.join(HERE, "golden", "see_tables.npz"))
    see = (z["coefEISEE_eb_table"], z["coefEISEE_rd_table"], z["coefEISEE_ts_table"], float(z["dTe_SEE"]))
    prm = dict(st["prm"], dTe_SEE=float(z["dTe_SEE"]))
    res = []

    def solve(aP, aE, aW, aN, aS, b, ib, jb):
        s = dict(ni=24, nj=16, i_bl=ib, j_bl=jb, aP=aP, aE=aE, aW=aW, aN=aN, aS=aS, b=b)
        x = orc.direct_solve(s)
        res.append(orc.residual(s, x)[1] / orc.residual(s, np.zeros_like(x))[1])
        return x

    out = fluid.solve_sg_pc(st["fields"], prm, geo, see, solve, species)
    assert out["ncount"] == 2 and max(res) < 1e-12
    n = out[species]
    assert (n[1:25, 1:17] > 0).all()
    if species == "rhoeps":
        rhoe = st["fields"]["rhoe"]
        Te = out["Te"]
        rmax = rhoe[1:25, 1:17].max()
        np.testing.assert_allclose(Te[1:25, 1:17], n[1:25, 1:17] / (1.5 * (rhoe[1:25, 1:17] + 1e-3 * rmax) * fluid.BOLTZ),
                                   rtol=1e-12)
        np.testing.assert_array_equal(Te[0, 1:17], Te[1, 1:17])
        np.testing.assert_array_equal(Te[25, 1:17], Te[24, 1:17])
    else:
        assert (n[0, 1:17] == 0).all()
        np.testing.assert_array_equal(n[25, 1:17], n[24, 1:17])
        np.testing.assert_array_equal(n[1:25, 17], n[1:25, 16])
