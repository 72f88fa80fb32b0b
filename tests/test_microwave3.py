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


# ---------------------------------------------------------------------------
# the cathode geometry: blocks of initialModule.hpp:219-345 and the boundary
# lists of InitialModule::makeBoundary read from the committed segment table
# ---------------------------------------------------------------------------
def _cathode(ni=194, nj=70, bmax=0.05, seed=2):
    import json
    import os
    from importlib import import_module
    wl = import_module("02_cathode-08_modulerev_b200.workloads")
    from oracle import microwave as mw
    w = wl.mw3_cathode(ni, nj, seed=seed, bmax=bmax)
    p = mw.cathode_mw_params(ni, nj)
    cells, xf, rf = mw.cathode_mw_blocks(p)
    masks = (mw.block_mask(ni, nj, *xf), mw.block_mask(ni, nj, *rf), mw.block_mask(ni, nj, *cells))
    here = os.path.dirname(os.path.abspath(__file__))
    with open(os.path.join(here, "golden", "mw_lists_cathode.json")) as f:
        table = json.load(f)
    lists = mw.cathode_mw_lists(cells, table)
    return w, p, mw, masks, lists, int(cells[1][0][0])


def test_cathode_lists_are_boundary_rows():
    """Every list entry is an unknown of its field, no entry repeats within a
    list, and the table's 59 segments cover the fixed counts of the 194 x 70
    grid."""
    w, p, mw, masks, lists, _ = _cathode()
    counts = {k: len(v) for k, v in lists.items()}
    assert sum(counts.values()) == 1644, counts
    for (f, side), ent in lists.items():
        m = masks["xrp".index(f)]
        ij = [(i, j) for i, j, _ in ent]
        assert len(set(ij)) == len(ij), (f, side)
        assert all(m[i, j] for i, j in ij), (f, side)
        assert all(0 <= c <= 7 for _, _, c in ent)


def test_cathode_direct_solution():
    w, p, mw, masks, lists, jflc = _cathode()
    s = mw.mag_system_lists(w["ne"], w["nu"], w["Bx"], w["Br"], w["epsr"], p, masks, lists, jflc)
    A, b, _ = mw.mag_rect_matrix(s)
    assert A.shape[0] == sum(int(m.sum()) for m in masks)
    assert np.max(np.diff(A.indptr)) <= 11
    E = mw.mag_rect_solve(s)
    x = mw.mag_pack(s, E)
    assert np.linalg.norm(A @ x - b) / np.linalg.norm(b) < 1e-11
    assert np.abs(E[1]).max() > 0.0  # driven by the feed (Er west, code 7)
    # without a field Ephi decouples and has no source
    s0 = mw.mag_system_lists(w["ne"], w["nu"], 0 * w["Bx"], 0 * w["Br"], w["epsr"], p, masks, lists, jflc)
    assert np.max(np.abs(mw.mag_rect_solve(s0)[2])) == 0.0


def test_rectangle_surgery_as_lists():
    """The rectangle's boundary rules written as the reference's lists give the
    same system through the list-driven surgery."""
    w, p, mw = _case()
    ni, nj = w["ni"], w["nj"]
    ref = mw.mag_rect_system(w["ne"], w["nu"], w["Bx"], w["Br"], w["epsr"], p)
    lists = mw.rect_mw_lists(ni, nj, p)
    s = mw.mag_system_lists(w["ne"], w["nu"], w["Bx"], w["Br"], w["epsr"], p, ref["masks"], lists, 0)
    for comp in ("x", "r", "p"):
        for k, v in ref[comp].items():
            scale = np.abs(v).max() + 1e-300
            assert np.max(np.abs(s[comp][k] - v)) <= 1e-14 * scale, (comp, k)
    for c in range(3):
        assert np.max(np.abs(s["b"][c] - ref["b"][c])) <= 1e-14 * (np.abs(ref["b"][c]).max() + 1e-300)


def test_ghosts_never_overwrite_unknowns():
    """On the cathode's and the rectangle's lists the post-processing writes only
    entries off the unknowns (what lets the device run a list's entries in
    parallel)."""
    w, p, mw, masks, lists, _ = _cathode()
    T = mw.ghost_targets(lists)
    for f, m in zip("xrp", masks):
        assert T[f] and not any(m[i, j] for i, j in T[f]), f
    pr = mw.er_rect_params(40, 16)
    T = mw.ghost_targets(mw.rect_mw_lists(40, 16, pr))
    for f, m in zip("xrp", mw.mag_masks(40, 16)):
        assert T[f] and not any(m[i, j] for i, j in T[f]), f


def test_ghost_pass_is_linear_in_the_solution():
    """With the port source off (J1r_exc = 0) and gr.Er = 0 the ghosts are
    linear in the planes (a size-independent property of :3026-3264)."""
    w, p, mw, masks, lists, jflc = _cathode()
    p = dict(p, J1r_exc=0.0)
    rng = np.random.default_rng(3)
    sh = masks[0].shape
    A = [rng.standard_normal(sh) + 1j * rng.standard_normal(sh) for _ in range(3)]
    B = [rng.standard_normal(sh) + 1j * rng.standard_normal(sh) for _ in range(3)]
    z = np.zeros(sh)
    ga = mw.mag_ghosts(A, z, w["epsr"], p, lists, jflc)
    gb = mw.mag_ghosts(B, z, w["epsr"], p, lists, jflc)
    gs = mw.mag_ghosts([a + 2.0 * b for a, b in zip(A, B)], z, w["epsr"], p, lists, jflc)
    for c in range(3):
        assert np.max(np.abs(gs[c] - (ga[c] + 2.0 * gb[c]))) <= 1e-12 * np.max(np.abs(gs[c]))


def test_port_of_a_matched_coax_wave():
    """A forward TEM wave Er = A / r exp(-i k z) in the feed seen through the
    reference plane's current and voltage (emfieldModule.hpp:7866-7935): the
    impedance is the coax's eta ln(r2/r1) / (2 pi) to the difference scheme's
    O((k dx)^2), so with that Z0 the plasma reflection vanishes, and with S = the
    identity two-port the forward power at the amplifier is the port's."""
    from oracle import microwave as mw
    ni, nj = 194, 70
    p = mw.cathode_mw_params(ni, nj)
    cells, xf, rf = mw.cathode_mw_blocks(p)
    eta = np.sqrt(mw.MU0 / mw.EPS0)
    Zc = eta * np.log(p["r2"] / p["r1"]) / (2.0 * np.pi)
    k = p["omegam"] * np.sqrt(mw.EPS0 * mw.MU0)
    x = (np.arange(ni + 2) - 0.5) * p["dx"]
    rface = np.maximum((np.arange(nj + 2) - 1.0) * p["dr"], p["dr"])
    A = 1e3
    E1r = A / rface[None, :] * np.exp(-1j * k * x)[:, None]
    z = np.zeros_like(E1r)
    prm = dict(dx=p["dx"], dr=p["dr"], rmin=0.0, omegam=p["omegam"], r1=p["r1"], r2=p["r2"], Z0=Zc, Pmw=8.0,
               S11=0j, S21=1 + 0j, S12=1 + 0j, S22=0j, flag_mwRef=1, i_ref=1, j_out=int(cells[1][4][1]) - 1,
               i_out0=int(cells[0][4][0]), i_out1=int(cells[0][4][1]), jf0=int(rf[1][5][0]), jf1=int(rf[1][5][1]))
    _, res = mw.mw_port_rescale(z, E1r, z, [z, z, z], None, np.ones(z.shape), 1.0, prm)
    assert abs(res["Zp"] / Zc - 1.0) < 1e-3
    assert abs(res["Gamma_p"]) < 1e-3
    assert res["P_fwd_all"] == pytest.approx(res["P_fwd"], rel=1e-12)
    assert res["P_fwd_all"] == pytest.approx(8.0, rel=1e-12)  # rescaled to Pmw
    # without any other field the power through the outlet row is zero
    assert res["P_out"] == 0.0


@pytest.mark.parametrize("shape", [(194, 70), (97, 35), (388, 140)])
def test_package_cathode_microwave_matches_oracle(shape):
    """The package's cathode microwave geometry (blocks and lists, used without
    the oracle by the bench) equals the oracle's, and its segment table is the
    golden fixture."""
    import json
    import os
    from importlib import import_module
    fl = import_module("02_cathode-08_modulerev_b200.fluid")
    from oracle import microwave as mw
    ni, nj = shape
    got = fl.cathode_microwave(ni, nj)
    p = mw.cathode_mw_params(ni, nj)
    cells, xf, rf = mw.cathode_mw_blocks(p)
    for a, b in zip(got["blocks"], (xf, rf, cells)):
        for x, y in zip(a, b):
            assert np.array_equal(np.asarray(x), np.asarray(y))
    here = os.path.dirname(os.path.abspath(__file__))
    with open(os.path.join(here, "golden", "mw_lists_cathode.json")) as f:
        fixture = json.load(f)
    with open(os.path.join(here, "..", "02_cathode-08_modulerev_b200", "data", "mw_lists_cathode.json")) as f:
        assert json.load(f) == fixture
    assert got["lists"] == mw.cathode_mw_lists(cells, fixture)
    assert got["j_flc_00"] == int(cells[1][0][0])
