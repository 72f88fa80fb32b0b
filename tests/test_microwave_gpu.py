"""GPU complex solves of the microwave path against the oracle and the
reference's coax calibration fixture (tests/golden/coax_er_deg*.csv)."""
import csv
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))


def _golden(n):
    g = np.zeros((194, 7), complex)
    for r in csv.DictReader(open(os.path.join(HERE, "golden", f"coax_er_deg{n}.csv"))):
        g[int(r["i"]) - 1, int(r["j"]) - 1] = float(r["Er(R)"]) + 1j * float(r["Er(I)"])
    return g


def test_coax_gpu_solve_reproduces_reference_fixture(pkg, cuda_device):
    from oracle import microwave as mw
    p = mw.coax_params()
    s = mw.coax_er_system(p)
    g = pkg.Grid(p["ni"], p["nj"], [[1, p["ni"]]], [[2, p["nj"]]])
    x = np.zeros((p["ni"] + 2, p["nj"] + 2), complex)
    st = g.c5_solve(s["aP"], s["aE"], s["aW"], s["aN"], s["aS"], s["b"], x, maxITR=400, error_cnv=1e-13)
    assert st.converged == 1, st.as_dict()
    ref = mw.solve_c5_direct(s)
    assert np.linalg.norm(x - ref) / np.linalg.norm(ref) < 1e-9
    Es, J, port = mw.coax_postprocess(x, p)
    for n in (0, 5):
        Er, _ = mw.coax_output(Es, J, p, n)
        gold = _golden(n)
        assert np.linalg.norm(Er - gold) / np.linalg.norm(gold) < 5e-6
    g.close()


def test_impedance_test_entry_point_reproduces_reference_fixture(pkg, cuda_device):
    """The impedance test as a product entry point (cth_mw_impedance_test: assembly,
    solve, ghosts, port and rescale on the device) against the reference's own
    calibration output (test/校正/result_deg0, 5 at print precision) and against the
    oracle's direct solve and post-processing."""
    import torch
    from oracle import microwave as mw
    p = mw.coax_params()
    ni, nj = p["ni"], p["nj"]
    g = pkg.Grid(ni, nj, [[1, ni]], [[2, nj]])
    epsr = g.to_device(p["epsr"])
    E = torch.zeros((nj + 2, g.ld), dtype=torch.complex128, device="cuda")
    prm = {k: p[k] for k in ("dx", "dr", "omegam", "J1r_exc", "r1", "r2", "Z0", "Pmw")}
    prm["rmin"] = p["rmin"]
    res = g.impedance_test(epsr, prm, E, maxITR=400, error_cnv=1e-13)
    assert res["solve"]["converged"] == 1, res
    got = np.ascontiguousarray(E[:, :ni + 2].cpu().numpy().T)
    s = mw.coax_er_system(p)
    Es, J, port = mw.coax_postprocess(mw.solve_c5_direct(s), p)
    assert np.linalg.norm(got - Es) / np.linalg.norm(Es) < 1e-9
    assert res["P_fwd"] == pytest.approx(port["P_fwd"], rel=1e-9)
    assert res["V"] == pytest.approx(port["V"], rel=1e-9)
    assert p["J1r_exc"] * res["J1r_exc_factor"] == pytest.approx(J, rel=1e-9)
    for n in (0, 5):
        Er, _ = mw.coax_output(got, p["J1r_exc"] * res["J1r_exc_factor"], p, n)
        gold = _golden(n)
        assert np.linalg.norm(Er - gold) / np.linalg.norm(gold) < 5e-6
    g.close()


def _plasma_helmholtz(ni, nj, seed, nu_lo=1e8, nu_hi=1e10, ne_hi=1e18):
    """Eφ-type complex 5-point system: r-weighted Laplacian + k0^2 eps_p with the
    cold-plasma permittivity eps_p = 1 - wp^2 / (w (w - i nu)), Dirichlet walls."""
    rng = np.random.default_rng(seed)
    w = 2.67e10
    dx = 10e-3 / ni
    dr = 5e-3 / nj
    r = (np.arange(nj + 2) - 0.5) * dr
    ne = 10 ** rng.uniform(15, np.log10(ne_hi), (ni + 2, nj + 2))
    nu = 10 ** rng.uniform(np.log10(nu_lo), np.log10(nu_hi), (ni + 2, nj + 2))
    wp2 = ne * 1.60217662e-19 ** 2 / (9.10938356e-31 * 8.8541878128e-12)
    epsp = 1.0 - wp2 / (w * (w - 1j * nu))
    k02 = (w / 299792458.0) ** 2
    sh = (ni + 2, nj + 2)
    aP = np.zeros(sh, complex); aE = np.zeros(sh, complex); aW = np.zeros(sh, complex)
    aN = np.zeros(sh, complex); aS = np.zeros(sh, complex); b = np.zeros(sh, complex)
    I, J = slice(1, ni + 1), slice(1, nj + 1)
    rc = r[J][None, :]
    rR = 0.5 * (r[1:nj + 1] + r[2:nj + 2])[None, :]
    rL = 0.5 * (r[1:nj + 1] + r[0:nj])[None, :]
    aE[I, J] = dr * dr
    aW[I, J] = dr * dr
    aN[I, J] = rR / rc * dx * dx
    aS[I, J] = rL / rc * dx * dx
    aP[I, J] = aE[I, J] + aW[I, J] + aN[I, J] + aS[I, J] + 1.0 / (rc * rc) * dx * dx * dr * dr \
        - k02 * epsp[I, J] * dx * dx * dr * dr
    b[I, J] = (rng.standard_normal((ni, nj)) + 1j * rng.standard_normal((ni, nj))) * dx * dx * dr * dr
    mask = np.zeros(sh, bool)
    mask[I, J] = True
    return dict(aP=aP, aE=aE, aW=aW, aN=aN, aS=aS, b=b, mask=mask)


@pytest.mark.parametrize("shape", [(64, 32), (100, 37)])
def test_plasma_helmholtz_vs_oracle(pkg, cuda_device, shape):
    from oracle import microwave as mw
    ni, nj = shape
    s = _plasma_helmholtz(ni, nj, seed=ni)
    g = pkg.Grid(ni, nj, [[1, ni]], [[1, nj]])
    x = np.zeros((ni + 2, nj + 2), complex)
    st = g.c5_solve(s["aP"], s["aE"], s["aW"], s["aN"], s["aS"], s["b"], x, maxITR=2000, error_cnv=1e-12)
    assert st.converged == 1, st.as_dict()
    ref = mw.solve_c5_direct(s)
    assert np.linalg.norm(x - ref) / np.linalg.norm(ref) < 1e-8
    g.close()


def _er_case(pkg, ni, nj, seed=2):
    from oracle import microwave as mw
    w = pkg.workloads.mw_er_rect(ni, nj, seed=seed)
    p = mw.er_rect_params(ni, nj)
    for k in ("dx", "dr", "omegam", "J1r_exc", "r1", "r2", "masse"):
        assert p[k] == pytest.approx(w["params"][k], rel=1e-15)
    return w, p, mw


@pytest.mark.parametrize("shape", [(64, 32), (50, 9)])
def test_mw_er_assembly_and_solve_vs_oracle(pkg, cuda_device, shape):
    ni, nj = shape
    w, p, mw = _er_case(pkg, ni, nj)
    ref = mw.er_rect_system(w["ne"], w["nu"], w["epsr"], p)
    g = pkg.Grid(ni, nj, w["i_bl"], w["j_bl"])
    planes = g.mw_er_assemble_dev(g.to_device(w["ne"]), g.to_device(w["nu"]), g.to_device(w["epsr"]), w["params"])
    for name, pl in zip(("aP", "aE", "aW", "aN", "aS", "b"), planes):
        got = pl[:, :ni + 2].cpu().numpy().T
        scale = np.abs(ref[name]).max() + 1e-300
        assert np.max(np.abs(got - ref[name])) / scale < 1e-13, name
    x = g.device_plane(1)[0].to(dtype=__import__("torch").complex128)
    st = g.c5_solve_dev(*planes, x, maxITR=200, error_cnv=1e-12)
    assert st.converged == 1, st.as_dict()
    xr = mw.solve_c5_direct(ref)
    xg = x[:, :ni + 2].cpu().numpy().T
    assert np.linalg.norm(xg - xr) / np.linalg.norm(xr) < 1e-8
    g.close()


def test_mw_er_full_size(pkg, cuda_device):
    """512 x 1024 Er system: converged residual recomputed on the CPU."""
    import torch
    ni, nj = 1024, 512
    w, p, mw = _er_case(pkg, ni, nj)
    g = pkg.Grid(ni, nj, w["i_bl"], w["j_bl"])
    planes = g.mw_er_assemble_dev(g.to_device(w["ne"]), g.to_device(w["nu"]), g.to_device(w["epsr"]), w["params"])
    x = torch.zeros_like(planes[0])
    st = g.c5_solve_dev(*planes, x, maxITR=200, error_cnv=1e-10)
    assert st.converged == 1 and st.iterations <= 60, st.as_dict()
    A = [pl[:, :ni + 2].cpu().numpy().T for pl in planes]
    xg = x[:, :ni + 2].cpu().numpy().T
    r = A[5] - A[0] * xg
    r[:-1] += A[1][:-1] * xg[1:]
    r[1:] += A[2][1:] * xg[:-1]
    r[:, :-1] += A[3][:, :-1] * xg[:, 1:]
    r[:, 1:] += A[4][:, 1:] * xg[:, :-1]
    m = np.zeros(r.shape, bool)
    m[1:ni + 1, 2:nj + 1] = True
    assert np.linalg.norm(r[m]) / np.linalg.norm(A[5][m]) < 2e-10
    g.close()


@pytest.mark.parametrize("kind", ["rectangle", "cathode"])
def test_energy_profile_matches_oracle(pkg, cuda_device, kind):
    """Absorbed microwave power (update_energy_profile, emfieldModule.hpp:7630-7790)
    with the magnetised conductivity tensor: J, Pabs planes and the volume
    integrals against the oracle, random fields, relative 1e-12."""
    import torch
    from oracle import microwave as omw
    geo = pkg.fluid.cathode_geometry() if kind == "cathode" else pkg.fluid.rectangle_geometry(48, 24)
    ni, nj = geo["ni"], geo["nj"]
    rng = np.random.default_rng(7)
    shp = (ni + 2, nj + 2)
    E = {k: rng.normal(size=shp) * 100 + 1j * rng.normal(size=shp) * 100 for k in ("E1x", "E1r", "E1p")}
    f = dict(rhoe=10 ** rng.uniform(15, 18, shp), nu_m1=10 ** rng.uniform(8, 10, shp),
             Bx=rng.uniform(-0.25, 0.25, shp), Br=rng.uniform(-0.25, 0.25, shp))
    dr = 5e-3 / nj
    prm = dict(dx=10e-3 / ni, dr=dr, rmin=0.0, omegam=2.67e10, masse=9.10938356e-31)
    g = pkg.Grid(ni, nj, geo["ib"], geo["jb"])
    gx = pkg.Grid(ni, nj, geo["fxi"], geo["fxj"])
    gr = pkg.Grid(ni, nj, geo["fri"], geo["frj"])
    fs = pkg.Fields(g)
    for k, v in f.items():
        fs.upload(k, v)
    dev = {k: torch.complex(g.to_device(v.real), g.to_device(v.imag)).contiguous() for k, v in E.items()}
    J = [torch.zeros_like(dev["E1x"]) for _ in range(3)]
    r = fs.update_energy_profile(gx, gr, prm, dev["E1x"], dev["E1r"], dev["E1p"], *J)
    blocks = lambda I, Jb: [(int(I[b][0]), int(I[b][1]), int(Jb[b][0]), int(Jb[b][1])) for b in range(len(I))]
    ref, P = omw.energy_profile(E["E1x"], E["E1r"], E["E1p"], f["rhoe"], f["nu_m1"], f["Bx"], f["Br"], prm,
                                blocks(geo["fxi"], geo["fxj"]), blocks(geo["fri"], geo["frj"]),
                                blocks(geo["ib"], geo["jb"]))
    for k, t in zip(("J1x", "J1r", "J1p"), J):
        got = t[:, :ni + 2].cpu().numpy().T
        assert np.abs(got - ref[k]).max() <= 1e-12 * np.abs(ref[k]).max(), k
    for k in ("Pabsx", "Pabsr", "Pabsp", "Pabs"):
        got = fs.download(k)
        assert np.abs(got - ref[k]).max() <= 1e-12 * np.abs(ref[k]).max(), k
    for a, b in zip((r["Px"], r["Pr"], r["Pp"]), P):
        assert a == pytest.approx(b, rel=1e-11)
    fs.close()
    for x in (g, gx, gr):
        x.close()


# ---------------------------------------------------------------------------
# the port / reflection / rescale part of update_energy_profile (:7792-8105)
# ---------------------------------------------------------------------------
def _port_case(pkg, seed=4, Z0=50.0):
    """Cathode grid; Er a forward TEM wave A / r exp(-i k z) on every r-face plus
    noise, Ex and Ephi noise; random Pabs and excitation current."""
    from oracle import microwave as omw
    geo = pkg.fluid.cathode_geometry()
    ni, nj = geo["ni"], geo["nj"]
    p = omw.cathode_mw_params(ni, nj)
    cells, xf, rf = omw.cathode_mw_blocks(p)
    rng = np.random.default_rng(seed)
    shp = (ni + 2, nj + 2)
    k = p["omegam"] * np.sqrt(omw.EPS0 * omw.MU0)
    x = (np.arange(ni + 2) - 0.5) * p["dx"]
    rf_ = (np.arange(nj + 2) - 1.0) * p["dr"]
    rf_[rf_ <= 0] = p["dr"]
    noise = lambda s: s * (rng.standard_normal(shp) + 1j * rng.standard_normal(shp))
    A = 1e3
    E = dict(E1x=noise(5.0), E1r=A / rf_[None, :] * np.exp(-1j * k * x)[:, None] + noise(5.0), E1p=noise(5.0))
    J = [noise(1e4) for _ in range(3)]
    Jexc = [None, noise(1e3), None]
    Pabs = 10 ** rng.uniform(3, 6, shp)
    prm = dict(dx=p["dx"], dr=p["dr"], rmin=0.0, omegam=p["omegam"], r1=p["r1"], r2=p["r2"], Z0=Z0, Pmw=8.0,
               S11=0.1 + 0.05j, S21=0.9 - 0.2j, S12=0.9 - 0.2j, S22=-0.05 + 0.1j, flag_mwRef=1, i_ref=1,
               j_out=int(cells[1][4][1]) - 1, i_out0=int(cells[0][4][0]), i_out1=int(cells[0][4][1]),
               jf0=int(rf[1][5][0]), jf1=int(rf[1][5][1]))
    # an absorbed power below the net forward power, so that the rescale is defined
    _, r1 = omw.mw_port_rescale(E["E1x"], E["E1r"], E["E1p"], J, Jexc, Pabs, 1.0, prm)
    power_sum = 0.3 * r1["P_fwd"] / r1["ratio"]
    return geo, E, J, Jexc, Pabs, prm, power_sum


def _cplx_dev(g, v):
    import torch
    return torch.complex(g.to_device(v.real), g.to_device(v.imag)).contiguous()


@pytest.mark.parametrize("flag", [1, 0])
def test_mw_port_rescale_matches_oracle(pkg, cuda_device, flag):
    from oracle import microwave as omw
    geo, E, J, Jexc, Pabs, prm, power_sum = _port_case(pkg)
    prm["flag_mwRef"] = flag
    ni, nj = geo["ni"], geo["nj"]
    g = pkg.Grid(ni, nj, geo["ib"], geo["jb"])
    fs = pkg.Fields(g)
    fs.upload("Pabs", Pabs)
    dev = {k: _cplx_dev(g, v) for k, v in E.items()}
    dJ = [_cplx_dev(g, v) for v in J]
    dX = [_cplx_dev(g, v) if v is not None else None for v in Jexc]
    res = fs.mw_port_rescale(prm, power_sum, dev["E1x"], dev["E1r"], dev["E1p"], *dJ, *dX)
    want, ref = omw.mw_port_rescale(E["E1x"], E["E1r"], E["E1p"], J, Jexc, Pabs, power_sum, prm)
    for k, v in ref.items():
        assert complex(res[k]) == pytest.approx(complex(v), rel=1e-10, abs=1e-300), k
    if flag:
        assert 0.0 < abs(ref["Gamma_p"]) < 1.0 and ref["pabs_factor"] > 0.0
    got = {"E1x": dev["E1x"], "E1r": dev["E1r"], "E1p": dev["E1p"], "J1x": dJ[0], "J1r": dJ[1], "J1p": dJ[2],
           "J1r_exc": dX[1]}
    for k, t in got.items():
        a = t[:, :ni + 2].cpu().numpy().T
        assert np.abs(a - want[k]).max() <= 1e-12 * np.abs(want[k]).max(), k
        if not flag:
            assert np.array_equal(a, {**E, "J1x": J[0], "J1r": J[1], "J1p": J[2], "J1r_exc": Jexc[1]}[k]), k
    assert np.abs(fs.download("Pabs") - want["Pabs"]).max() <= 1e-12 * np.abs(want["Pabs"]).max()
    fs.close(); g.close()


def test_mw_port_rescale_nonfinite_leaves_planes(pkg, cuda_device):
    """A zero absorbed power (flag_mwRef = 0) gives an infinite ratio: the call
    reports it and rescales nothing."""
    geo, E, J, Jexc, Pabs, prm, _ = _port_case(pkg)
    prm["flag_mwRef"] = 0
    g = pkg.Grid(geo["ni"], geo["nj"], geo["ib"], geo["jb"])
    fs = pkg.Fields(g)
    fs.upload("Pabs", Pabs)
    with pytest.raises(pkg.capi.CathodeError):
        fs.mw_port_rescale(prm, 0.0)
    assert np.array_equal(fs.download("Pabs")[1:-1, 1:-1], Pabs[1:-1, 1:-1]) or \
        np.array_equal(fs.download("Pabs"), Pabs)
    fs.close(); g.close()


def test_mw_divergence_matches_oracle(pkg, cuda_device):
    """output_phase's divergence diagnostics (cth_mw_divergence, outputModule.hpp:43-105)
    on the cathode's six cell blocks at 97 x 35 against the oracle's loops."""
    from oracle import microwave as omw
    ni, nj = 97, 35
    p = omw.cathode_mw_params(ni, nj)
    cells, _, _ = omw.cathode_mw_blocks(p)
    g = pkg.Grid(ni, nj, cells[0], cells[1])
    rng = np.random.default_rng(12)
    shp = (ni + 2, nj + 2)
    F = [rng.standard_normal(shp) + 1j * rng.standard_normal(shp) for _ in range(6)]
    F[3:] = [1e3 * f for f in F[3:]]
    dev = [_cplx_dev(g, f) for f in F]
    divE, divJ, divEJ, rep = g.mw_divergence(*dev, p["dx"], p["dr"], 0.0, p["omegam"])
    want = omw.divergence(*F, dict(p, rmin=0.0), omw.block_mask(ni, nj, *cells))
    assert rep == pytest.approx(want[3], rel=1e-13)
    for got, ref in zip((divE, divJ, divEJ), want[:3]):
        got = np.swapaxes(got[:, :ni + 2].cpu().numpy(), 0, 1)
        assert np.abs(got - ref).max() <= 1e-12 * np.abs(ref).max()
    g.close()
