"""GPU magnetised 3-component microwave system (cth_mw3) against the oracle's
restatement of solve_Microwave (include/emfieldModule.hpp:2249-2998)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _case(pkg, ni, nj, bmax=0.05, seed=2):
    from oracle import microwave as mw
    w = pkg.workloads.mw3_rect(ni, nj, seed=seed, bmax=bmax)
    p = mw.er_rect_params(ni, nj)
    for k in ("dx", "dr", "omegam", "J1r_exc", "r1", "r2", "masse"):
        assert p[k] == pytest.approx(w["params"][k], rel=1e-15)
    return w, p, mw


def _device(pkg, w):
    g = pkg.Grid(w["ni"], w["nj"], [[1, w["ni"]]], [[1, w["nj"]]])
    planes = [g.to_device(w[k]) for k in ("ne", "nu", "Bx", "Br", "epsr")]
    return g, planes


def _to_ij(t, ni):
    """(..., nj+2, ld) device planes -> numpy (..., ni+2, nj+2)."""
    return np.swapaxes(t[..., :ni + 2].cpu().numpy(), -1, -2)


def _rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


@pytest.mark.parametrize("shape", [(64, 32), (50, 9)])
def test_mw3_assembly_matches_oracle(pkg, cuda_device, shape):
    ni, nj = shape
    w, p, mw = _case(pkg, ni, nj)
    ref = mw.mag_rect_system(w["ne"], w["nu"], w["Bx"], w["Br"], w["epsr"], p)
    g, planes = _device(pkg, w)
    m = pkg.Microwave3(ni, nj)
    m.assemble_dev(*planes, w["params"])
    a, b = m.coefficients()
    a, b = _to_ij(a, ni), _to_ij(b, ni)
    names = (mw.MAG_X, mw.MAG_R, mw.MAG_P)
    for c, comp in enumerate(("x", "r", "p")):
        slots = dict(zip(("P", "E", "W", "N", "S"), range(5)))
        if c == 0:
            slots.update(NE=5, SE=6, NW=7, SW=8, EE=9, WW=10)
        elif c == 1:
            slots.update(NE=5, SE=6, NW=7, SW=8, NN=9, SS=10)
        else:
            slots.update(EE=5, WW=6, NN=7, SS=8)
        for name in names[c]:
            want = ref[comp][name]
            got = a[c, slots[name]]
            scale = np.abs(want).max() + 1e-300
            assert np.max(np.abs(got - want)) / scale < 1e-12, (comp, name)
        scale = np.abs(ref["b"][c]).max() + 1e-300
        assert np.max(np.abs(b[c] - ref["b"][c])) / scale < 1e-12, (comp, "b")
    m.close(); g.close()


def test_mw3_operator_matches_oracle(pkg, cuda_device):
    import torch
    ni, nj = 64, 32
    w, p, mw = _case(pkg, ni, nj)
    ref = mw.mag_rect_system(w["ne"], w["nu"], w["Bx"], w["Br"], w["epsr"], p)
    A, _, _ = mw.mag_rect_matrix(ref)
    rng = np.random.default_rng(7)
    x = rng.standard_normal(A.shape[0]) + 1j * rng.standard_normal(A.shape[0])
    fields = mw.mag_unpack(ref, x)
    g, planes = _device(pkg, w)
    m = pkg.Microwave3(ni, nj)
    m.assemble_dev(*planes, w["params"])
    x3 = m.planes(3)
    for c in range(3):
        # junk off the unknowns must be ignored
        full = fields[c] + (~ref["masks"][c]) * (1.0 + 1.0j)
        x3[c, :, :ni + 2] = torch.from_numpy(np.ascontiguousarray(full.T)).to(x3.device)
    y = _to_ij(m.apply_dev(x3), ni)
    y_ref = mw.mag_unpack(ref, A @ x)
    for c in range(3):
        assert _rel(y[c], y_ref[c]) < 1e-13, c
    m.close(); g.close()


@pytest.mark.parametrize("shape,bmax", [((64, 32), 0.05), ((96, 40), 0.02), ((64, 32), 0.0), ((128, 64), 0.2)])
def test_mw3_solve_matches_direct(pkg, cuda_device, shape, bmax):
    """Against the sparse direct solve; bmax = 0.2 T puts the electron cyclotron
    resonance (0.152 T at w = 2.67e10 rad/s) inside the domain."""
    ni, nj = shape
    w, p, mw = _case(pkg, ni, nj, bmax=bmax)
    ref = mw.mag_rect_system(w["ne"], w["nu"], w["Bx"], w["Br"], w["epsr"], p)
    E_ref = mw.mag_rect_solve(ref)
    g, planes = _device(pkg, w)
    m = pkg.Microwave3(ni, nj)
    m.assemble_dev(*planes, w["params"])
    E, st = m.solve_dev(maxITR=400, error_cnv=1e-12)
    assert st.converged == 1, st.as_dict()
    E = _to_ij(E, ni)
    x, x_ref = mw.mag_pack(ref, E), mw.mag_pack(ref, E_ref)
    assert _rel(x, x_ref) < 1e-8, (_rel(x, x_ref), st.as_dict())
    if bmax == 0.0:
        assert np.max(np.abs(E[2])) == 0.0  # Ephi decouples and has no source
    m.close(); g.close()


def test_mw3_full_size(pkg, cuda_device):
    """512 x 1024 magnetised system: converged, residual recomputed with the
    device operator."""
    import torch
    ni, nj = 1024, 512
    w, p, mw = _case(pkg, ni, nj)
    g, planes = _device(pkg, w)
    m = pkg.Microwave3(ni, nj)
    m.assemble_dev(*planes, w["params"])
    E, st = m.solve_dev(maxITR=300, error_cnv=1e-10)
    print("mw3 512x1024:", st.as_dict())
    assert st.converged == 1, st.as_dict()
    _, b = m.coefficients()
    r = b - m.apply_dev(E)
    rel = float(torch.linalg.vector_norm(r) / torch.linalg.vector_norm(b))
    assert rel < 2e-10, rel
    m.close(); g.close()


def test_mw3_graph_equals_launches(pkg, cuda_device):
    """The captured graph with its device-side loop and the kernel-by-kernel
    path give the same fields bit for bit and the same iteration count."""
    ni, nj = 96, 40
    w, p, mw = _case(pkg, ni, nj)
    g, planes = _device(pkg, w)
    out = {}
    for graphs in (True, False):
        m = pkg.Microwave3(ni, nj)
        m.set_graphs(graphs)
        m.assemble_dev(*planes, w["params"])
        E, st = m.solve_dev(maxITR=200, error_cnv=1e-11)
        E2, st2 = m.solve_dev(maxITR=200, error_cnv=1e-11)  # second call reuses the graph
        assert st.converged == 1 and st2.iterations == st.iterations
        assert np.array_equal(E.cpu().numpy(), E2.cpu().numpy())
        out[graphs] = (E.cpu().numpy(), st.iterations)
        m.close()
    assert out[True][1] == out[False][1]
    assert np.array_equal(out[True][0], out[False][0])
    g.close()


# ---------------------------------------------------------------------------
# the cathode geometry: six blocks per field and the boundary lists of
# InitialModule::makeBoundary (the committed segment table, evaluated on the
# grid's cell blocks)
# ---------------------------------------------------------------------------
SLOTS = ({"P": 0, "E": 1, "W": 2, "N": 3, "S": 4, "NE": 5, "SE": 6, "NW": 7, "SW": 8, "EE": 9, "WW": 10},
         {"P": 0, "E": 1, "W": 2, "N": 3, "S": 4, "NE": 5, "SE": 6, "NW": 7, "SW": 8, "NN": 9, "SS": 10},
         {"P": 0, "E": 1, "W": 2, "N": 3, "S": 4, "EE": 5, "WW": 6, "NN": 7, "SS": 8})


def _cathode(pkg, ni=194, nj=70, bmax=0.05, seed=2):
    import json
    import os
    from oracle import microwave as mw
    w = pkg.workloads.mw3_cathode(ni, nj, seed=seed, bmax=bmax)
    p = mw.cathode_mw_params(ni, nj)
    for k in ("dx", "dr", "omegam", "J1r_exc", "r1", "r2", "masse"):
        assert p[k] == pytest.approx(w["params"][k], rel=1e-15)
    cells, xf, rf = mw.cathode_mw_blocks(p)
    masks = (mw.block_mask(ni, nj, *xf), mw.block_mask(ni, nj, *rf), mw.block_mask(ni, nj, *cells))
    here = os.path.dirname(os.path.abspath(__file__))
    with open(os.path.join(here, "golden", "mw_lists_cathode.json")) as f:
        lists = mw.cathode_mw_lists(cells, json.load(f))
    jflc = int(cells[1][0][0])
    ref = mw.mag_system_lists(w["ne"], w["nu"], w["Bx"], w["Br"], w["epsr"], p, masks, lists, jflc)
    m = pkg.Microwave3(ni, nj, blocks=(xf, rf, cells))
    m.set_boundary(lists, jflc)
    g, planes = _device(pkg, w)
    m.assemble_dev(*planes, w["params"])
    return w, mw, ref, m, g


def test_mw3_cathode_assembly_matches_oracle(pkg, cuda_device):
    ni, nj = 194, 70
    w, mw, ref, m, g = _cathode(pkg, ni, nj)
    a, b = m.coefficients()
    a, b = _to_ij(a, ni), _to_ij(b, ni)
    for c, comp in enumerate(("x", "r", "p")):
        for name, want in ref[comp].items():
            got = a[c, SLOTS[c][name]]
            scale = np.abs(want).max() + 1e-300
            assert np.max(np.abs(got - want)) / scale < 1e-12, (comp, name)
        scale = np.abs(ref["b"][c]).max() + 1e-300
        assert np.max(np.abs(b[c] - ref["b"][c])) / scale < 1e-12, (comp, "b")
    assert np.abs(ref["b"][1]).max() > 0.0  # the feed drives Er
    m.close(); g.close()


def test_mw3_cathode_operator_matches_oracle(pkg, cuda_device):
    import torch
    ni, nj = 194, 70
    w, mw, ref, m, g = _cathode(pkg, ni, nj)
    A, _, _ = mw.mag_rect_matrix(ref)
    rng = np.random.default_rng(11)
    x = rng.standard_normal(A.shape[0]) + 1j * rng.standard_normal(A.shape[0])
    fields = mw.mag_unpack(ref, x)
    x3 = m.planes(3)
    for c in range(3):
        full = fields[c] + (~ref["masks"][c]) * (1.0 + 1.0j)  # junk off the unknowns is ignored
        x3[c, :, :ni + 2] = torch.from_numpy(np.ascontiguousarray(full.T)).to(x3.device)
    y = _to_ij(m.apply_dev(x3), ni)
    y_ref = mw.mag_unpack(ref, A @ x)
    for c in range(3):
        assert _rel(y[c], y_ref[c]) < 1e-13, c
        assert np.all(y[c][~ref["masks"][c]] == 0)
    m.close(); g.close()


@pytest.mark.parametrize("bmax", [0.05, 0.0, 0.2])
def test_mw3_cathode_solve_matches_direct(pkg, cuda_device, bmax):
    """Against the sparse direct solve of the oracle's system on the cathode
    (194 x 70); bmax = 0.2 T crosses the electron cyclotron resonance."""
    ni, nj = 194, 70
    w, mw, ref, m, g = _cathode(pkg, ni, nj, bmax=bmax)
    E_ref = mw.mag_rect_solve(ref)
    E, st = m.solve_dev(maxITR=600, error_cnv=1e-12)
    print("mw3 cathode", bmax, st.as_dict())
    assert st.converged == 1, st.as_dict()
    E = _to_ij(E, ni)
    x, x_ref = mw.mag_pack(ref, E), mw.mag_pack(ref, E_ref)
    assert _rel(x, x_ref) < 1e-8, (_rel(x, x_ref), st.as_dict())
    for c in range(3):
        assert np.all(E[c][~ref["masks"][c]] == 0)
    if bmax == 0.0:
        assert np.max(np.abs(E[2])) == 0.0
    m.close(); g.close()


def test_mw3_set_boundary_rejects_bad_lists(pkg, cuda_device):
    from oracle import microwave as mw
    ni, nj = 194, 70
    p = mw.cathode_mw_params(ni, nj)
    cells, xf, rf = mw.cathode_mw_blocks(p)
    m = pkg.Microwave3(ni, nj, blocks=(xf, rf, cells))
    i0, j0 = int(cells[0][0][0]), int(cells[1][0][0])
    bad = [{("p", "W"): [(i0, j0, 0), (i0, j0, 0)]},          # repeated within a list
           {("p", "W"): [(1, 1, 0)]},                          # not an unknown (inside the cathode body)
           {("p", "W"): [(i0, j0, 8)]}]                        # code outside 0..7
    for lists in bad:
        with pytest.raises(pkg.capi.CathodeError):
            m.set_boundary(lists, j0)
    m.set_boundary({("p", "W"): [(i0, j0, 0)], ("p", "E"): [(i0, j0, 0)]}, j0)  # same row in two lists is fine
    m.close()


def _junk_planes(m, ni, seed):
    """Complex planes with values everywhere: the unknowns and earlier ghosts."""
    import torch
    rng = np.random.default_rng(seed)
    full = [rng.standard_normal((ni + 2, m.nj + 2)) + 1j * rng.standard_normal((ni + 2, m.nj + 2)) for _ in range(3)]
    x3 = m.planes(3)
    for c in range(3):
        x3[c, :, :ni + 2] = torch.from_numpy(np.ascontiguousarray(full[c].T)).to(x3.device)
    return full, x3


@pytest.mark.parametrize("geometry", ["cathode", "rectangle"])
def test_mw3_ghosts_match_oracle(pkg, cuda_device, geometry):
    """The boundary post-processing on planes with values everywhere (the ghosts
    read before they are written are earlier ones), gr.Er random: every entry of
    the three planes as the oracle's restatement, to rounding."""
    import torch
    if geometry == "cathode":
        ni, nj = 194, 70
        w, mw, ref, m, g = _cathode(pkg, ni, nj)
        from oracle import microwave as omw
        p = omw.cathode_mw_params(ni, nj)
        cells, _, _ = omw.cathode_mw_blocks(p)
        import json, os
        with open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "mw_lists_cathode.json")) as f:
            lists = omw.cathode_mw_lists(cells, json.load(f))
        jflc = int(cells[1][0][0])
    else:
        ni, nj = 64, 32
        w, p, mw = _case(pkg, ni, nj)
        g, planes = _device(pkg, w)
        m = pkg.Microwave3(ni, nj)
        m.assemble_dev(*planes, w["params"])
        lists, jflc = mw.rect_mw_lists(ni, nj, p), 0
    full, x3 = _junk_planes(m, ni, 5)
    er_dc = np.random.default_rng(6).standard_normal((ni + 2, nj + 2))
    m.fill_ghosts(x3, g.to_device(w["epsr"]), w["params"], Er_dc=g.to_device(er_dc))
    got = _to_ij(x3, ni)
    want = mw.mag_ghosts(full, er_dc, w["epsr"], p, lists, jflc)
    targets = mw.ghost_targets(lists)
    for c, f in enumerate("xrp"):
        assert np.max(np.abs(got[c] - want[c])) <= 1e-14 * np.max(np.abs(want[c])), f
        changed = np.argwhere(want[c] != full[c])
        assert len(changed) > 0 and all((int(a), int(b)) in targets[f] for a, b in changed)
    m.close(); g.close()


def test_mw3_solve_then_ghosts_matches_direct(pkg, cuda_device):
    """solve_Microwave end to end on the cathode: the solve writes the unknowns
    and keeps the earlier ghosts, the post-processing writes the new ones; all
    entries against the oracle's direct solve and ghost pass."""
    ni, nj = 194, 70
    w, mw, ref, m, g = _cathode(pkg, ni, nj)
    from oracle import microwave as omw
    import json, os
    p = omw.cathode_mw_params(ni, nj)
    cells, _, _ = omw.cathode_mw_blocks(p)
    with open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "mw_lists_cathode.json")) as f:
        lists = omw.cathode_mw_lists(cells, json.load(f))
    full, E = _junk_planes(m, ni, 9)
    E, st = m.solve_dev(maxITR=600, error_cnv=1e-12, out=E)
    assert st.converged == 1
    got0 = _to_ij(E, ni)
    for c in range(3):
        off = ~ref["masks"][c]
        assert np.array_equal(got0[c][off], full[c][off])  # ghosts kept
    er_dc = np.zeros((ni + 2, nj + 2))
    m.fill_ghosts(E, g.to_device(w["epsr"]), w["params"], Er_dc=g.to_device(er_dc))
    got = _to_ij(E, ni)
    E_ref = mw.mag_rect_solve(ref)
    start = [np.where(ref["masks"][c], E_ref[c], full[c]) for c in range(3)]
    want = mw.mag_ghosts(start, er_dc, w["epsr"], p, lists, int(cells[1][0][0]))
    for c in range(3):
        on = ref["masks"][c]
        assert _rel(got[c][on], want[c][on]) < 1e-8, c
        assert _rel(got[c], want[c]) < 1e-8, c
    m.close(); g.close()


def test_mw3_set_cycle(pkg, cuda_device):
    """More smoothing per level re-captures the solve and reaches the same
    solution; sweeps outside 1..8 are refused."""
    ni, nj = 64, 32
    w, p, mw = _case(pkg, ni, nj)
    ref = mw.mag_rect_system(w["ne"], w["nu"], w["Bx"], w["Br"], w["epsr"], p)
    x_ref = mw.mag_pack(ref, mw.mag_rect_solve(ref))
    g, planes = _device(pkg, w)
    m = pkg.Microwave3(ni, nj)
    m.assemble_dev(*planes, w["params"])
    for nu in ((1, 1), (2, 3), (1, 1)):
        m.set_cycle(*nu)
        E, st = m.solve_dev(maxITR=200, error_cnv=1e-12)
        assert st.converged == 1
        assert _rel(mw.mag_pack(ref, _to_ij(E, ni)), x_ref) < 1e-8, nu
    for bad in ((0, 1), (1, 9)):
        with pytest.raises(pkg.capi.CathodeError):
            m.set_cycle(*bad)
    m.close(); g.close()


@pytest.mark.parametrize("geometry", ["rectangle", "cathode"])
def test_mw3_gauss_seidel_matches_direct(pkg, cuda_device, geometry):
    """The block Gauss-Seidel preconditioner reaches the direct solution, in the
    captured graph and kernel by kernel alike."""
    if geometry == "cathode":
        w, mw, ref, m, g = _cathode(pkg, 194, 70)
        ni = 194
    else:
        ni, nj = 96, 40
        w, p, mw = _case(pkg, ni, nj)
        ref = mw.mag_rect_system(w["ne"], w["nu"], w["Bx"], w["Br"], w["epsr"], p)
        g, planes = _device(pkg, w)
        m = pkg.Microwave3(ni, nj)
        m.assemble_dev(*planes, w["params"])
    x_ref = mw.mag_pack(ref, mw.mag_rect_solve(ref))
    m.set_preconditioner(1)
    its = []
    for graphs in (True, False):
        m.set_graphs(graphs)
        E, st = m.solve_dev(maxITR=600, error_cnv=1e-12)
        assert st.converged == 1, st.as_dict()
        assert _rel(mw.mag_pack(ref, _to_ij(E, ni)), x_ref) < 1e-8
        its.append(st.iterations)
    assert its[0] == its[1]
    print("mw3 gauss-seidel", geometry, its[0])
    with pytest.raises(pkg.capi.CathodeError):
        m.set_preconditioner(2)
    m.close(); g.close()


@pytest.mark.parametrize("geometry,bmax,prec", [("rectangle", 0.05, 0), ("rectangle", 0.2, 1), ("cathode", 0.05, 0),
                                                ("cathode", 0.2, 0), ("cathode", 0.05, 1)])
def test_mw3_mixed_precision_matches_direct(pkg, cuda_device, geometry, bmax, prec):
    """FP32 complex V-cycles inside the FP64 BiCGStab reach the direct solution
    to the same tolerance as the FP64 preconditioner (the recurrence, the
    operator products and the stopping test stay FP64), in the captured graph
    and kernel by kernel alike; switching back to FP64 gives the FP64 result.
    Iterations: the same on the rectangle; 1.6-1.8 times the FP64 count on the
    cathode (a longer, more indefinite domain, where the preconditioner's
    rounding is amplified), which the test records but does not bound."""
    if geometry == "cathode":
        w, mw, ref, m, g = _cathode(pkg, 194, 70, bmax=bmax)
        ni = 194
    else:
        ni, nj = 96, 40
        w, p, mw = _case(pkg, ni, nj, bmax=bmax)
        ref = mw.mag_rect_system(w["ne"], w["nu"], w["Bx"], w["Br"], w["epsr"], p)
        g, planes = _device(pkg, w)
        m = pkg.Microwave3(ni, nj)
        m.assemble_dev(*planes, w["params"])
    x_ref = mw.mag_pack(ref, mw.mag_rect_solve(ref))
    m.set_preconditioner(prec)
    E64, st64 = m.solve_dev(maxITR=800, error_cnv=1e-12)
    assert st64.converged == 1, st64.as_dict()
    m.set_precision(pkg.capi.CTH_PREC_MIXED)
    its = []
    for graphs in (True, False):
        m.set_graphs(graphs)
        E, st = m.solve_dev(maxITR=800, error_cnv=1e-12)
        assert st.converged == 1, st.as_dict()
        assert _rel(mw.mag_pack(ref, _to_ij(E, ni)), x_ref) < 1e-8
        its.append(st.iterations)
    assert its[0] == its[1]
    print("mw3 mixed", geometry, bmax, prec, "iterations fp64", st64.iterations, "mixed", its[0])
    if geometry == "rectangle":
        assert its[0] <= st64.iterations + 2
    m.set_precision(pkg.capi.CTH_PREC_FP64)
    E2, st2 = m.solve_dev(maxITR=800, error_cnv=1e-12)
    assert st2.iterations == st64.iterations
    assert np.array_equal(E2.cpu().numpy(), E64.cpu().numpy())
    with pytest.raises(pkg.capi.CathodeError):
        m.set_precision(7)
    m.close(); g.close()


@pytest.mark.parametrize("geometry", ["rectangle", "cathode"])
def test_mw3_initial_guess(pkg, cuda_device, geometry):
    """The solve from an initial guess: the converged solution itself ends the
    solve at once (0 iterations, or 1 where its true residual b - A x sits just
    above the tolerance that the recurrence's residual met); the solution scaled
    by 1.001 (relative residual 1e-3) converges in fewer iterations to the direct
    solution; a guess
    worse than zero is rejected on the device and the result is the zero-start
    solve bit for bit, in the graph and kernel by kernel."""
    import torch
    if geometry == "cathode":
        w, mw, ref, m, g = _cathode(pkg, 194, 70)
        ni = 194
    else:
        ni, nj = 96, 40
        w, p, mw = _case(pkg, ni, nj)
        ref = mw.mag_rect_system(w["ne"], w["nu"], w["Bx"], w["Br"], w["epsr"], p)
        g, planes = _device(pkg, w)
        m = pkg.Microwave3(ni, nj)
        m.assemble_dev(*planes, w["params"])
    x_ref = mw.mag_pack(ref, mw.mag_rect_solve(ref))
    for graphs in (True, False):
        m.set_graphs(graphs)
        E0, st0 = m.solve_dev(maxITR=600, error_cnv=1e-12)
        assert st0.converged == 1 and st0.guess == 0
        E1, st1 = m.solve_dev(maxITR=600, error_cnv=1e-12, x0=E0)
        assert st1.guess == 1 and st1.iterations <= 1 and st1.converged == 1, st1.as_dict()
        if st1.iterations == 0:
            assert torch.equal(E1, E0)
        assert _rel(mw.mag_pack(ref, _to_ij(E1, ni)), x_ref) < 1e-8
        # the solution at 1.001 times the excitation: residual 1e-3 ||b|| (the system is linear)
        Ep = E0 * 1.001
        E2, st2 = m.solve_dev(maxITR=600, error_cnv=1e-12, x0=Ep)
        assert st2.guess == 1 and st2.guess_residual == pytest.approx(1e-3, rel=1e-3) and st2.converged == 1
        assert st2.iterations < st0.iterations, (st2.iterations, st0.iterations)
        assert _rel(mw.mag_pack(ref, _to_ij(E2, ni)), x_ref) < 1e-8
        E3, st3 = m.solve_dev(maxITR=600, error_cnv=1e-12, x0=E0 * 1e6)
        assert st3.guess == -1 and st3.iterations == st0.iterations
        assert torch.equal(E3, E0)
        print("mw3 guess", geometry, graphs, "zero", st0.iterations, "perturbed", st2.iterations,
              f"guess residual {st2.guess_residual:.1e}")
    m.close(); g.close()
