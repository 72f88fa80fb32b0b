"""Parity of the CUDA 5-point solves with the oracle, through the C ABI.

SMG replacement: bit-level parity is not defined (HYPRE SMG stops at a
residual tolerance), so the GPU solution is compared with the oracle's exact
solve at relative L2 <= 1e-8 after converging to ||b-Ax||/||b|| < 1e-11, and
the FP64 residual of the returned solution is recomputed on the CPU.
SOR replacement: red-black and lexicographic SOR share the fixed point; both
are run to a tight update tolerance and compared at relative L2 <= 1e-9.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL_SOLVE = 1e-11      # stopping tolerance given to the solver
TOL_PARITY = 1e-8      # relative L2 vs the oracle's exact solve


def _solve(pkg, s, precision, maxITR=40, tol=TOL_SOLVE, x0=None):
    x = np.zeros((s["ni"] + 2, s["nj"] + 2)) if x0 is None else x0
    st = pkg.solver_SMG(s["aP"], s["aE"], s["aW"], s["aN"], s["aS"], s["b"], s["i_bl"], s["j_bl"],
                        len(s["i_bl"]), maxITR, tol, 0, x, precision=precision)
    return x, st


@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("shape", [(96, 48), (200, 100), (37, 23), (5, 3), (64, 1), (1, 40)])
def test_smg_slab_vs_oracle(pkg, orc, cuda_device, precision, shape):
    ni, nj = shape
    s = pkg.workloads.poisson_slab(ni=ni, nj=nj, seed=1)
    x, st = _solve(pkg, s, precision)
    assert st.converged == 1 and st.residual < TOL_SOLVE, st.as_dict()
    ref = orc.direct_solve(s)
    err = np.linalg.norm(x - ref) / np.linalg.norm(ref)
    assert err < TOL_PARITY, err
    _, rn, bn = orc.residual(s, x)
    assert rn / bn < 2 * TOL_SOLVE


@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("kw", [dict(aniso=100.0), dict(aniso=0.01), dict(jump=30.0, diag_extra=0.5),
                                dict(blocks=([[1, 40], [41, 64]], [[1, 32], [10, 20]])),
                                dict(blocks=([[3, 3], [1, 64]], [[1, 32], [5, 5]]))])
def test_smg_random_vs_oracle(pkg, orc, cuda_device, precision, kw):
    s = pkg.workloads.random_mmatrix(64, 32, seed=11, **kw)
    x0 = np.full((66, 34), -3.0)
    x, st = _solve(pkg, s, precision, maxITR=60, x0=x0)
    assert st.converged == 1, st.as_dict()
    ref = orc.direct_solve(s, solution=np.full((66, 34), -3.0))
    m = orc.active_mask(64, 32, s["i_bl"], s["j_bl"])
    assert np.all(x[m == 0] == -3.0)  # only grid cells are written
    err = np.linalg.norm((x - ref)[m == 1]) / np.linalg.norm(ref[m == 1])
    assert err < TOL_PARITY, err


def test_smg_zero_rhs_and_status(pkg, orc, cuda_device):
    s = pkg.workloads.poisson_slab(ni=32, nj=16)
    s["b"][:] = 0.0
    x = np.full((34, 18), 5.0)
    _, st = _solve(pkg, s, 1, x0=x)
    assert st.converged == 1 and st.iterations == 0
    assert np.all(x[1:-1, 1:-1] == 0.0) and np.all(x[0, :] == 5.0)


def test_smg_not_converged_and_nonfinite(pkg, orc, cuda_device):
    s = pkg.workloads.poisson_slab(ni=64, nj=32)
    _, st = _solve(pkg, s, 0, maxITR=1, tol=1e-14)
    assert st.converged == 0 and st.iterations == 1
    s["b"][10, 10] = np.nan
    _, st = _solve(pkg, s, 0)
    assert st.nonfinite == 1 and st.converged == 0


def test_smg_deterministic(pkg, cuda_device):
    s = pkg.workloads.poisson_slab(ni=128, nj=64)
    x1, _ = _solve(pkg, s, 1)
    x2, _ = _solve(pkg, s, 1)
    assert np.array_equal(x1, x2)


@pytest.mark.parametrize("precision", [0, 1])
def test_smg_full_size_device_path(pkg, orc, cuda_device, precision):
    """512 x 1024 r-z slab system on device-resident planes: residual property."""
    s = pkg.workloads.poisson_slab(ni=1024, nj=512, seed=1)
    g = pkg.Grid(s["ni"], s["nj"], s["i_bl"], s["j_bl"])
    planes = [g.to_device(s[k]) for k in ("aP", "aE", "aW", "aN", "aS", "b")]
    x = g.device_plane(1)[0]
    st = g.smg_solve_dev(*planes, x, maxITR=30, error_cnv=1e-10, precision=precision)
    assert st.converged == 1 and st.iterations <= 20, st.as_dict()
    rn, bn = g.residual_dev(*planes, x)
    assert rn / bn < 1e-10
    xh = g.to_host(x)
    _, rn2, bn2 = orc.residual(s, xh)
    assert rn2 / bn2 < 1e-10
    g.close()


@pytest.mark.parametrize("shape", [(24, 16), (31, 9)])
def test_sor_vs_oracle(pkg, orc, cuda_device, shape):
    ni, nj = shape
    s = pkg.workloads.random_mmatrix(ni, nj, seed=2, diag_extra=0.2)
    x0 = np.zeros((ni + 2, nj + 2))
    x0[0, :] = 0.3  # non-grid (ghost) values are read by solver_SOR
    xg = x0.copy()
    st = pkg.solver_SOR(s["aP"], s["aE"], s["aW"], s["aN"], s["aS"], s["b"], s["i_bl"], s["j_bl"], 1,
                        1.9, 50000, 1e-13, 0, xg)
    assert st.converged == 1
    xc, n, e = orc.sor_solve(s, alpha=1.9, maxITR=50000, error_cnv=1e-13, solution=x0.copy())
    assert np.all(xg[0, :] == 0.3)
    err = np.linalg.norm(xg - xc) / np.linalg.norm(xc)
    assert err < 1e-9, err


def test_sor_loop_exit_count(pkg, cuda_device):
    s = pkg.workloads.random_mmatrix(16, 8, seed=1)
    x = np.zeros((18, 10))
    st = pkg.solver_SOR(s["aP"], s["aE"], s["aW"], s["aN"], s["aS"], s["b"], s["i_bl"], s["j_bl"], 1,
                        1.9, 5, 1e-30, 0, x)
    assert st.iterations == 6 and st.converged == 0


def test_smg_graph_and_stream_paths_agree(pkg, orc, cuda_device):
    """The captured-graph solve (device-side cycle loop) and the kernel-by-kernel
    solve give bit-identical results; the graph is reused for new arrays."""
    s = pkg.workloads.poisson_slab(ni=200, nj=100, seed=1)
    g = pkg.Grid(s["ni"], s["nj"], s["i_bl"], s["j_bl"])
    planes = [g.to_device(s[k]) for k in ("aP", "aE", "aW", "aN", "aS", "b")]
    for prec in (0, 1):
        x1 = g.device_plane(1)[0]
        st1 = g.smg_solve_dev(*planes, x1, maxITR=30, error_cnv=1e-11, precision=prec)
        g.set_graphs(False)
        x2 = g.device_plane(1)[0]
        st2 = g.smg_solve_dev(*planes, x2, maxITR=30, error_cnv=1e-11, precision=prec)
        g.set_graphs(True)
        assert st1.converged == 1 and st1.iterations == st2.iterations
        assert st1.residual == st2.residual
        assert bool((x1 == x2).all())
    s2 = pkg.workloads.poisson_slab(ni=200, nj=100, seed=7, V_bias=-5.0)
    planes2 = [g.to_device(s2[k]) for k in ("aP", "aE", "aW", "aN", "aS", "b")]
    x3 = g.device_plane(1)[0]
    st3 = g.smg_solve_dev(*planes2, x3, maxITR=30, error_cnv=1e-11, precision=1)
    ref = orc.direct_solve(s2)
    err = np.linalg.norm(g.to_host(x3) - ref) / np.linalg.norm(ref)
    assert st3.converged == 1 and err < TOL_PARITY
    g.close()


@pytest.mark.parametrize("shape", [(200, 100), (1024, 512)])
def test_smg_fused_tail_matches_level_launches(pkg, cuda_device, shape):
    """The coarse levels of at most 16 rows run as one cluster launch per cycle;
    the same relaxations in the same order as one launch per relaxation, so the
    iteration counts are equal and the solutions agree to rounding."""
    ni, nj = shape
    s = pkg.workloads.poisson_slab(ni=ni, nj=nj, seed=3)
    g = pkg.Grid(s["ni"], s["nj"], s["i_bl"], s["j_bl"])
    planes = [g.to_device(s[k]) for k in ("aP", "aE", "aW", "aN", "aS", "b")]
    for prec in (0, 1):
        g.set_tail(True)
        x1 = g.device_plane(1)[0]
        n0 = g.launch_count()
        st1 = g.smg_solve_dev(*planes, x1, maxITR=30, error_cnv=1e-11, precision=prec)
        n_fused = g.launch_count() - n0
        g.set_tail(False)
        x2 = g.device_plane(1)[0]
        n0 = g.launch_count()
        st2 = g.smg_solve_dev(*planes, x2, maxITR=30, error_cnv=1e-11, precision=prec)
        n_level = g.launch_count() - n0
        assert st1.converged == 1 and st2.converged == 1
        assert st1.iterations == st2.iterations
        a, b = x1.cpu().numpy(), x2.cpu().numpy()
        assert np.linalg.norm(a - b) <= 1e-12 * np.linalg.norm(b)
        assert n_fused < n_level
    g.close()


def test_complex_fused_tail_matches_level_launches(pkg, cuda_device):
    import torch
    from test_microwave_gpu import _er_case
    ni, nj = 128, 64
    w, p, mw = _er_case(pkg, ni, nj)
    g = pkg.Grid(ni, nj, w["i_bl"], w["j_bl"])
    planes = g.mw_er_assemble_dev(g.to_device(w["ne"]), g.to_device(w["nu"]), g.to_device(w["epsr"]), w["params"])
    out = []
    for tail in (True, False):
        g.set_tail(tail)
        x = torch.zeros_like(planes[0])
        st = g.c5_solve_dev(*planes, x, maxITR=200, error_cnv=1e-11)
        assert st.converged == 1, st.as_dict()
        out.append((st.iterations, x.cpu().numpy()))
    assert out[0][0] == out[1][0]
    assert np.linalg.norm(out[0][1] - out[1][1]) <= 1e-10 * np.linalg.norm(out[1][1])
    g.close()


def test_smg_initial_guess(pkg, cuda_device):
    """Solve from a caller's guess: accepted when its relative residual is below
    the threshold (fewer cycles, same stopping rule), rejected otherwise (then
    bit-identical to the zero start); an exact guess stops before any cycle."""
    import torch
    s = pkg.workloads.poisson_slab(ni=200, nj=100, seed=5)
    g = pkg.Grid(s["ni"], s["nj"], s["i_bl"], s["j_bl"])
    planes = [g.to_device(s[k]) for k in ("aP", "aE", "aW", "aN", "aS", "b")]
    for prec in (0, 1):
        x_ref = g.device_plane(1)[0]
        st0 = g.smg_solve_dev(*planes, x_ref, maxITR=30, error_cnv=1e-11, precision=prec)
        assert st0.converged == 1 and st0.guess == 0 and st0.guess_residual == -1.0
        gen = torch.Generator(device=x_ref.device).manual_seed(1)
        near = x_ref * (1.0 + 1e-3 * torch.randn(x_ref.shape, generator=gen, device=x_ref.device,
                                                 dtype=x_ref.dtype))
        x1 = g.device_plane(1)[0]
        st1 = g.smg_solve_guess_dev(*planes, near, x1, max_guess_relres=0.5, maxITR=30, error_cnv=1e-11,
                                    precision=prec)
        assert st1.converged == 1 and st1.guess == 1 and 0.0 < st1.guess_residual < 0.5
        assert st1.iterations < st0.iterations and st1.residual < 1e-11
        far = 1e6 * torch.randn(x_ref.shape, generator=gen, device=x_ref.device, dtype=x_ref.dtype)
        x2 = g.device_plane(1)[0]
        st2 = g.smg_solve_guess_dev(*planes, far, x2, max_guess_relres=0.5, maxITR=30, error_cnv=1e-11,
                                    precision=prec)
        assert st2.guess == -1 and st2.guess_residual > 0.5
        assert st2.iterations == st0.iterations and bool((x2 == x_ref).all())
        x3 = x_ref.clone()
        st3 = g.smg_solve_guess_dev(*planes, x3, x3, max_guess_relres=0.5, maxITR=30, error_cnv=1e-10,
                                    precision=prec)
        assert st3.guess == 1 and st3.iterations == 0 and st3.converged == 1
        assert bool((x3 == x_ref).all())
    g.close()


def test_time_relax_reports_level_times(pkg, cuda_device):
    """The pipelined relaxation timing runs on the last solve's operator and
    leaves the next solve's result unchanged."""
    s = pkg.workloads.poisson_slab(ni=200, nj=100, seed=2)
    g = pkg.Grid(s["ni"], s["nj"], s["i_bl"], s["j_bl"])
    planes = [g.to_device(s[k]) for k in ("aP", "aE", "aW", "aN", "aS", "b")]
    x1 = g.device_plane(1)[0]
    st1 = g.smg_solve_dev(*planes, x1, maxITR=30, error_cnv=1e-11, precision=1)
    for level in (0, 1):
        us, by = g.time_relax(1, level, reps=5)
        assert us > 0 and by > 0
    x2 = g.device_plane(1)[0]
    st2 = g.smg_solve_dev(*planes, x2, maxITR=30, error_cnv=1e-11, precision=1)
    assert st1.iterations == st2.iterations and bool((x1 == x2).all())
    g.close()
