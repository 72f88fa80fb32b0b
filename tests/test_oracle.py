"""CPU checks of the oracle (test infrastructure) against exact solves and
restated reference behaviour."""
import numpy as np
import pytest


def test_smg_restatement_matches_direct_slab(pkg, orc):
    s = pkg.workloads.poisson_slab(ni=128, nj=64, seed=1)
    xd = orc.direct_solve(s)
    xm, rc, it, rel = orc.smg_solve(s, maxITR=40, error_cnv=1e-12)
    assert rc == 0 and rel < 1e-12
    assert np.linalg.norm(xm - xd) / np.linalg.norm(xd) < 1e-10
    r, rn, bn = orc.residual(s, xd)
    assert rn / bn < 1e-12


@pytest.mark.parametrize("kw", [dict(aniso=100.0), dict(aniso=0.01), dict(jump=30.0, diag_extra=0.5),
                                dict(blocks=([[1, 40], [41, 64]], [[1, 32], [10, 20]]))])
def test_smg_restatement_random(pkg, orc, kw):
    s = pkg.workloads.random_mmatrix(64, 32, seed=3, **kw)
    xd = orc.direct_solve(s)
    xm, rc, it, rel = orc.smg_solve(s, maxITR=60, error_cnv=1e-12)
    assert rc == 0, (it, rel)
    assert np.linalg.norm(xm - xd) / np.linalg.norm(xd) < 1e-9


def test_direct_writes_grid_cells_only(pkg, orc):
    s = pkg.workloads.random_mmatrix(20, 12, seed=5, blocks=([[1, 10], [11, 20]], [[1, 12], [3, 6]]))
    x = np.full((22, 14), 7.0)
    orc.direct_solve(s, solution=x)
    m = orc.active_mask(20, 12, s["i_bl"], s["j_bl"])
    assert np.all(x[m == 0] == 7.0)
    assert np.all(x[m == 1] != 7.0)


def test_sor_restatement_fixed_point(pkg, orc):
    # with zero non-grid values SOR's fixed point is the box-union solution
    s = pkg.workloads.random_mmatrix(24, 16, seed=7, diag_extra=0.1)
    xs, n, e = orc.sor_solve(s, alpha=1.9, maxITR=20000, error_cnv=1e-13)
    xd = orc.direct_solve(s)
    assert e <= 1e-13
    assert np.linalg.norm(xs - xd) / np.linalg.norm(xd) < 1e-10


def test_sor_restatement_loop_exit(pkg, orc):
    # do { ncount++; sweep; if (ncount > maxITR) break; } while (error > tol)
    s = pkg.workloads.random_mmatrix(16, 8, seed=1)
    _, n, e = orc.sor_solve(s, alpha=1.9, maxITR=5, error_cnv=1e-30)
    assert n == 6


def _calc_res_np(vn, vo, blocks, eps, flag):
    ib, jb = blocks
    sel = np.zeros(vn.shape, bool)
    for (i0, i1), (j0, j1) in zip(ib, jb):
        sel[i0:i1 + 1, j0:j1 + 1] = True
    d = (vn - vo)[sel]
    o = vo[sel]
    if flag == 0:
        return np.max(np.abs(d))
    if flag == 1:
        return np.sqrt(np.mean(d * d / (o * o + eps)))
    if flag == 2:
        return np.max(np.abs(d)) / np.max(np.abs(o))
    return np.sqrt(np.sum(d * d) / np.sum(o * o))


@pytest.mark.parametrize("flag", [0, 1, 2, 3])
def test_calc_res(orc, flag):
    rng = np.random.default_rng(flag)
    vn = rng.standard_normal((12, 9))
    vo = rng.standard_normal((12, 9))
    blocks = ([[1, 5], [6, 10]], [[1, 7], [2, 4]])
    got = orc.calc_res(10, 7, blocks[0], blocks[1], vn, vo, 1e-3, flag)
    assert got == pytest.approx(_calc_res_np(vn, vo, blocks, 1e-3, flag), rel=1e-13)
