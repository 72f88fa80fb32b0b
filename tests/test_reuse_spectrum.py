"""Why a kept multigrid hierarchy needs the in-solve retry: on the slab potential
system (workloads.poisson_slab, 96 x 48), the defect correction with the EXACT
inverse of an old operator A0 applied to a new operator A1 converges with the
spectral radius of I - A0^-1 A1.  A smooth relative change of every coefficient
(what a time step does) gives a radius of about the change itself; the same east
couplings times 1 - 5e-3 -- a row-relative change of 1.7e-3, inside the reuse
tolerance of the GPU test -- shifts the row sums of a nearly singular operator and
gives a radius above 1: no preconditioner built from A0 converges on A1, so the
solve must rebuild (tests/test_reuse_gpu.py::test_graphs_off_agrees uses this
case).  CPU only (scipy sparse LU)."""
import numpy as np
import pytest

sp = pytest.importorskip("scipy.sparse")
sla = pytest.importorskip("scipy.sparse.linalg")

NI, NJ = 96, 48


def _matrix(s):
    idx = -np.ones((NI + 2, NJ + 2), int)
    idx[1:-1, 1:-1] = np.arange(NI * NJ).reshape(NI, NJ)
    rows, cols, vals = [], [], []
    for i in range(1, NI + 1):
        for j in range(1, NJ + 1):
            p = idx[i, j]
            rows.append(p)
            cols.append(p)
            vals.append(s["aP"][i, j])
            for key, (di, dj) in (("aE", (1, 0)), ("aW", (-1, 0)), ("aN", (0, 1)), ("aS", (0, -1))):
                q = idx[i + di, j + dj]
                if q >= 0:   # couplings to non-grid cells are dropped, as in the solver
                    rows.append(p)
                    cols.append(q)
                    vals.append(-s[key][i, j])
    return sp.csc_matrix((vals, (rows, cols)), shape=(NI * NJ, NI * NJ))


def _radius(A0, A1):
    lu = sla.splu(A0)
    op = sla.LinearOperator(A0.shape, matvec=lambda v: v - lu.solve(A1 @ v))
    return float(abs(sla.eigs(op, k=1, which="LM", return_eigenvectors=False, maxiter=5000, tol=1e-8)[0]))


def test_lagged_exact_preconditioner_radius(pkg):
    s = pkg.workloads.poisson_slab(ni=NI, nj=NJ, seed=1)
    A0 = _matrix(s)
    z = np.linspace(0.0, 1.0, NI + 2)[:, None]
    r = np.linspace(0.0, 1.0, NJ + 2)[None, :]
    f = 1.0 + 5e-4 * np.sin(3.0 * z) * np.cos(2.0 * r)
    smooth = dict(s, **{k: s[k] * f for k in ("aP", "aE", "aW", "aN", "aS")})
    rho_smooth = _radius(A0, _matrix(smooth))
    shifted = dict(s, aE=s["aE"] * (1.0 - 5e-3))
    rho_shift = _radius(A0, _matrix(shifted))
    rowrel = float(np.max(np.abs(shifted["aE"] - s["aE"])[1:-1, 1:-1] / np.abs(s["aP"][1:-1, 1:-1])))
    print("radius smooth", rho_smooth, "row-sum shift", rho_shift, "row-relative change", rowrel)
    assert rho_smooth < 1e-3
    assert rowrel < 1e-2 and rho_shift > 1.0
