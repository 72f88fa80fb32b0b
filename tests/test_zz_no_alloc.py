"""The allocation-free residual entry point agrees with the grid-based one.

cth_residual_noalloc exists for callers that may not allocate device memory
when they need a residual (their own pool owns the device memory, or a loop
cannot take the synchronisation an allocation may cause).  It keeps its
scratch in a static device array shared by all calls, so this test calls it
several times in a row with different inputs, small then large then small
again (a later call must not see an earlier call's mask or partial sums, in
particular the leftovers of a larger plane), and compares each result with
cth_residual_dev.
This file is collected last so that a stop-at-first-failure run has already
run every other test.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _noalloc(pkg, g, planes, x, r):
    import torch
    L = pkg.capi.load()
    ib = np.ascontiguousarray(g.i_bl.reshape(-1), dtype=np.int32)
    jb = np.ascontiguousarray(g.j_bl.reshape(-1), dtype=np.int32)
    rn = ctypes.c_double()
    bn = ctypes.c_double()
    s = torch.cuda.current_stream()
    rc = L.cth_residual_noalloc(g.ni, g.nj, g.ld, ib.ctypes.data_as(pkg.capi._ip), jb.ctypes.data_as(pkg.capi._ip),
                                g.n_bl, *[p.data_ptr() for p in planes], x.data_ptr(), r.data_ptr(),
                                ctypes.byref(rn), ctypes.byref(bn), s.cuda_stream)
    pkg.capi.check(rc, allow_positive=False)
    return rn.value, bn.value


def test_residual_noalloc_matches_grid_entry_point(pkg, cuda_device):
    import torch
    cases = [
        pkg.workloads.random_mmatrix(96, 40, seed=21, blocks=([[1, 60], [61, 96]], [[1, 40], [8, 30]])),
        pkg.workloads.poisson_slab(ni=200, nj=100, seed=3),
    ]
    for s in cases + cases[::-1]:
        g = pkg.Grid(s["ni"], s["nj"], s["i_bl"], s["j_bl"])
        planes = [g.to_device(s[k]) for k in ("aP", "aE", "aW", "aN", "aS", "b")]
        rng = np.random.default_rng(s["ni"])
        x = g.to_device(rng.standard_normal((s["ni"] + 2, s["nj"] + 2)))
        r_ref = g.device_plane(1)[0]
        rn_ref, bn_ref = g.residual_dev(*planes, x, r_ref)
        r_new = torch.full_like(r_ref, 123.0)
        rn, bn = _noalloc(pkg, g, planes, x, r_new)
        torch.cuda.synchronize()
        # both entry points write r over the (nj+2) x (ni+2) index space only
        n = s["ni"] + 2
        assert torch.equal(r_new[:, :n], r_ref[:, :n])
        assert rn == pytest.approx(rn_ref, rel=1e-14, abs=0.0)
        assert bn == pytest.approx(bn_ref, rel=1e-14, abs=0.0)
        g.close()


def test_residual_noalloc_rejects_oversize(pkg, cuda_device):
    import torch
    L = pkg.capi.load()
    ni, nj = 4094, 4094
    ld = 4096
    ib = np.array([1, ni], dtype=np.int32)
    jb = np.array([1, nj], dtype=np.int32)
    d = torch.zeros(1, dtype=torch.float64, device="cuda")
    rc = L.cth_residual_noalloc(ni, nj, ld, ib.ctypes.data_as(pkg.capi._ip), jb.ctypes.data_as(pkg.capi._ip), 1,
                                *([d.data_ptr()] * 8), None, None, None)
    assert rc == pkg.capi.CTH_ERR_ARG
    assert "CTH_NOALLOC_MAX_PLANE" in pkg.capi.last_error()
