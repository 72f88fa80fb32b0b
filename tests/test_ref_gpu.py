"""The device path against the reference's own code (oracle/_ref: FluidModule and
InitialModule compiled from the unmodified reference headers; its linear solves
are the exact box-union solve that HYPRE SMG converges to).

* The drop-in: the reference's fluidModule.hpp compiled against
  include/cathode_solver.hpp (oracle/_ref/libref_dropin.so), so that its own
  time step calls solver_SMG on the GPU through libcathode_b200.so, gives the
  reference's fields.
* The device time step (cth_fluid_step) against the reference's loop body on
  its cathode geometry at 194 x 70: relative L2 over the fluid cells of phi,
  n_e, n_i, Te and the cell-centred |E| (outputModule.hpp:310-311) within 1e-8
  after 100 steps in FP64, solver tolerance 1e-14 (both sides converged; the
  remaining difference is the exp() of the device against the C library's,
  which differ by one ulp on ~6 % of arguments)."""
import numpy as np
import pytest

import refpin
import test_fluid_step_gpu as T

pytestmark = pytest.mark.gpu
NORM_FIELDS = ("phi", "rhoe", "rhoi", "Te")


@pytest.fixture(scope="module")
def ref():
    from oracle import ref as R
    if not (R.available() and R.available(dropin=True)):
        pytest.skip("oracle/_ref libraries not built (they are built from the reference sources)")
    return R


def _reference_case(geo, st, cfg, dropin=False):
    c = refpin.case(geo["ni"], geo["nj"], width_neutIn=geo["width_neutIn"], dropin=dropin)
    refpin.put_step(c, st, cfg)
    c.call("update_transport_coef")
    return c


def _norms(get_a, c, m):
    r = c.table("r")
    out = {k: refpin.rel_l2(get_a(k), c.field(k), m) for k in NORM_FIELDS}
    out["|E|"] = refpin.rel_l2(refpin.emag(get_a("Ex"), get_a("Er"), r), refpin.emag(c.field("Ex"), c.field("Er"), r),
                               m)
    return out


@pytest.mark.parametrize("precision", [0, 1])
def test_dropin_runs_the_reference_time_step_on_gpu(pkg, orc, cuda_device, ref, precision):
    """Three whole steps of the reference's own loop body, once with every
    solver_SMG call (ions, potential, electron density and energy, neutrals) on
    the GPU through the header-only drop-in and once with the exact solve."""
    nstep = 3
    geo, ogeo, st, cfg = T.setup(pkg, "cathode", fp64=True)
    for blk in ("ion", "rhoe", "eps", "neutral"):
        cfg["params"][blk].update(error_cnv_SOR=1e-13, maxITR_SOR=100)
    cfg["params"]["phi"].update(error_cnv_SOR_phi=1e-13, maxITR_SOR_phi=100)
    ref.dropin_precision(precision)
    exact = _reference_case(geo, st, cfg)
    gpu = _reference_case(geo, st, cfg, dropin=True)
    for _ in range(nstep):
        exact.call("step")
        gpu.call("step")
    m = refpin.fluid_mask(exact)
    norms = _norms(gpu.field, exact, m)
    for k, v in norms.items():
        assert v < 1e-9, (k, v)


def test_device_steps_match_reference_code(pkg, orc, cuda_device, ref):
    geo, ogeo, st, cfg = T.setup(pkg, "cathode", fp64=True)
    P = cfg["params"]
    c = _reference_case(geo, st, cfg)
    g, gx, gr, fs = T.device_fields(pkg, geo, st, cfg)
    m = refpin.fluid_mask(c)
    done = 0
    for n in (20, 100):
        for _ in range(n - done):
            r = fs.fluid_step(gx, gr, P)
            assert r["solver_rc"] == 0, r
            c.call("step")
        done = n
        assert P["itime"] == c.param("itime") == n
        norms = _norms(fs.download, c, m)
        for k, v in norms.items():
            assert v < 1e-8, (n, k, v)
    # the other prognostic fields follow
    for k in ("rhon", "rhom", "rhoeps", "Uix", "Uir"):
        assert refpin.rel_l2(fs.download(k), c.field(k), m) < 1e-8, k
    fs.close()
    for x in (g, gx, gr):
        x.close()
