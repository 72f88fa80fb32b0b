"""GPU transport-coefficient update (FluidModule::update_transport_coef,
fluidModule.hpp:5799-5976) against the oracle on the reference's rate tables
(tests/golden/rate_tables.npz), on the cathode's five fluid blocks and on the
r-z rectangle."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))

OUTPUTS = ("nu_ano_IAT", "Mache", "nu_elas", "nu_exc", "nu_excReso", "nu_excMeta", "nu_ionz", "nu_ionzStep",
           "nu_excStep", "nu_super", "nu_m", "nu_m1", "rate_ionize", "nui_m", "rate_eloss", "delossdeps",
           "mu_para", "mu_xx", "mu_rr", "mu_xr", "mu_perp", "mu_min")
INPUTS = ("rhoe", "rhoi", "rhon", "rhom", "Te", "Bx", "Br", "nu_ano", "nu_ano_IAT", "Uip", "Uix", "rhoUex",
          "Uir", "rhoUer")


def _tables():
    z = np.load(os.path.join(HERE, "golden", "rate_tables.npz"))
    return {k: z[k] for k in z.files if k not in ("dTe", "dEi")}, float(z["dTe"]), float(z["dEi"])


def _run(pkg, ni, nj, flags, seed, dr=None):
    from oracle import fluid
    st = pkg.workloads.plasma_state(ni, nj, seed=seed, dr=dr)
    f, prm = st["fields"], dict(st["prm"])
    tb, dTe, dEi = _tables()
    prm.update(dTe=dTe, dEi=dEi)
    ref = fluid.update_transport_coef(f, tb, prm, flags)
    g = pkg.Grid(ni, nj, [[1, ni]], [[1, nj]])
    fs = pkg.Fields(g)
    for k in INPUTS:
        fs.upload(k, f[k])
    fs.set_flags(flags)
    for k, v in tb.items():
        fs.set_table(k, v)
    fs.update_transport_coef(prm)
    got = {k: fs.download(k) for k in OUTPUTS}
    fs.close()
    g.close()
    return ref, got


def _compare(ref, got, rtol=1e-12):
    for k in OUTPUTS:
        a, b = got[k], ref[k]
        scale = np.abs(b).max() + 1e-300
        err = np.abs(a - b) / (np.abs(b) + 1e-12 * scale)
        assert np.isfinite(a).all(), k
        assert err.max() < rtol, (k, err.max(), np.unravel_index(err.argmax(), err.shape))


def test_transport_cathode_blocks(pkg, cuda_device):
    from oracle import fluid
    ib, jb = fluid.cathode_blocks()
    flags = fluid.cathode_flags(194, 70, ib, jb)
    ref, got = _run(pkg, 194, 70, flags, seed=11, dr=0.014 / 70)
    _compare(ref, got)
    # the anomalous frequency is set on the fluid cells only
    assert (got["nu_ano_IAT"][flags == 0] == 0).all() and (got["nu_ano_IAT"][flags != 0] > 0).all()


@pytest.mark.parametrize("ni,nj,seed", [(64, 48, 1), (130, 33, 2), (1, 1, 3)])
def test_transport_rectangle(pkg, cuda_device, ni, nj, seed):
    from oracle import fluid
    ref, got = _run(pkg, ni, nj, fluid.rectangle_flags(ni, nj), seed)
    _compare(ref, got)


def test_transport_missing_table_is_an_error(pkg, cuda_device):
    from oracle import fluid
    g = pkg.Grid(8, 8, [[1, 8]], [[1, 8]])
    fs = pkg.Fields(g)
    fs.set_flags(fluid.rectangle_flags(8, 8))
    tb, dTe, dEi = _tables()
    for k in list(tb)[:-1]:
        fs.set_table(k, tb[k])
    prm = dict(pkg.workloads.plasma_state(8, 8)["prm"], dTe=dTe, dEi=dEi)
    with pytest.raises(pkg.capi.CathodeError):
        fs.update_transport_coef(prm)
    fs.close()
    g.close()


@pytest.mark.parametrize("adp", [0, 1])
def test_check_cfl(pkg, cuda_device, adp):
    from oracle import fluid
    st = pkg.workloads.sg_state(64, 48, seed=9)
    f = st["fields"]
    g = pkg.Grid(64, 48, [[1, 64]], [[1, 48]])
    fs = pkg.Fields(g)
    for k in ("rhoe", "mu_para", "Te", "rhoUex", "rhoUer"):
        fs.upload(k, f[k])
    prm = dict(dt=1e-10, CFL=0.5, masse=pkg.workloads.MASSE, rmin=0.0, dr=5e-3 / 48, flag_adp_dt=adp)
    got = fs.check_cfl(**prm)
    ref = fluid.check_cfl(f, prm)
    for k in ("rhoe_max", "mu_max", "Te_max", "dt_min", "dt", "CFL"):
        assert got[k] == pytest.approx(ref[k], rel=1e-14), k
    assert got["ue_max"] == pytest.approx(ref["ue_max"], rel=1e-13)
    fs.close()
    g.close()


def test_batched_field_transfers(pkg, cuda_device):
    """upload_many / download_many move the same bits as the per-field calls."""
    import torch
    g = pkg.Grid(40, 24, np.array([[1, 40]]), np.array([[1, 24]]))
    fs = pkg.Fields(g)
    rng = np.random.default_rng(0)
    names = ("rhoe", "rhoi", "Te", "phi")
    src = {k: torch.from_numpy(rng.normal(size=(42, 26))).pin_memory().numpy() for k in names}
    fs.upload_many(src)
    for k in names:
        assert np.array_equal(fs.download(k), src[k]), k
    other = {k: rng.normal(size=(42, 26)) for k in names}
    for k in names:
        fs.upload(k, other[k])
    out = {k: np.zeros((42, 26)) for k in names}
    fs.download_many(out, stream=torch.cuda.current_stream())
    for k in names:
        assert np.array_equal(out[k], other[k]), k
    fs.close()
    g.close()
