"""GPU ion sub-step (solve_Uix_tmp, solve_Uir_tmp, solve_Uip_tmp, solve_rhoi_constTe,
correct_Ui_constTe; fluidModule.hpp:123-2072) against the oracle's loop-by-loop
restatement, on the reference's cathode blocks and on the rectangle."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
INPUTS = ("Uix", "Uir", "Uip", "rhoi", "phi", "Ex", "Er", "Bx", "Br", "rate_ionize", "nui_m", "rhoUix", "rhoUir",
          "rhoUix_wall", "rhoUir_wall")
OUTPUTS = ("Uix", "Uir", "Uip", "rhoi", "rhoUix", "rhoUir", "rhoUix_wall", "rhoUir_wall", "Uix_old", "rhoi_old")


def _rel(a, b):
    return np.abs(a - b).max() / (np.abs(b).max() + 1e-300)


def _case(pkg, kind):
    if kind == "cathode":
        return pkg.fluid.cathode_geometry(), 0.0388, 0.014
    return pkg.fluid.rectangle_geometry(96, 64), 10e-3, 5e-3


@pytest.mark.parametrize("flag_error", [3, 0])
@pytest.mark.parametrize("kind", ["cathode", "rectangle"])
def test_ion_step_fp64(pkg, orc, cuda_device, kind, flag_error):
    import oracle
    from oracle import fluid
    geo, Lz, Lr = _case(pkg, kind)
    ogeo = fluid.cathode_geometry() if kind == "cathode" else fluid.rectangle_geometry(96, 64)
    st = pkg.workloads.ion_state(geo["ni"], geo["nj"], seed=41, Lz=Lz, Lr=Lr)
    f, prm = st["fields"], dict(st["prm"], precision=0, error_cnv_SOR=1e-14, maxITR_SOR=200, flag_error=flag_error)

    def solver(ib, jb):
        def solve(aP, aE, aW, aN, aS, b, i_bl, j_bl):
            return oracle.direct_solve(dict(ni=geo["ni"], nj=geo["nj"], i_bl=i_bl, j_bl=j_bl, aP=aP, aE=aE, aW=aW,
                                            aN=aN, aS=aS, b=b))
        return solve

    ref = fluid.ion_step(f, prm, ogeo, solver(0, 0), solver(0, 0), solver(0, 0))
    g = pkg.Grid(geo["ni"], geo["nj"], geo["ib"], geo["jb"])
    gx = pkg.Grid(geo["ni"], geo["nj"], geo["fxi"], geo["fxj"])
    gr = pkg.Grid(geo["ni"], geo["nj"], geo["fri"], geo["frj"])
    fs = pkg.Fields(g)
    for k in INPUTS:
        fs.upload(k, f[k])
    fs.set_flags(geo["flags"])
    fs.set_ion_geometry(geo)
    res = fs.ion_step(gx, gr, prm)
    assert res["solver_rc"] == 0, res
    for k in OUTPUTS:
        got = fs.download(k)
        assert _rel(got, ref[k]) < 1e-10, (k, _rel(got, ref[k]), np.unravel_index(np.abs(got - ref[k]).argmax(), got.shape))
    for k in ("rhoi", "Uix", "Uir", "Uip"):
        assert res["error_" + k] == pytest.approx(ref["error_" + k], rel=1e-8), k
    fs.close()
    for x in (g, gx, gr):
        x.close()


def test_ion_program_rejects_out_of_range(pkg, cuda_device):
    g = pkg.Grid(16, 8, [[1, 16]], [[1, 8]])
    fs = pkg.Fields(g)
    a = (pkg.capi.IonOp * 1)()
    for f_, v in zip(pkg.capi.ION_OP_FIELDS, (6, 1, 16, 8, 8, 0, 2, 0, 0, 0, 0, 0)):   # target row 10 > nj+1
        setattr(a[0], f_, v)
    import ctypes
    rc = fs._L.cth_ion_program_upload(fs._h, 1, ctypes.addressof(a), 1)
    assert rc == pkg.capi.CTH_ERR_ARG
    fs.close()
    g.close()
