"""GPU neutral sweeps (update_rhon, update_rhom; fluidModule.hpp:4963-5792)
against the oracle's loop-by-loop restatement, on the reference's cathode blocks
(with its gas inlet) and on the rectangle with an inlet on the outer wall."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
OUTPUTS = ("rhon", "rhom", "rhoUnx", "rhoUnr", "rhoUnx_wall", "rhoUnr_wall", "rhoUmx", "rhoUmr", "rhoUmx_wall",
           "rhoUmr_wall", "rhon_old", "rhom_old")


def _rel(a, b):
    return np.abs(a - b).max() / (np.abs(b).max() + 1e-300)


@pytest.mark.parametrize("kind", ["cathode", "rectangle"])
def test_neutrals_fp64(pkg, orc, cuda_device, kind):
    import oracle
    from oracle import fluid
    if kind == "cathode":
        geo, ogeo, Lz, Lr = pkg.fluid.cathode_geometry(), fluid.cathode_geometry(), 0.0388, 0.014
    else:
        geo = pkg.fluid.rectangle_geometry(96, 64, width_neutIn=2.03e-3)
        ogeo, Lz, Lr = fluid.rectangle_geometry(96, 64), 10e-3, 5e-3
    st = pkg.workloads.neutral_state(geo["ni"], geo["nj"], seed=51, Lz=Lz, Lr=Lr)
    f = st["fields"]
    prm = dict(st["prm"], precision=0, error_cnv_SOR=1e-14, maxITR_SOR=200, xL=geo["xL"], x6=geo["x6"],
               width_neutIn=geo["width_neutIn"])

    def solve(aP, aE, aW, aN, aS, b, ib, jb):
        return oracle.direct_solve(dict(ni=geo["ni"], nj=geo["nj"], i_bl=ib, j_bl=jb, aP=aP, aE=aE, aW=aW, aN=aN,
                                        aS=aS, b=b))

    ref = fluid.update_neutrals(f, prm, ogeo, solve)
    g = pkg.Grid(geo["ni"], geo["nj"], geo["ib"], geo["jb"])
    fs = pkg.Fields(g)
    for k, v in f.items():
        fs.upload(k, v)
    fs.set_flags(geo["flags"])
    res = fs.update_neutrals(prm, geo["pos_boxes"])
    assert res["solver_rc"] == 0, res
    for k in OUTPUTS:
        got = fs.download(k)
        assert _rel(got, ref[k]) < 1e-10, (k, _rel(got, ref[k]), np.unravel_index(np.abs(got - ref[k]).argmax(), got.shape))
    assert res["error_rhon"] == pytest.approx(ref["error_rhon"], rel=1e-6)
    assert res["error_rhom"] == pytest.approx(ref["error_rhom"], rel=1e-6)
    fs.close()
    g.close()
