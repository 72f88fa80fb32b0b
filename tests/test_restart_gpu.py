"""Restart files of the device-resident state (cth_restart_write / _wait / _read)
against the reference: the writer gives the bytes of the reference's own
OutputModule::output (oracle/_ref) for the same state, the reader gives the
state of the reader restated loop by loop over the reference's wall segments
(oracle/restart.py, pinned to the reference's file in tests/test_restart.py),
and a write followed by a read restores every variable the format carries back
(Te through eV to 4e-16)."""
import os

import numpy as np
import pytest

import refpin

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def stepped(pkg):
    from oracle import ref as R
    if not R.available():
        pytest.skip("oracle/_ref/libref.so not built (it is built from the reference sources)")
    import tempfile
    import test_fluid_step_gpu as T
    geo, ogeo, st, cfg = T.setup(pkg, "cathode", fp64=True)
    c = refpin.case(geo["ni"], geo["nj"], width_neutIn=geo["width_neutIn"])
    refpin.put_step(c, st, cfg)
    c.call("update_transport_coef")
    for _ in range(3):
        c.call("step")
    d = tempfile.mkdtemp()
    path = c.output(d)
    return dict(c=c, geo=geo, ogeo=ogeo, cfg=cfg, path=path, dir=d)


def _store(pkg, geo, state=None):
    ni, nj = geo["ni"], geo["nj"]
    g = pkg.Grid(ni, nj, geo["ib"], geo["jb"])
    gx = pkg.Grid(ni, nj, geo["fxi"], geo["fxj"])
    gr = pkg.Grid(ni, nj, geo["fri"], geo["frj"])
    fs = pkg.Fields(g)
    fs.set_geometry(geo)
    for k, v in (state or {}).items():
        fs.upload(k, v)
    return g, gx, gr, fs


def _close(objs):
    g, gx, gr, fs = objs
    fs.close()
    for x in (g, gx, gr):
        x.close()


def _coords(pkg, c):
    x, r = pkg.fluid.cell_coordinates(c.ni, c.nj, c.param("dx"), c.param("dr"))
    np.testing.assert_array_equal(x, c.table("x"))
    np.testing.assert_array_equal(r, c.table("r"))
    return x, r


def test_device_writer_is_the_reference_writer(pkg, cuda_device, stepped):
    from oracle import restart
    c = stepped["c"]
    objs = _store(pkg, stepped["geo"], {k: c.field(k) for k in restart.COLUMNS})
    x, r = _coords(pkg, c)
    out = os.path.join(stepped["dir"], "device_restart.csv")
    objs[3].write_restart(out, x, r)
    objs[3].restart_wait()
    assert open(out, "rb").read() == open(stepped["path"], "rb").read()
    _close(objs)


def test_write_is_ordered_before_later_work_on_its_stream(pkg, cuda_device, stepped):
    """The write returns once its copies are queued; a step queued after it on
    the same stream does not reach the file."""
    import torch
    from oracle import restart
    c = stepped["c"]
    geo, cfg = stepped["geo"], stepped["cfg"]
    state = {k: c.field(k) for k in restart.COLUMNS}
    objs = _store(pkg, geo, state)
    g, gx, gr, fs = objs
    fs.set_ion_geometry(geo)
    for k, v in cfg["tables"].items():
        fs.set_table(k, v)
    for k, v in cfg["see"].items():
        fs.set_table(k, v)
    for k in ("Bx", "Br", "Ex", "Er", "nu_ano", "nu_ano_IAT", "Pabs", "rhoUex_wall", "rhoUer_wall"):
        fs.upload(k, c.field(k))
    fs.update_transport_coef(cfg["params"]["transport"])
    for k, v in state.items():      # the reference's planes again (the transport update recomputed rate_ionize)
        fs.upload(k, v)
    x, r = _coords(pkg, c)
    s = torch.cuda.Stream()
    out = os.path.join(stepped["dir"], "device_restart_async.csv")
    fs.write_restart(out, x, r, stream=s)
    P = {k: (dict(v) if isinstance(v, dict) else v) for k, v in cfg["params"].items()}
    P["itime"] = 3
    fs.fluid_step(gx, gr, P, stream=s)
    fs.restart_wait()
    assert open(out, "rb").read() == open(stepped["path"], "rb").read()
    assert not np.array_equal(fs.download("rhoe"), state["rhoe"])   # the step did run
    _close(objs)


def test_device_reader_matches_restated_reader(pkg, cuda_device, stepped):
    from oracle import restart
    c = stepped["c"]
    x, r = _coords(pkg, c)
    dx, dr, V = c.param("dx"), c.param("dr"), c.param("V_bias")
    want = restart.read(open(stepped["path"]).read(), {}, stepped["ogeo"], x, r, dx, dr, V)
    objs = _store(pkg, stepped["geo"])
    g, gx, gr, fs = objs
    info = fs.read_restart(stepped["path"], gx, gr, x, r, dx, dr, V)
    assert info == dict(rows=(c.ni + 2) * (c.nj + 2), variables_read=39, unknown_columns=0)
    for k in restart.REGISTRY + ("Ex", "Er"):
        np.testing.assert_array_equal(fs.download(k), want[k], err_msg=k)
    _close(objs)


def test_round_trip_restores_the_state(pkg, cuda_device, stepped):
    from oracle import restart
    c = stepped["c"]
    x, r = _coords(pkg, c)
    state = {k: c.field(k) for k in restart.COLUMNS}
    a = _store(pkg, stepped["geo"], state)
    path = os.path.join(stepped["dir"], "round_trip.csv")
    a[3].write_restart(path, x, r)
    a[3].restart_wait()
    b = _store(pkg, stepped["geo"])
    b[3].read_restart(path, b[1], b[2], x, r, c.param("dx"), c.param("dr"), c.param("V_bias"))
    fluid = stepped["geo"]["flags"] != 0
    for k in restart.REGISTRY:
        got, ref = b[3].download(k), np.where(np.abs(state[k]) < 1e-100, 0.0, state[k])
        if k == "rhoe":
            ref = ref * fluid
        if k in ("Te", "Te_old"):
            np.testing.assert_allclose(got, ref, rtol=4e-16, atol=0, err_msg=k)
        elif k == "phi":
            np.testing.assert_array_equal(got[fluid], ref[fluid])
        else:
            np.testing.assert_array_equal(got, ref, err_msg=k)
    _close(a)
    _close(b)


def test_reader_rejects_broken_files(pkg, cuda_device, stepped):
    c = stepped["c"]
    x, r = _coords(pkg, c)
    lines = open(stepped["path"]).read().split("\n")
    objs = _store(pkg, stepped["geo"])
    g, gx, gr, fs = objs
    bad = lines[7].split(",")
    bad[3] = "5.0"
    cases = {
        "missing cell": lines[:-3],
        "duplicated cell": lines[:4] + [lines[3]] + lines[4:],
        "coordinate": lines[:7] + [",".join(bad)] + lines[8:],
        "required column": [lines[0].replace("i,j,x,r,", "i,j,x,rr,")] + lines[1:],
        "index out of range": lines[:9] + ["999" + lines[9][lines[9].index(","):]] + lines[10:],
    }
    fs.upload("rhoe", c.field("rhoe"))
    before = fs.download("rhoe")
    for msg, ls in cases.items():
        p = os.path.join(stepped["dir"], "broken.csv")
        open(p, "w").write("\n".join(ls))
        with pytest.raises(pkg.capi.CathodeError) as e:
            fs.read_restart(p, gx, gr, x, r, c.param("dx"), c.param("dr"), c.param("V_bias"))
        assert e.value.code == pkg.capi.CTH_ERR_ARG and msg in str(e.value), (msg, str(e.value))
    np.testing.assert_array_equal(fs.download("rhoe"), before)   # a rejected file changes nothing
    _close(objs)
