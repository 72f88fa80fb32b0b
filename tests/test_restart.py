"""Restart files of the reference's format (CPU part): the oracle's writer gives
the bytes of the reference's own OutputModule::output (compiled from the
unmodified outputModule.hpp into oracle/_ref/libref.so), and the oracle's
reader takes them back to the reference's state."""
import os

import numpy as np
import pytest

import refpin


@pytest.fixture(scope="module")
def stepped(pkg):
    """The reference's own state after 3 steps of the synthetic discharge on the
    cathode, and the restart file its writer makes of it."""
    from oracle import ref as R
    R.build()
    if not R.available():
        pytest.skip("oracle/_ref/libref.so not built: the reference sources are needed to build it")
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
    return dict(c=c, geo=geo, ogeo=ogeo, cfg=cfg, path=path, text=open(path).read())


def test_oracle_writer_is_the_reference_writer(stepped):
    from oracle import restart
    c = stepped["c"]
    fields = {k: c.field(k) for k in restart.COLUMNS}
    assert restart.write(fields, c.table("x"), c.table("r")) == stepped["text"]


def test_oracle_reader_takes_back_the_reference_state(stepped):
    from oracle import restart
    c = stepped["c"]
    ogeo = stepped["ogeo"]
    x, r = c.table("x"), c.table("r")
    s = restart.read(stepped["text"], {}, ogeo, x, r, c.param("dx"), c.param("dr"), c.param("V_bias"))
    fluid = c.int_field("jdgBnd_flc") == 1
    for k in restart.REGISTRY:
        want = c.field(k)
        if k == "rhoe":
            want = want * fluid
        if k in ("Te", "Te_old"):   # K -> eV -> K: two roundings each way
            np.testing.assert_allclose(s[k], want, rtol=4e-16, atol=0, err_msg=k)
        elif k != "phi":            # phi: the reader rewrites the wall ghosts
            np.testing.assert_array_equal(s[k], np.where(np.abs(want) < 1e-100, 0.0, want), err_msg=k)
    np.testing.assert_array_equal(s["phi"][fluid], c.field("phi")[fluid])


def test_oracle_reader_rejects_broken_files(stepped):
    from oracle import restart
    c = stepped["c"]
    x, r = c.table("x"), c.table("r")
    lines = stepped["text"].split("\n")
    args = ({}, stepped["ogeo"], x, r, c.param("dx"), c.param("dr"), 20.0)
    with pytest.raises(ValueError, match="missing cell"):
        restart.read("\n".join(lines[:-3]) + "\n", *args)
    with pytest.raises(ValueError, match="duplicated"):
        restart.read("\n".join(lines[:3] + [lines[2]] + lines[3:]), *args)
    bad = lines[5].split(",")
    bad[2] = "1.0"
    with pytest.raises(ValueError, match="coordinate"):
        restart.read("\n".join(lines[:5] + [",".join(bad)] + lines[6:]), *args)
