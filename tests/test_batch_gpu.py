"""Batched instances (I-V sweeps): concurrent steps of independent discharges
from host worker threads give exactly the fields of the same steps run one
instance after another (no state is shared), and the autotuner's choices keep
the solves converged."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FIELDS = ("rhoe", "rhoi", "Te", "phi", "rhon", "rhom", "Uix")


@pytest.mark.parametrize("reuse_tol", [0.0, 1e-3])
def test_batched_steps_equal_sequential(pkg, cuda_device, reuse_tol):
    """reuse_tol > 0: the instances keep their multigrid hierarchies; the decisions
    are made on each instance's own device words, so batched = sequential still."""
    B = pkg.batch
    sizes = ((32, 64), (64, 128))
    specs = B.instance_specs(6, 5, sizes)
    a = B.make_instances(pkg, specs, reuse_tol=reuse_tol)
    b = B.make_instances(pkg, specs, reuse_tol=reuse_tol)
    wall, rc, secs = B.batch_steps(a, steps=3, nthreads=3)
    assert rc == [0] * 6 and wall > 0
    B.sequential_steps(b, steps=3)
    if reuse_tol:
        reused = sum(c["g"].reuse_stats(1, slot)["reuses"] for c in a for slot in range(7))
        assert reused > 0
    for ca, cb in zip(a, b):
        assert ca["P"]["itime"] == cb["P"]["itime"] == 3
        for k in FIELDS:
            assert np.array_equal(ca["fs"].download(k), cb["fs"].download(k)), k
    B.close(a)
    B.close(b)


def test_autotune_keeps_solves_converged(pkg, cuda_device):
    B = pkg.batch
    cases = B.sweep_instances(pkg, n=3, seed=9, sizes=((64, 128),))
    choice = B.autotune(cases, candidates=[(1, 1, True), (2, 1, True), (1, 1, False)], steps=2)
    assert set(choice) == {"64x128"}
    wall, rc, _ = B.batch_steps(cases, steps=2, nthreads=3)
    assert rc == [0, 0, 0]
    B.close(cases)


def test_batched_microwave_updates_follow_each_instance_power(pkg, cuda_device):
    """Instances with the loop's microwave update (here every 3 steps): the
    batched run equals the sequential one bit for bit, each instance ran its
    updates, and its absorbed power was rescaled to its own Pmw (the store's
    Pabs integrates to Pmw after the update, as the port part reports)."""
    B = pkg.batch
    specs = B.instance_specs(4, seed=7, sizes=((32, 64), (64, 128)))
    a = B.make_instances(pkg, specs, microwave=True, ndiv_mw=3)
    b = B.make_instances(pkg, specs, microwave=True, ndiv_mw=3)
    wall, rc, _ = B.batch_steps(a, steps=6, nthreads=2)
    assert rc == [0] * 4
    B.sequential_steps(b, steps=6)
    for ca, cb in zip(a, b):
        assert ca["mw_stats"]["runs"] == 2
        for k in FIELDS + ("Pabs",):
            assert np.array_equal(ca["fs"].download(k), cb["fs"].download(k)), k
        # one more update on the batched instance: its power after the rescale is the instance's Pmw
        out = ca["mwu"].run(ca["gx"], ca["gr"])
        assert out["rc"] == 0 and out["solve"]["converged"] == 1
        assert out["power_sum"] * out["ratio"] == pytest.approx(ca["Pmw"], rel=1e-9)
    assert len({round(c["Pmw"], 6) for c in a}) == 4
    B.close(a)
    B.close(b)
