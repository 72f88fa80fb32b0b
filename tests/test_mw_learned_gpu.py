"""The learned warm start of the microwave solve: the network's input features
against a numpy restatement, the untrained network (zero output layer) reproducing
the previous-fields start exactly, and a short training whose guess starts the
solve without changing its answer."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
NI, NJ = 128, 64


def _discharge(pkg, **kw):
    return pkg.discharge.RectangleDischarge(pkg, NI, NJ, seed=4, ndiv_mw=5, **kw)


def test_mw_features_match_numpy(pkg, cuda_device):
    import torch
    L = pkg.learned
    d = _discharge(pkg)
    for _ in range(5):
        d.step()
    net = L.UNet(NJ, NI, cin=L.MW_CIN, cout=L.MW_COUT)
    gen = torch.Generator(device="cuda").manual_seed(3)
    E = torch.randn(d.e3.shape, dtype=torch.complex128, device="cuda", generator=gen)
    x = net.mw_features(d.fs, E, escale=0.5).cpu().numpy()
    ne, nu, Bx, Br = (d.fs.download(k) for k in ("rhoe", "nu_m1", "Bx", "Br"))
    En = E.cpu().numpy()
    want = np.zeros((NJ, NI, 9), np.float64)
    want[..., 0] = np.log10(np.maximum(ne[1:NI + 1, 1:NJ + 1], 1.0)).T
    want[..., 1] = np.log10(np.maximum(nu[1:NI + 1, 1:NJ + 1], 1.0)).T
    want[..., 2] = np.sqrt(Bx ** 2 + Br ** 2)[1:NI + 1, 1:NJ + 1].T
    for c in range(3):
        want[..., 3 + 2 * c] = 0.5 * En[c, 1:NJ + 1, 1:NI + 1].real
        want[..., 4 + 2 * c] = 0.5 * En[c, 1:NJ + 1, 1:NI + 1].imag
    np.testing.assert_allclose(x, want, rtol=2e-6, atol=1e-30)
    net.close()
    d.close()


def test_untrained_network_guess_is_the_previous_fields(pkg, cuda_device):
    """A zero output layer predicts no change: the guess equals the previous
    fields scaled to the new excitation bit for bit, so the update with the
    network takes the same start, iterations and result as the previous-fields
    warm start."""
    import torch
    L = pkg.learned
    net = L.UNet(NJ, NI, cin=L.MW_CIN, cout=L.MW_COUT)
    a = _discharge(pkg)
    b = _discharge(pkg)
    a.mw.set_net(net)
    b2 = pkg.discharge.MicrowaveUpdate(b.fs, b.m3, b.mw_params, b.port, ndiv_mw=5, E3=b.e3, J3=b.j3, warm_start=True)
    b.mw.close()
    b.mw = b2
    for _ in range(10):
        ra = a.step()
        rb = b.step()
        if "mw" in ra:
            assert ra["mw"]["solve"]["iterations"] == rb["mw"]["solve"]["iterations"]
            assert ra["mw"]["solve"]["guess"] == rb["mw"]["solve"]["guess"]
    assert ra["mw"]["solve"]["guess"] == 1              # the second update started from the previous fields
    assert torch.equal(a.e3, b.e3)
    g = net.mw_guess(a.fs, a.e3, 2.0, 3.0)
    assert torch.equal(g, a.e3 * 1.5)
    a.close()
    b.close()
    net.close()


def test_trained_network_starts_the_solve_without_changing_it(pkg, cuda_device):
    import torch
    L = pkg.learned
    net = L.UNet(NJ, NI, cin=L.MW_CIN, cout=L.MW_COUT)
    X, Y, mask = L.collect_mw_snapshots(pkg, net, NI, NJ, runs=3, nsteps=30, ndiv_mw=5)
    assert X.shape[1:] == (NJ, NI, 9) and Y.shape[1:] == (NJ, NI, 6) and X.shape[0] >= 6
    stats = L.mw_fit_stats(X, Y, mask)
    net.set_stats(stats)
    Xn, Yn = L.mw_normalise(X, Y, stats)
    losses = L.mw_train(net, Xn, Yn, mask, epochs=3)
    assert losses[-1] < losses[0]
    net.check()
    rec = L.mw_evaluate(pkg, net, NI, NJ, runs=1, nsteps=30, ndiv_mw=5, tol=1e-8)
    assert rec["updates"] >= 3
    # every start reaches the tolerance; the network's guess is either taken or rejected on the device
    d = _discharge(pkg)
    d.mw.set_net(net)
    ref = _discharge(pkg)
    for _ in range(15):
        r = d.step()
        ref.step()
        if "mw" in r:
            assert r["mw"]["rc"] == 0 and r["mw"]["solve"]["converged"] == 1
    a, b = d.e3.cpu().numpy(), ref.e3.cpu().numpy()
    assert np.linalg.norm(a - b) <= 1e-7 * np.linalg.norm(b)
    print("learned microwave", {k: rec[k] for k in ("zero", "previous", "network", "network_rejected")})
    d.close()
    ref.close()
    net.close()
