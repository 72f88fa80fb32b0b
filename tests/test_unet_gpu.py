"""The learned warm-start network on the GPU: forward output and parameter
gradients of the library's tensor-core kernels against the numpy oracle (bf16
rounding points emulated for the output, 2e-2 relative L2; gradients measured
against the exact float64 network, see the test), training
on a synthetic regression, and the warm start of the potential solve against
the plain zero start and the previous-step guess."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


@pytest.mark.parametrize("shape", [(16, 32), (24, 40)])
def test_forward_and_gradients_match_oracle(pkg, cuda_device, shape):
    """Device output and gradients against the oracle.  The exact network
    (float64) is the reference for the gradients: the device's error per layer
    must stay within 2.5x (+0.03) of the error that the oracle's own bf16
    rounding points produce (about 0.04-0.17 per layer here: bf16 activations
    flip ReLU gates), and the whole gradient must point the same way."""
    import torch
    from oracle import unet
    H, W = shape
    rng = np.random.default_rng(2)
    vec = unet.init_params(seed=4)
    vec = vec + (0.01 * rng.normal(size=vec.size)).astype(np.float32)
    vec[-(3 * 32 + 3):] = rng.normal(0.0, 0.2, size=3 * 32 + 3)
    x = rng.normal(size=(H, W, 6)).astype(np.float32)
    dout = rng.normal(size=(H, W, 3)).astype(np.float32)
    net = pkg.learned.UNet(H, W, params=vec)
    xt = torch.from_numpy(x).cuda()
    out = net.forward(xt).cpu().numpy()
    ref, cache = unet.forward(vec, x, bf16=True)
    assert _rel(out, ref) < 2e-2, _rel(out, ref)
    net.backward(torch.from_numpy(dout).cuda())
    torch.cuda.synchronize()
    g = net.grads()
    gb = unet.backward(vec, cache, dout)
    _, c64 = unet.forward(vec.astype(np.float64), x.astype(np.float64), bf16=False)
    g64 = unet.backward(vec.astype(np.float64), c64, dout.astype(np.float64))
    off = 0
    rows = []
    for name, ci, co, _ in unet.layer_shapes():
        n = co * 9 * ci + co
        e_dev, e_bf = _rel(g[off:off + n], g64[off:off + n]), _rel(gb[off:off + n], g64[off:off + n])
        rows.append((name, round(e_dev, 4), round(e_bf, 4)))
        off += n
    print(shape, rows)
    for name, e_dev, e_bf in rows:
        assert e_dev <= 2.5 * e_bf + 0.03, (name, e_dev, e_bf)
    cos = float(g @ g64 / (np.linalg.norm(g) * np.linalg.norm(g64)))
    cos_bf = float(gb @ g64 / (np.linalg.norm(gb) * np.linalg.norm(g64)))
    assert cos > cos_bf - 0.01 and cos > 0.95, (cos, cos_bf)
    net.close()


@pytest.mark.parametrize("shape", [(16, 32), (40, 64)])
def test_open_gates_match_oracle_tightly(pkg, cuda_device, shape):
    """With positive inputs, weights and biases every ReLU gate stays open, so the
    bf16 rounding of the activations cannot flip a gate and the network is linear:
    the device (bf16 operands, FP32 accumulation in tensor memory) and the oracle's
    bf16 emulation differ only by accumulation order and the bf16 rounding it moves
    (one unit in the last place, 2^-8 relative, in a few elements).  Measured:
    output 2.1-2.6e-4 relative L2, gradients 1e-5 ... 2.6e-4 per layer against the
    oracle's bf16 gradients.  Bars: 1e-3 and 2e-3 (cosine > 0.99999), twenty to a
    hundred times tighter than the bounds of the gate-flipping case above."""
    import torch
    from oracle import unet
    H, W = shape
    rng = np.random.default_rng(11)
    parts = []
    for name, ci, co, _ in unet.layer_shapes():
        fan = 9 * (6 if name == "e0a" else ci)
        w = rng.uniform(0.0, 2.0 / fan, size=(co, 3, 3, ci))
        if name == "e0a":
            w[..., 6:] = 0.0
        parts += [w.ravel(), np.full(co, 0.1)]
    parts += [rng.normal(0.0, 0.2, size=3 * 32), rng.normal(0.0, 0.2, size=3)]
    vec = np.concatenate(parts).astype(np.float32)
    x = rng.uniform(0.5, 1.5, size=(H, W, 6)).astype(np.float32)
    dout = rng.normal(size=(H, W, 3)).astype(np.float32)
    net = pkg.learned.UNet(H, W, params=vec)
    out = net.forward(torch.from_numpy(x).cuda()).cpu().numpy()
    ref, cache = unet.forward(vec, x, bf16=True)
    assert min(float(a.min()) for k, a in cache["act"].items() if k != "in") > 0.0   # every gate open
    e_out = _rel(out, ref)
    net.backward(torch.from_numpy(dout).cuda())
    torch.cuda.synchronize()
    g = net.grads()
    gb = unet.backward(vec, cache, dout)
    off, rows = 0, []
    for name, ci, co, _ in unet.layer_shapes():
        n = co * 9 * ci + co
        rows.append((name, round(_rel(g[off:off + n], gb[off:off + n]), 5)))
        off += n
    cos = float(g @ gb / (np.linalg.norm(g) * np.linalg.norm(gb)))
    print(shape, "output", e_out, "gradients per layer", rows, "cosine", cos)
    assert e_out < 1e-3, e_out
    assert all(e < 2e-3 for _, e in rows), rows
    assert cos > 0.99999, cos
    net.close()


def test_training_reduces_loss(pkg, cuda_device):
    """Adam on a smooth synthetic target (a blurred, rescaled input channel)."""
    import torch
    H, W = 32, 64
    net = pkg.learned.UNet(H, W, seed=0)
    net.set_loss_weights([0.0, 0.0, 1.0])
    g = torch.Generator(device="cuda").manual_seed(0)
    X = torch.randn((8, H, W, 6), generator=g, device="cuda")
    k = torch.ones((1, 1, 5, 5), device="cuda") / 25.0
    Y = torch.zeros((8, H, W, 3), device="cuda")
    Y[..., 2] = 3.0 * torch.nn.functional.conv2d(X[..., 0].unsqueeze(1), k, padding=2).squeeze(1) + 0.5
    mask = torch.ones((H, W), device="cuda")
    first = last = None
    for ep in range(60):
        tot = 0.0
        for q in range(8):
            tot += net.train_step(X[q].contiguous(), Y[q].contiguous(), mask, H * W, 2e-3)
        if first is None:
            first = tot / 8
        last = tot / 8
    assert last < 0.1 * first, (first, last)
    net.close()


def test_learned_warm_start_of_the_potential(pkg, cuda_device):
    """Snapshots of plain runs (64 x 128 cells, two seeds), training, then steps
    of an unseen discharge with the first potential solve started from zero,
    from the previous step's correction and from the network's guess (the
    previous correction plus the predicted change).  All reach the same
    stopping rule; the trained guess is better than zero and no worse than the
    previous-step guess it refines."""
    L = pkg.learned
    ni, nj = 128, 64
    net = L.UNet(nj, ni, seed=0)
    X, Y, mask = L.collect_snapshots(pkg, net, ni, nj, nsteps=30, seeds=[11, 12, 13])
    stats = L.fit_stats(X, Y, mask)
    net.set_stats(stats)
    Xn, Yn = L.normalise(X, Y, stats)
    losses = L.train(net, Xn, Yn, mask, epochs=10, lr=5e-4)
    assert losses[-1] < losses[0]
    recs = {}
    for ws in (0, 2, 1, 3):
        c = L.make_case(pkg, ni, nj, seed=99, V_bias=25.0)
        L.run_steps(pkg, c, 3, warm_start=2)  # same history for every variant
        recs[ws] = L.run_steps(pkg, c, 6, warm_start=ws, net=net)
        L.close_case(c)
    for ws, rec in recs.items():
        for r in rec:
            assert r["residual"] <= 1e-10
    learned = recs[1]
    assert all(r["guess"] in (1, 2, -1) for r in learned)
    assert learned[0]["net_ran"] == 1
    res = [r["guess_residual"] for r in learned]
    prev = [r["guess_residual"] for r in recs[2]]
    print("first-solve cycles zero/prev/learned:", [np.mean([r["cycles"] for r in recs[w]]) for w in (0, 2, 1)],
          "guess residual prev/learned:", np.mean(prev), np.mean(res))
    # the device takes the better of the network's guess and the previous step's
    assert np.mean(res) < 1.0 and np.mean(res) <= np.mean(prev) * (1.0 + 1e-9)
    # the network's guess alone (mode 3): taken whenever its residual is below
    # the threshold, same stopping rule, no more cycles than from zero
    alone = recs[3]
    assert all(r["net_ran"] == 1 and r["guess"] in (1, -1) for r in alone)
    assert np.mean([r["cycles"] for r in alone]) <= np.mean([r["cycles"] for r in recs[0]])
    net.close()


@pytest.mark.parametrize("shape", [(24, 40), (16, 296), (160, 1024), (512, 1024)])
def test_tensor_core_paths_agree(pkg, cuda_device, shape):
    """The tcgen05 convolutions (accumulator in tensor memory) and the warp-level
    mma.sync convolutions give the same network output and gradients up to
    accumulation order, over partial and several 128-pixel tiles; the two larger
    images reach the tiles of two and four output rows per tensor-core tile.
    The paths sum the input channels in different chunks (32 vs 16), so the bf16
    activations round differently and some ReLU gates flip: outputs agree to
    1e-2, gradients to the bf16 error scale (each path is bounded against the
    exact network in the oracle test; its bf16 oracle sits 4-17 % from it per
    layer), relative 0.2 with cosine > 0.97, where a tiling or layout error
    gives differences of order one."""
    import torch
    from oracle import unet
    H, W = shape
    rng = np.random.default_rng(5)
    vec = unet.init_params(seed=6)
    vec[-(3 * 32 + 3):] = rng.normal(0.0, 0.2, size=3 * 32 + 3)
    x = torch.from_numpy(rng.normal(size=(H, W, 6)).astype(np.float32)).cuda()
    dout = torch.from_numpy(rng.normal(size=(H, W, 3)).astype(np.float32)).cuda()
    res = {}
    for tc in (True, False):
        net = pkg.learned.UNet(H, W, params=vec)
        net.set_tensor_cores(tc)
        out = net.forward(x)
        net.backward(dout)
        net.check()
        res[tc] = (out.cpu().numpy(), net.grads())
        net.close()
    g1, g0 = res[True][1], res[False][1]
    cos = float(g1 @ g0 / (np.linalg.norm(g1) * np.linalg.norm(g0)))
    print(shape, "output", _rel(res[True][0], res[False][0]), "gradients", _rel(g1, g0), "cosine", cos)
    assert _rel(res[True][0], res[False][0]) < 1e-2, _rel(res[True][0], res[False][0])
    assert _rel(g1, g0) < 0.2 and cos > 0.97, (_rel(g1, g0), cos)


def test_bounded_waits_report_and_recover(pkg, cuda_device):
    """The tcgen05 kernel's mbarrier waits are bounded: with the loads withheld
    (nothing in flight) every wait runs out, the kernel frees its tensor memory
    and returns, check() reports the failure once, and the next forward pass on
    the same network is correct again."""
    import torch
    from oracle import unet
    H, W = 16, 40
    rng = np.random.default_rng(3)
    vec = unet.init_params(seed=4)
    vec[-(3 * 32 + 3):] = rng.normal(0.0, 0.2, size=3 * 32 + 3)
    x = rng.normal(size=(H, W, 6)).astype(np.float32)
    net = pkg.learned.UNet(H, W, params=vec)
    net.set_wait_test(True, polls=2048)
    net.forward(torch.from_numpy(x).cuda())
    with pytest.raises(RuntimeError, match="gave up waiting"):
        net.check()
    net.check()  # reported once
    net.set_wait_test(False)
    out = net.forward(torch.from_numpy(x).cuda()).cpu().numpy()
    net.check()
    ref, _ = unet.forward(vec, x, bf16=True)
    assert _rel(out, ref) < 2e-2
    net.close()
