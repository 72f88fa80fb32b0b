"""The learned warm-start network on the CPU: the oracle's backward pass against
central finite differences (float64, exact network), and the parameter layout
shared by the oracle and the package."""
import numpy as np


def test_oracle_backward_matches_finite_differences():
    from oracle import unet
    rng = np.random.default_rng(0)
    H, W = 8, 16
    vec = unet.init_params(seed=1).astype(np.float64)
    vec += 0.01 * rng.normal(size=vec.size)  # nonzero biases
    vec[-(3 * 32 + 3):] = rng.normal(0.0, 0.2, size=3 * 32 + 3)  # nonzero output layer
    x = rng.normal(size=(H, W, 6))
    dout = rng.normal(size=(H, W, 3))
    out, cache = unet.forward(vec, x, bf16=False)
    g = unet.backward(vec, cache, dout)
    assert g.shape == vec.shape
    # probe parameters of every layer (weights and biases) and of the output layer
    probes = []
    off = 0
    for name, ci, co, _ in unet.layer_shapes():
        nw = co * 9 * ci
        w = vec[off:off + nw].reshape(co, 3, 3, ci)
        idx = np.argwhere(w != 0)
        k = idx[rng.integers(len(idx))]
        probes.append(off + np.ravel_multi_index(tuple(k), w.shape))
        probes.append(off + nw + int(rng.integers(co)))
        off += nw + co
    probes.append(off + 5)
    probes.append(vec.size - 1)
    eps = 1e-6
    for p in probes:
        vp, vm = vec.copy(), vec.copy()
        vp[p] += eps
        vm[p] -= eps
        fp = np.sum(unet.forward(vp, x, bf16=False)[0] * dout)
        fm = np.sum(unet.forward(vm, x, bf16=False)[0] * dout)
        fd = (fp - fm) / (2 * eps)
        assert abs(fd - g[p]) <= 1e-5 * max(1.0, abs(fd)), (p, fd, g[p])


def test_parameter_layout_is_shared(pkg):
    from oracle import unet
    assert [(n, ci, co) for n, ci, co, _ in unet.layer_shapes()] == pkg.learned.layer_shapes()
    a = unet.init_params(seed=3)
    b = pkg.learned.init_params(seed=3)
    assert a.shape == b.shape and np.array_equal(a, b)
    assert unet.nparams() == a.size


def test_bf16_rounding_matches_definition():
    from oracle import unet
    v = np.array([1.0, 1.00390625, 1.005859375, -3.14159, 65504.0, 1e-40], np.float32)
    r = unet.to_bf16(v)
    # nearest bf16: 8 significant bits
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == np.float32(1.0078125)
    assert abs(r[3] + 3.140625) < 1e-6
