"""CPU restatement of the learned warm-start network (numpy).

TEST INFRASTRUCTURE ONLY (checker; the product never imports it).

The network has no counterpart in the reference: it is the 4-level U-Net of the
device library (3x3 convolutions with ReLU, 2x2 average pooling, nearest 2x
upsampling, skip concatenations, 1x1 linear output layer), restated with the
same parameter order so a parameter vector drives both.  Images are NHWC
(H, W, C).  ``bf16=True`` rounds where the device rounds (input, weights, every
stored activation and activation gradient) so the comparison isolates
accumulation order; ``bf16=False`` in float64 gives the exact network for
finite-difference checks of the backward pass.
"""
from __future__ import annotations

import numpy as np

BASE = 32
CPAD = 32
NAMES = ("e0a", "e0b", "e1a", "e1b", "e2a", "e2b", "ba", "bb", "d2a", "d2b", "d1a", "d1b", "d0a", "d0b")


def to_bf16(x):
    """Round float32 values to bfloat16 (nearest even), returned as float32."""
    x = np.ascontiguousarray(x, dtype=np.float32)
    u = x.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32)


def layer_shapes(cin=6, cout=3, base=BASE):
    """(name, cin, cout, level) of the convolutions in forward order."""
    C = [base, 2 * base, 4 * base, 8 * base]
    out = []
    for l in range(3):
        out.append((NAMES[2 * l], CPAD if l == 0 else C[l - 1], C[l], l))
        out.append((NAMES[2 * l + 1], C[l], C[l], l))
    out.append(("ba", C[2], C[3], 3))
    out.append(("bb", C[3], C[3], 3))
    for k, l in enumerate((2, 1, 0)):
        out.append((NAMES[8 + 2 * k], 3 * C[l], C[l], l))
        out.append((NAMES[9 + 2 * k], C[l], C[l], l))
    return out


def nparams(cin=6, cout=3, base=BASE):
    n = sum(co * 9 * ci + co for _, ci, co, _ in layer_shapes(cin, cout, base))
    return n + cout * base + cout


def unpack(vec, cin=6, cout=3, base=BASE):
    """Parameter vector -> dict name -> (W [cout, 3, 3, cin], b [cout]) plus 'head'."""
    P, off = {}, 0
    for name, ci, co, _ in layer_shapes(cin, cout, base):
        w = vec[off:off + co * 9 * ci].reshape(co, 3, 3, ci)
        off += co * 9 * ci
        b = vec[off:off + co]
        off += co
        P[name] = (w, b)
    wh = vec[off:off + cout * base].reshape(cout, base)
    off += cout * base
    P["head"] = (wh, vec[off:off + cout])
    return P


def init_params(seed=0, cin=6, cout=3, base=BASE):
    """He-normal weights (fan-in of the real input channels), zero biases, zero output layer."""
    rng = np.random.default_rng(seed)
    parts = []
    for name, ci, co, _ in layer_shapes(cin, cout, base):
        fan = 9 * (cin if name == "e0a" else ci)
        w = rng.normal(0.0, np.sqrt(2.0 / fan), size=(co, 3, 3, ci))
        if name == "e0a":
            w[..., cin:] = 0.0
        parts += [w.ravel(), np.zeros(co)]
    # zero output layer: the untrained network predicts no change
    parts += [np.zeros(cout * base), np.zeros(cout)]
    return np.concatenate(parts).astype(np.float32)


def _conv(x, w, b, dt):
    H, W, _ = x.shape
    xp = np.pad(x, ((1, 1), (1, 1), (0, 0)))
    out = np.zeros((H, W, w.shape[0]), dt)
    for dy in range(3):
        for dx in range(3):
            out += xp[dy:dy + H, dx:dx + W, :] @ w[:, dy, dx, :].T.astype(dt)
    if b is not None:
        out += b.astype(dt)
    return out


def _conv_dx(dy_, w, dt):
    H, W, _ = dy_.shape
    dxp = np.zeros((H + 2, W + 2, w.shape[3]), dt)
    for dy in range(3):
        for dx in range(3):
            dxp[dy:dy + H, dx:dx + W, :] += dy_ @ w[:, dy, dx, :].astype(dt)
    return dxp[1:-1, 1:-1]


def _conv_dw(dy_, x, dt):
    H, W, _ = dy_.shape
    xp = np.pad(x, ((1, 1), (1, 1), (0, 0)))
    dw = np.zeros((dy_.shape[2], 3, 3, x.shape[2]), dt)
    for dy in range(3):
        for dx in range(3):
            dw[:, dy, dx, :] = np.einsum("hwo,hwi->oi", dy_, xp[dy:dy + H, dx:dx + W, :])
    return dw, dy_.sum(axis=(0, 1))


def _pool(x):
    H, W, C = x.shape
    return x.reshape(H // 2, 2, W // 2, 2, C).mean(axis=(1, 3))


def _up(x):
    return x.repeat(2, axis=0).repeat(2, axis=1)


def forward(vec, x, cin=6, cout=3, base=BASE, bf16=True):
    """Returns (output [H, W, cout], cache for backward)."""
    dt = np.float32 if bf16 else np.float64
    rnd = to_bf16 if bf16 else (lambda a: a)
    P = unpack(np.asarray(vec, dt), cin, cout, base)
    W_ = {k: (rnd(w), b) for k, (w, b) in P.items() if k != "head"}
    H, Wd, _ = x.shape
    xin = np.zeros((H, Wd, CPAD), dt)
    xin[..., :cin] = x
    xin = rnd(xin)
    act = {"in": xin}

    def conv(name, inp):
        w, b = W_[name]
        y = rnd(np.maximum(_conv(inp, w, b, dt), 0))
        act[name] = y
        return y

    h = xin
    skips = []
    for l in range(3):
        h = conv(NAMES[2 * l], h)
        s = conv(NAMES[2 * l + 1], h)
        skips.append(s)
        h = rnd(_pool(s))
        act[f"pool{l}"] = h
    h = conv("ba", h)
    h = conv("bb", h)
    for k, l in enumerate((2, 1, 0)):
        cat = np.concatenate([skips[l], _up(h)], axis=2)
        act[f"cat{l}"] = cat
        h = conv(NAMES[8 + 2 * k], cat)
        h = conv(NAMES[9 + 2 * k], h)
    wh, bh = P["head"]
    out = h @ wh.T.astype(dt) + bh.astype(dt)
    return out, dict(act=act, W=W_, head=(wh, bh), dt=dt, rnd=rnd, cin=cin, cout=cout, base=base)


def backward(vec, cache, dout):
    """Gradient vector of sum(dout * output) (same order as the parameters)."""
    act, W_, dt, rnd = cache["act"], cache["W"], cache["dt"], cache["rnd"]
    wh, bh = cache["head"]
    grads = {}
    y = act["d0b"]
    dout = np.asarray(dout, dt)
    grads["head"] = (np.einsum("hwc,hwk->ck", dout, y), dout.sum(axis=(0, 1)))
    g = rnd((dout @ wh.astype(dt)) * (y > 0))

    def conv_b(name, inp, g_out, gate):
        w, _ = W_[name]
        grads[name] = _conv_dw(g_out, inp, dt)
        if gate is None:
            return None
        d = _conv_dx(g_out, w, dt)
        return d * (gate > 0) if gate is not False else d

    C = [cache["base"] * m for m in (1, 2, 4, 8)]
    dskip = {}
    for l in (0, 1, 2):
        nb, na = NAMES[13 - 2 * l], NAMES[12 - 2 * l]
        g_a = rnd(conv_b(nb, act[na], g, act[na]))
        gcat = rnd(conv_b(na, act[f"cat{l}"], g_a, act[f"cat{l}"]))
        dskip[l] = gcat[..., :C[l]]
        gu = gcat[..., C[l]:]
        H2, W2 = gu.shape[0] // 2, gu.shape[1] // 2
        g = rnd(gu.reshape(H2, 2, W2, 2, -1).sum(axis=(1, 3)))
    g_ba = rnd(conv_b("bb", act["ba"], g, act["ba"]))
    gp = rnd(conv_b("ba", act["pool2"], g_ba, False))
    for l in (2, 1, 0):
        skip = act[NAMES[2 * l + 1]]
        ds = rnd(dskip[l] + (_up(gp) * 0.25) * (skip > 0))
        g_e = rnd(conv_b(NAMES[2 * l + 1], act[NAMES[2 * l]], ds, act[NAMES[2 * l]]))
        inp = act["in"] if l == 0 else act[f"pool{l - 1}"]
        gp = conv_b(NAMES[2 * l], inp, g_e, None if l == 0 else False)
        if gp is not None:
            gp = rnd(gp)
    parts = []
    for name, _, _, _ in layer_shapes(cache["cin"], cache["cout"], cache["base"]):
        dw, db = grads[name]
        parts += [dw.ravel(), db.ravel()]
    parts += [grads["head"][0].ravel(), grads["head"][1].ravel()]
    return np.concatenate(parts)
