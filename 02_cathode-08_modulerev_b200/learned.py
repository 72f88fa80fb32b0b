"""Learned warm start of the potential predictor-corrector.

No counterpart in the reference (its SMG solves always start from zero).  A
4-level U-Net of the device library (``cth_unet_*``: hand-written bf16
tensor-core convolutions, forward and backward, Adam) maps the state before the
potential sweep -- log10 n_e, log10 nu_m, |B| and the first corrections of
the two previous steps -- to the change of this step's first correction from the previous
one; the guess is the previous correction plus that change (an untrained,
zero-output network is the plain previous-step guess).  The multigrid then
starts from that guess and converges to the unchanged tolerance; a guess whose
relative residual exceeds ``guess_max_relres`` is dropped on the device and
the solve starts from zero (the plain method stays the fallback and the reference point).

This module drives the library: network handle, snapshot collection from plain
runs, training, and the warm-started time step.  Tensors are torch CUDA tensors
used as device memory; every arithmetic step of the network runs in the
library's kernels.
"""
from __future__ import annotations

import ctypes
import time

import numpy as np

from . import capi

CIN, COUT, BASE = 6, 3, 32
CHANNELS_IN = ("log10_ne", "log10_nu_m", "absB", "E_mw", "dphi_prev2", "dphi_prev")
CHANNELS_OUT = ("re_E_mw", "im_E_mw", "dphi")


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


def layer_shapes(base=BASE):
    """(name, cin, cout) of the 14 convolutions in the library's parameter order."""
    C = [base, 2 * base, 4 * base, 8 * base]
    names = ("e0a", "e0b", "e1a", "e1b", "e2a", "e2b", "ba", "bb", "d2a", "d2b", "d1a", "d1b", "d0a", "d0b")
    out = []
    for l in range(3):
        out += [(names[2 * l], 32 if l == 0 else C[l - 1], C[l]), (names[2 * l + 1], C[l], C[l])]
    out += [("ba", C[2], C[3]), ("bb", C[3], C[3])]
    for k, l in enumerate((2, 1, 0)):
        out += [(names[8 + 2 * k], 3 * C[l], C[l]), (names[9 + 2 * k], C[l], C[l])]
    return out


def init_params(seed=0, cin=CIN, cout=COUT, base=BASE):
    """He-normal convolution weights (fan-in of the real input channels), zero biases, zero output layer."""
    rng = np.random.default_rng(seed)
    parts = []
    for name, ci, co in layer_shapes(base):
        fan = 9 * (cin if name == "e0a" else ci)
        w = rng.normal(0.0, np.sqrt(2.0 / fan), size=(co, 3, 3, ci))
        if name == "e0a":
            w[..., cin:] = 0.0
        parts += [w.ravel(), np.zeros(co)]
    # zero output layer: the untrained network predicts no change
    parts += [np.zeros(cout * base), np.zeros(cout)]
    return np.concatenate(parts).astype(np.float32)


class UNet:
    """Handle of a device U-Net of H x W pixels (6 input, 3 output channels)."""

    def __init__(self, H: int, W: int, device: int = 0, seed: int = 0, params=None):
        self._L = capi.load()
        self.H, self.W, self.device = H, W, device
        self.handle = self._L.cth_unet_create(H, W, CIN, COUT, BASE, device)
        if not self.handle:
            raise RuntimeError(capi.last_error())
        self.n = int(self._L.cth_unet_nparams(self.handle))
        self.t = 0
        self.stats = np.array([0.0] * 6 + [1.0] * 6 + [0.0] * 3 + [1.0] * 3, np.float32)
        self.set_params(init_params(seed) if params is None else params)
        self.set_stats(self.stats)

    def close(self):
        if self.handle:
            self._L.cth_unet_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # parameters ----------------------------------------------------------
    def set_params(self, vec):
        v = np.ascontiguousarray(vec, dtype=np.float32)
        if v.size != self.n:
            raise ValueError(f"expected {self.n} parameters, got {v.size}")
        capi.check(self._L.cth_unet_set_params(self.handle, v.ctypes.data, self.n), allow_positive=False)
        self.t = 0

    def params(self) -> np.ndarray:
        v = np.empty(self.n, np.float32)
        capi.check(self._L.cth_unet_get_params(self.handle, v.ctypes.data, self.n), allow_positive=False)
        return v

    def grads(self) -> np.ndarray:
        v = np.empty(self.n, np.float32)
        capi.check(self._L.cth_unet_get_grads(self.handle, v.ctypes.data, self.n), allow_positive=False)
        return v

    def launch_count(self) -> int:
        """Kernels launched by forward passes and predictions since creation."""
        return int(self._L.cth_unet_launch_count(self.handle))

    def set_grid_limit(self, ctas: int):
        """At most ctas CTAs for the persistent tensor-core convolutions (0: all SMs)."""
        capi.check(self._L.cth_unet_set_grid_limit(self.handle, int(ctas)), allow_positive=False)

    def set_wait_test(self, stall: bool, polls: int = 1 << 20):
        """Test of the tensor-core kernel's bounded waits: with stall the kernel
        issues no loads, every wait runs out and check() reports it."""
        capi.check(self._L.cth_unet_set_wait_test(self.handle, int(stall), int(polls)), allow_positive=False)

    def set_smoothing(self, passes: int):
        """5-point smoothing passes applied to the predicted change before it
        becomes the potential solve's guess (default 0)."""
        capi.check(self._L.cth_unet_set_smoothing(self.handle, int(passes)), allow_positive=False)

    def set_tensor_cores(self, tcgen05: bool):
        """Convolutions on tcgen05 (default) or on the warp-level mma.sync kernel."""
        capi.check(self._L.cth_unet_set_tensor_cores(self.handle, int(tcgen05)), allow_positive=False)

    def check(self):
        """Synchronise and raise if a tensor-core convolution's wait gave up."""
        capi.check(self._L.cth_unet_check(self.handle), allow_positive=False)

    def set_stats(self, stats):
        self.stats = np.ascontiguousarray(stats, dtype=np.float32).copy()
        capi.check(self._L.cth_unet_set_stats(self.handle, self.stats.ctypes.data), allow_positive=False)

    def set_loss_weights(self, w):
        a = np.ascontiguousarray(w, dtype=np.float32)
        capi.check(self._L.cth_unet_set_loss_weights(self.handle, a.ctypes.data), allow_positive=False)

    def save(self, path):
        np.savez(path, params=self.params(), stats=self.stats, H=self.H, W=self.W)

    @classmethod
    def load(cls, path, device=0):
        z = np.load(path)
        net = cls(int(z["H"]), int(z["W"]), device=device, params=z["params"])
        net.set_stats(z["stats"])
        return net

    # passes ----------------------------------------------------------------
    def _stream(self, stream):
        import torch
        return (stream if stream is not None else torch.cuda.current_stream(self.device)).cuda_stream

    def forward(self, x, stream=None):
        """x: (H, W, 6) float32 CUDA tensor -> (H, W, 3) float32."""
        import torch
        out = torch.empty((self.H, self.W, COUT), dtype=torch.float32, device=x.device)
        capi.check(self._L.cth_unet_forward(self.handle, _ptr(x.contiguous()), _ptr(out), self._stream(stream)),
                   allow_positive=False)
        return out

    def backward(self, dout, stream=None):
        """Parameter gradients of sum(dout * forward(x)) after forward(x)."""
        capi.check(self._L.cth_unet_backward(self.handle, _ptr(dout.contiguous()), self._stream(stream)),
                   allow_positive=False)

    def train_step(self, x, target, mask, msum: float, lr: float, stream=None) -> float:
        self.t += 1
        loss = ctypes.c_double()
        capi.check(self._L.cth_unet_train_step(self.handle, _ptr(x), _ptr(target), _ptr(mask), float(msum),
                                               float(lr), self.t, self._stream(stream), ctypes.byref(loss)),
                   allow_positive=False)
        return loss.value

    def features(self, fields, stream=None):
        import torch
        out = torch.empty((self.H, self.W, CIN), dtype=torch.float32, device=f"cuda:{self.device}")
        capi.check(self._L.cth_unet_features(self.handle, fields._h, _ptr(out), self._stream(stream)),
                   allow_positive=False)
        return out

    def predict_dphi(self, fields, stream=None):
        capi.check(self._L.cth_unet_predict_dphi(self.handle, fields._h, self._stream(stream)),
                   allow_positive=False)


# ---------------------------------------------------------------------------
# snapshots, training, evaluation
# ---------------------------------------------------------------------------
def make_case(pkg, ni, nj, seed, V_bias, device=0, Lz=10e-3, Lr=5e-3):
    """A seeded discharge on the r-z rectangle: grids, field store, parameters."""
    geo = pkg.fluid.rectangle_geometry(ni, nj, width_neutIn=2.03e-3)
    ds = pkg.workloads.discharge_state(ni, nj, Lz=Lz, Lr=Lr, seed=seed)
    cfg = pkg.workloads.discharge_params(geo, ds["dr"], Lr)
    g = pkg.Grid(ni, nj, geo["ib"], geo["jb"], device=device)
    gx = pkg.Grid(ni, nj, geo["fxi"], geo["fxj"], device=device)
    gr = pkg.Grid(ni, nj, geo["fri"], geo["frj"], device=device)
    fs = pkg.Fields(g)
    fs.set_flags(geo["flags"])
    fs.set_ghost_rules(geo["ghosts"])
    fs.set_energy_keep_walls(geo.get("energy_keep_walls", []))
    fs.set_ion_geometry(geo)
    for k, v in cfg["tables"].items():
        fs.set_table(k, v)
    for k, v in cfg["see"].items():
        fs.set_table(k, v)
    for k, v in ds["fields"].items():
        fs.upload(k, v)
    fs.upload("rhoe_old", ds["fields"]["rhoe"])
    P = cfg["params"]
    P["phi"]["V_bias"] = float(V_bias)
    fs.update_transport_coef(P["transport"])
    return dict(g=g, gx=gx, gr=gr, fs=fs, P=P, geo=geo)


def close_case(c):
    c["fs"].close()
    for k in ("g", "gx", "gr"):
        c[k].close()


def collect_snapshots(pkg, net, ni, nj, nsteps, seeds, bias_range=(-10.0, 60.0), precision=1, skip=2,
                      device=0):
    """Plain runs (previous-step warm start, same stopping rule as from zero) of
    nsteps steps per seed; snapshot k pairs the
    state before step k (features, previous correction) with the change of
    step k's first potential correction from the previous one.  Returns (X [n, H, W, 6], Y [n, H, W, 3], mask [H, W])
    as un-normalised CUDA tensors (net's stats must be the identity)."""
    import torch
    Xs, Ys = [], []
    rng = np.random.default_rng(12345)
    for sd in seeds:
        c = make_case(pkg, ni, nj, sd, rng.uniform(*bias_range), device=device)
        fs, P = c["fs"], c["P"]
        for blk in ("ion", "rhoe", "eps", "neutral"):
            P[blk]["precision"] = precision
        P["phi"].update(precision=precision, warm_start=2, guess_max_relres=1.0)
        for k in range(nsteps):
            x = net.features(fs)
            r = fs.fluid_step(c["gx"], c["gr"], P)
            if r["solver_rc"] != 0:
                raise RuntimeError(f"solve did not converge while collecting snapshots: {r}")
            if k >= skip:
                # target: the change of the first correction from the previous step's
                y = torch.zeros((net.H, net.W, COUT), dtype=torch.float32, device=x.device)
                d = fs.plane("dphi_prev")[1:nj + 1, 1:ni + 1]
                y[:nj, :ni, 2] = d.to(torch.float32) - x[:nj, :ni, 5]
                Xs.append(x)
                Ys.append(y)
        close_case(c)
    mask = torch.zeros((net.H, net.W), dtype=torch.float32, device=Xs[0].device)
    mask[:nj, :ni] = 1.0
    return torch.stack(Xs), torch.stack(Ys), mask


def fit_stats(X, Y, mask):
    """Per-channel mean / std over the grid pixels (channels without spread: 0 / 1)."""
    import torch
    m = mask.bool()
    xin = X[:, m]                   # [n, npix, 6]
    yout = Y[:, m]

    def ms(a):
        mu = a.double().mean(dim=(0, 1))
        sd = a.double().std(dim=(0, 1))
        sd = torch.where(sd > 1e-30, sd, torch.ones_like(sd))
        return mu.cpu().numpy(), sd.cpu().numpy()
    im, isd = ms(xin)
    om, osd = ms(yout)
    im[3], isd[3] = 0.0, 1.0
    for k in (0, 1):
        om[k], osd[k] = 0.0, 1.0
    return np.concatenate([im, isd, om, osd]).astype(np.float32)


def normalise(X, Y, stats):
    import torch
    st = torch.as_tensor(stats, device=X.device)
    Xn = (X - st[0:6]) / st[6:12]
    Yn = (Y - st[12:15]) / st[15:18]
    return Xn.contiguous(), Yn.contiguous()


def train(net, Xn, Yn, mask, epochs=4, lr=1e-3, seed=0, log=None):
    """Adam on the masked MSE of the correction channel, one snapshot per step."""
    net.set_loss_weights([0.0, 0.0, 1.0])
    msum = float(mask.sum().item())
    rng = np.random.default_rng(seed)
    losses = []
    for ep in range(epochs):
        order = rng.permutation(Xn.shape[0])
        tot = 0.0
        for q in order:
            tot += net.train_step(Xn[q], Yn[q], mask, msum, lr)
        losses.append(tot / len(order))
        if log:
            log(f"epoch {ep}: mean loss {losses[-1]:.4e}")
    return losses


def heldout_error(net, Xn, Yn, mask):
    """Relative L2 error of the predicted change of the correction on held-out snapshots."""
    errs = []
    m = mask.bool()
    for q in range(Xn.shape[0]):
        o = net.forward(Xn[q])
        st = net.stats
        pred = o[..., 2][m] * float(st[17]) + float(st[14])
        ref = Yn[q][..., 2][m] * float(st[17]) + float(st[14])
        errs.append(float((pred - ref).norm() / ref.norm().clamp_min(1e-300)))
    return errs


def run_steps(pkg, c, nsteps, warm_start, net=None, precision=1):
    """nsteps fluid steps of a case with the given warm start; per-step record of
    the first potential solve and the step's device time."""
    import torch
    fs, P = c["fs"], c["P"]
    for blk in ("ion", "rhoe", "eps", "neutral"):
        P[blk]["precision"] = precision
    P["phi"].update(precision=precision, warm_start=warm_start, guess_max_relres=1.0)
    P["net"] = net if warm_start in (1, 3) else None
    rec = []
    s = torch.cuda.current_stream()
    for _ in range(nsteps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(s)
        r = fs.fluid_step(c["gx"], c["gr"], P, stream=s)
        e1.record(s)
        e1.synchronize()
        if r["solver_rc"] != 0:
            raise RuntimeError(f"solve did not converge: {r}")
        f = r["phi_first"]
        rec.append(dict(cycles=f["iterations"], guess=f["guess"], guess_residual=f["guess_residual"],
                        residual=f["residual"], ms=e0.elapsed_time(e1), phi_iterations=r["iterations"]["phi"],
                        net_ran=r["net_ran"]))
    P["net"] = None
    return rec


def now():
    return time.perf_counter()
