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
MW_CIN, MW_COUT = 9, 6     # the microwave network: log n_e, log nu_m1, |B|, previous E; change of E
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
    """Handle of a device U-Net of H x W pixels (cin input, cout output channels:
    6 / 3 for the potential correction, 9 / 6 for the microwave fields)."""

    def __init__(self, H: int, W: int, device: int = 0, seed: int = 0, params=None, cin: int = CIN,
                 cout: int = COUT):
        self._L = capi.load()
        self.H, self.W, self.device, self.cin, self.cout = H, W, device, cin, cout
        self.handle = self._L.cth_unet_create(H, W, cin, cout, BASE, device)
        if not self.handle:
            raise RuntimeError(capi.last_error())
        self.n = int(self._L.cth_unet_nparams(self.handle))
        self.t = 0
        self.stats = np.array([0.0] * cin + [1.0] * cin + [0.0] * cout + [1.0] * cout, np.float32)
        self.set_params(init_params(seed, cin, cout) if params is None else params)
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
        np.savez(path, params=self.params(), stats=self.stats, H=self.H, W=self.W, cin=self.cin, cout=self.cout)

    @classmethod
    def load(cls, path, device=0):
        z = np.load(path)
        cin = int(z["cin"]) if "cin" in z else CIN
        cout = int(z["cout"]) if "cout" in z else COUT
        net = cls(int(z["H"]), int(z["W"]), device=device, params=z["params"], cin=cin, cout=cout)
        net.set_stats(z["stats"])
        return net

    # passes ----------------------------------------------------------------
    def _stream(self, stream):
        import torch
        return (stream if stream is not None else torch.cuda.current_stream(self.device)).cuda_stream

    def forward(self, x, stream=None):
        """x: (H, W, cin) float32 CUDA tensor -> (H, W, cout) float32."""
        import torch
        out = torch.empty((self.H, self.W, self.cout), dtype=torch.float32, device=x.device)
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

    def mw_features(self, fields, E3, escale=1.0, stream=None):
        """Input of the microwave network (H, W, 9) from the store and the previous
        fields E3 ((3, nj+2, ld) complex128, the store's layout) times escale
        (1 / the excitation they were solved with)."""
        import torch
        out = torch.empty((self.H, self.W, MW_CIN), dtype=torch.float32, device=f"cuda:{self.device}")
        capi.check(self._L.cth_unet_mw_features(self.handle, fields._h, _ptr(E3), float(escale), _ptr(out),
                                                self._stream(stream)), allow_positive=False)
        return out

    def mw_guess(self, fields, Eprev, jprev=1.0, jnow=1.0, stream=None):
        """(jnow / jprev) Eprev + jnow x the predicted change per unit excitation,
        same layout (jprev: the excitation Eprev was solved with; jnow: the next)."""
        import torch
        out = torch.empty_like(Eprev)
        capi.check(self._L.cth_unet_mw_guess(self.handle, fields._h, _ptr(Eprev), float(jprev), float(jnow),
                                             _ptr(out), self._stream(stream)), allow_positive=False)
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


# ---------------------------------------------------------------------------
# the microwave warm start: a second network (9 input, 6 output channels) maps
# log n_e, log nu_m1, |B| and the previous microwave fields to their change;
# the solve starts from previous + change when the device-side residual test
# takes it (cth_mw_update_set_net), so the network never changes the answer
# ---------------------------------------------------------------------------
def mw_target(E_new, j_new, E_prev, j_prev, ni, nj, H, W):
    """(H, W, 6) float32: real and imaginary parts of the change of Ex, Er, Ephi
    per unit excitation (E_new / j_new - E_prev / j_prev) at grid cell (i, j) ->
    pixel (j-1, i-1) (E planes: (3, nj+2, ld) complex128)."""
    import torch
    d = (E_new / j_new - E_prev / j_prev)[:, 1:nj + 1, 1:ni + 1]
    y = torch.zeros((H, W, MW_COUT), dtype=torch.float32, device=E_new.device)
    for c in range(3):
        y[:nj, :ni, 2 * c] = d[c].real.to(torch.float32)
        y[:nj, :ni, 2 * c + 1] = d[c].imag.to(torch.float32)
    return y


def collect_mw_snapshots(pkg, net, ni, nj, runs, nsteps, ndiv_mw, seed=2024, device=0, precision=1):
    """Plain discharges (``runs`` of them: state seed, bias U(-10, 60) V and
    microwave power U(2, 16) W drawn from ``seed``) with the microwave update
    every ``ndiv_mw`` steps for ``nsteps`` steps; one snapshot per update after
    the first pairs the network's input before the solve (the state and the
    previous fields) with the change of the fields.  Returns (X [n, H, W, 9],
    Y [n, H, W, 6], mask [H, W]) un-normalised (the net's stats must be the
    identity)."""
    import torch
    rng = np.random.default_rng(seed)
    Xs, Ys = [], []
    for _ in range(runs):
        d = pkg.discharge.RectangleDischarge(pkg, ni, nj, seed=int(rng.integers(1 << 30)), device=device,
                                             precision=precision, ndiv_mw=ndiv_mw,
                                             Pmw=float(rng.uniform(2.0, 16.0)), V_bias=float(rng.uniform(-10.0, 60.0)))
        try:
            updates, j_prev = 0, None
            for _ in range(nsteps):
                r = d.fs.fluid_step(d.gx, d.gr, d.P)
                if r["solver_rc"] != 0:
                    break
                if d.mw.due(d.P["itime"]):
                    E_prev = d.e3.clone()
                    j_now = d.J1r_exc
                    x = net.mw_features(d.fs, E_prev, escale=1.0 / j_prev) if updates > 0 else None
                    out = d.microwave()
                    if out["rc"] != 0:
                        break
                    if updates > 0:
                        Xs.append(x)
                        Ys.append(mw_target(d.e3, j_now, E_prev, j_prev, ni, nj, net.H, net.W))
                    updates += 1
                    j_prev = j_now
        finally:
            d.close()
    mask = torch.zeros((net.H, net.W), dtype=torch.float32, device=Xs[0].device)
    mask[:nj, :ni] = 1.0
    return torch.stack(Xs), torch.stack(Ys), mask


def mw_fit_stats(X, Y, mask):
    """Per-channel mean and standard deviation over the masked pixels (inputs
    and outputs), in the library's layout (2 cin + 2 cout values)."""
    import torch
    m = mask.bool()

    def ms(a):
        v = a[:, m, :].reshape(-1, a.shape[-1]).to(torch.float64)
        mu = v.mean(0)
        sd = v.std(0)
        sd = torch.where(sd > 1e-30, sd, torch.ones_like(sd))
        return mu.cpu().numpy(), sd.cpu().numpy()
    im, isd = ms(X)
    om, osd = ms(Y)
    return np.concatenate([im, isd, om, osd]).astype(np.float32)


def mw_normalise(X, Y, stats):
    import torch
    st = torch.as_tensor(stats, device=X.device)
    ci, co = MW_CIN, MW_COUT
    Xn = (X - st[0:ci]) / st[ci:2 * ci]
    Yn = (Y - st[2 * ci:2 * ci + co]) / st[2 * ci + co:2 * ci + 2 * co]
    return Xn.contiguous(), Yn.contiguous()


def mw_train(net, Xn, Yn, mask, epochs=8, lr=5e-4, seed=0, log=None):
    """Adam on the masked MSE of all six output channels, one snapshot per step."""
    net.set_loss_weights([1.0] * MW_COUT)
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


def mw_evaluate(pkg, net, ni, nj, runs, nsteps, ndiv_mw, tol=1e-8, seed=7, device=0, precision=1):
    """Held-out discharges: at every microwave update after the first, the same
    assembled system solved to ``tol`` from zero (the state advances with this
    solution), from the previous fields and from the network's guess.  Returns
    per-start iteration counts and solve times, the network's inference time and
    how often the device-side test rejected its guess (fallback to zero)."""
    import torch
    rng = np.random.default_rng(seed)
    rec = dict(zero=[], previous=[], network=[], zero_ms=[], previous_ms=[], network_ms=[], inference_ms=[],
               network_guess_residual=[], previous_guess_residual=[], network_rejected=0, previous_rejected=0,
               updates=0)
    s = torch.cuda.current_stream()

    def timed(fn):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(s)
        out = fn()
        e1.record(s)
        e1.synchronize()
        return out, e0.elapsed_time(e1)

    for _ in range(runs):
        d = pkg.discharge.RectangleDischarge(pkg, ni, nj, seed=int(rng.integers(1 << 30)), device=device,
                                             precision=precision, ndiv_mw=ndiv_mw, mw_tol=tol,
                                             Pmw=float(rng.uniform(2.0, 16.0)), V_bias=float(rng.uniform(-10.0, 60.0)))
        try:
            j_prev = None
            for _ in range(nsteps):
                r = d.fs.fluid_step(d.gx, d.gr, d.P)
                if r["solver_rc"] != 0:
                    break
                if not d.mw.due(d.P["itime"]):
                    continue
                E_prev = d.e3.clone()
                j_now = d.J1r_exc
                if j_prev is None:                 # the first update: nothing to start from
                    out = d.microwave(stream=s)
                    if out["rc"] != 0:
                        break
                    j_prev = j_now
                    continue
                guess, t_inf = timed(lambda: net.mw_guess(d.fs, E_prev, j_prev, j_now, stream=s))
                prev = E_prev * (j_now / j_prev)   # the previous fields at the new excitation
                out = d.microwave(stream=s)        # assembles, solves from zero, advances the discharge
                if out["rc"] != 0:
                    break
                j_prev = j_now
                scratch = d.m3.planes(3)
                (_, sz), t0 = timed(lambda: d.m3.solve_dev(maxITR=400, error_cnv=tol, out=scratch, stream=s))
                (_, sp), t1 = timed(lambda: d.m3.solve_dev(maxITR=400, error_cnv=tol, out=scratch, x0=prev,
                                                           stream=s))
                (_, sn), t2 = timed(lambda: d.m3.solve_dev(maxITR=400, error_cnv=tol, out=scratch, x0=guess,
                                                           stream=s))
                rec["zero"].append(sz.iterations)
                rec["previous"].append(sp.iterations)
                rec["network"].append(sn.iterations)
                rec["zero_ms"].append(t0)
                rec["previous_ms"].append(t1)
                rec["network_ms"].append(t2)
                rec["inference_ms"].append(t_inf)
                rec["previous_guess_residual"].append(sp.guess_residual)
                rec["network_guess_residual"].append(sn.guess_residual)
                rec["network_rejected"] += int(sn.guess == -1)
                rec["previous_rejected"] += int(sp.guess == -1)
                rec["updates"] += 1
        finally:
            d.close()
    return rec
