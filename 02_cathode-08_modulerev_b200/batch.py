"""Batched discharges on one GPU: the bias-voltage / microwave-power sweeps for
I-V curves (no counterpart in the reference, which runs one discharge per
process).  ``cth_batch_steps`` advances many independent instances -- each a
complete time loop with its own grids, field store and stream -- from host
worker threads; ``autotune`` picks the smoother sweeps per level and the fused
coarse tail for each grid size by timing a few steps (every choice meets the
same stopping rule, so only the speed changes)."""
from __future__ import annotations

import ctypes
import itertools

import numpy as np

from . import capi, fluid, learned

SIZES = ((64, 128), (128, 256), (192, 384), (256, 512))   # (r cells, z cells)


def sweep_instances(pkg, n=64, seed=3, sizes=SIZES, device=0, precision=1):
    """Seeded instances of the sweep: grid size drawn from ``sizes``, bias
    U(-10, 60) V, microwave power U(2, 16) W (recorded; the fluid step reads the
    absorbed power as a field), discharge state seeded per instance."""
    rng = np.random.default_rng(seed)
    cases = []
    for k in range(n):
        nj, ni = sizes[int(rng.integers(len(sizes)))]
        V = float(rng.uniform(-10.0, 60.0))
        Pmw = float(rng.uniform(2.0, 16.0))
        c = learned.make_case(pkg, ni, nj, seed=int(rng.integers(1 << 30)), V_bias=V, device=device)
        c.update(ni=ni, nj=nj, V_bias=V, Pmw=Pmw)
        set_precision(c, precision)
        cases.append(c)
    return cases


def set_precision(c, precision):
    P = c["P"]
    for blk in ("ion", "rhoe", "eps", "neutral"):
        P[blk]["precision"] = precision
    P["phi"]["precision"] = precision


def set_cycle(c, nu_pre, nu_post, tail):
    for k in ("g", "gx", "gr"):
        c[k].set_cycle(nu_pre, nu_post)
        c[k].set_tail(tail)


def batch_steps(cases, steps: int, nthreads: int):
    """Advance every case by ``steps`` steps concurrently; returns (wall seconds,
    per-case status, per-case seconds)."""
    L = capi.load()
    n = len(cases)
    items = (capi.BatchItem * n)()
    keep = []
    for k, c in enumerate(cases):
        sp = fluid.step_params(c["P"])
        keep.append(sp)
        items[k].fs = c["fs"]._h
        items[k].gx = c["gx"]._h
        items[k].gr = c["gr"]._h
        items[k].params = ctypes.pointer(sp)
    wall = ctypes.c_double()
    rc = L.cth_batch_steps(items, n, steps, nthreads, ctypes.byref(wall))
    for c, sp in zip(cases, keep):
        fluid.step_params_back(sp, c["P"])
    if rc < 0:
        raise capi.CathodeError(rc, capi.last_error())
    return wall.value, [items[k].rc for k in range(n)], [items[k].seconds for k in range(n)]


def sequential_steps(cases, steps: int):
    """The same steps one case after another on the caller's thread (host clock)."""
    import time
    import torch
    t0 = time.perf_counter()
    for c in cases:
        for _ in range(steps):
            r = c["fs"].fluid_step(c["gx"], c["gr"], c["P"])
            if r["solver_rc"] != 0:
                raise RuntimeError(f"solve did not converge: {r}")
    torch.cuda.synchronize()
    return time.perf_counter() - t0


def autotune(cases, candidates=None, steps=3):
    """Per grid size: time ``steps`` steps of one instance for each (nu_pre,
    nu_post, tail) candidate (CUDA events) and apply the fastest to every
    instance of that size.  Returns {size: (choice, ms per step)}."""
    import torch
    if candidates is None:
        candidates = list(itertools.product((1, 2), (1, 2), (True, False)))
    by_size = {}
    for c in cases:
        by_size.setdefault((c["nj"], c["ni"]), []).append(c)
    out = {}
    for size, group in by_size.items():
        c = group[0]
        best = None
        for cand in candidates:
            set_cycle(c, *cand)
            c["fs"].fluid_step(c["gx"], c["gr"], c["P"])   # graphs for this cycle shape
            s = torch.cuda.current_stream()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(s)
            for _ in range(steps):
                c["fs"].fluid_step(c["gx"], c["gr"], c["P"], stream=s)
            e1.record(s)
            e1.synchronize()
            ms = e0.elapsed_time(e1) / steps
            if best is None or ms < best[1]:
                best = (cand, ms)
        for g in group:
            set_cycle(g, *best[0])
        out[f"{size[0]}x{size[1]}"] = dict(nu_pre=best[0][0], nu_post=best[0][1], tail=best[0][2],
                                            ms_per_step=best[1], instances=len(group))
    return out


def close(cases):
    for c in cases:
        learned.close_case(c)
