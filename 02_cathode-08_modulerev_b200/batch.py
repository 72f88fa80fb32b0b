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


def instance_specs(n=64, seed=3, sizes=SIZES):
    """The whole sweep as seeded specs, drawn in one order so that an instance does
    not depend on how the sweep is later split: index, grid size drawn from
    ``sizes`` (ni z cells, nj r cells), bias U(-10, 60) V, microwave power
    U(2, 16) W, and the seed of its discharge state."""
    rng = np.random.default_rng(seed)
    specs = []
    for k in range(n):
        nj, ni = sizes[int(rng.integers(len(sizes)))]
        V = float(rng.uniform(-10.0, 60.0))
        Pmw = float(rng.uniform(2.0, 16.0))
        specs.append(dict(index=k, ni=int(ni), nj=int(nj), V_bias=V, Pmw=Pmw, seed=int(rng.integers(1 << 30))))
    return specs


def partition(specs, world: int, steps=None):
    """Split the instances over ``world`` ranks, balanced by cells x steps: the
    largest cost first, each to the rank with the least cost so far (ties to the
    lower rank).  ``steps`` is one count for all or a list per instance.  Returns
    one sorted list of instance indices per rank; deterministic, so every rank
    computes the same split without communicating."""
    if world < 1:
        raise ValueError("world must be >= 1")
    n = len(specs)
    st = [steps] * n if steps is None or np.isscalar(steps) else list(steps)
    cost = [s["ni"] * s["nj"] * (1 if st[k] is None else st[k]) for k, s in enumerate(specs)]
    order = sorted(range(n), key=lambda k: (-cost[k], specs[k]["index"]))
    load = [0] * world
    out = [[] for _ in range(world)]
    for k in order:
        r = min(range(world), key=lambda q: (load[q], q))
        load[r] += cost[k]
        out[r].append(specs[k]["index"])
    return [sorted(x) for x in out]


def make_instances(pkg, specs, device=0, precision=1, microwave=False, ndiv_mw=100, reuse_tol=0.0):
    """Build the instances of ``specs`` on one GPU (grids, field store, parameters).
    microwave=True gives each instance the loop's microwave update every
    ``ndiv_mw`` steps (its own magnetised system, absorbed power rescaled to the
    instance's Pmw), so that the power axis of the sweep drives the heating.
    reuse_tol > 0 lets each instance's equations keep their multigrid hierarchies
    (Grid.set_reuse on its three grids)."""
    from .discharge import MicrowaveUpdate, rect_port
    from .solvers import Microwave3
    cases = []
    for sp in specs:
        c = learned.make_case(pkg, sp["ni"], sp["nj"], seed=sp["seed"], V_bias=sp["V_bias"], device=device)
        c.update(ni=sp["ni"], nj=sp["nj"], V_bias=sp["V_bias"], Pmw=sp["Pmw"], index=sp["index"])
        set_precision(c, precision)
        for k in ("g", "gx", "gr"):
            c[k].set_reuse(reuse_tol)
        if microwave:
            ni, nj = sp["ni"], sp["nj"]
            c["fs"].upload("epsr_mw", np.ones((ni + 2, nj + 2)))
            prm = dict(pkg.workloads.mw_er_rect(ni, nj, seed=2)["params"])
            c["m3"] = Microwave3(ni, nj, device=device)
            c["mwu"] = MicrowaveUpdate(c["fs"], c["m3"], prm, rect_port(prm, sp["Pmw"]), ndiv_mw=ndiv_mw)
        cases.append(c)
    return cases


def sweep_instances(pkg, n=64, seed=3, sizes=SIZES, device=0, precision=1, microwave=False):
    """Seeded instances of the sweep: grid size drawn from ``sizes``, bias
    U(-10, 60) V, microwave power U(2, 16) W (with microwave=True the instance's
    microwave update rescales its absorbed power to it), discharge state seeded
    per instance."""
    return make_instances(pkg, instance_specs(n, seed, sizes), device=device, precision=precision,
                          microwave=microwave)


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
        if c.get("mwu") is not None:
            items[k].mw = c["mwu"]._h
    wall = ctypes.c_double()
    rc = L.cth_batch_steps(items, n, steps, nthreads, ctypes.byref(wall))
    for k, (c, sp) in enumerate(zip(cases, keep)):
        fluid.step_params_back(sp, c["P"])
        c["anode"] = dict(I=items[k].I_Anode, Ii=items[k].Ii_Anode, Ie=items[k].Ie_Anode)
        if c.get("mwu") is not None:
            m = c.setdefault("mw_stats", dict(runs=0))
            m["runs"] += items[k].mw_runs
            if items[k].mw_runs:
                m.update(power_sum=items[k].mw_power_sum, J1r_exc=items[k].mw_J1r_exc)
    if rc < 0:
        raise capi.CathodeError(rc, capi.last_error())
    return wall.value, [items[k].rc for k in range(n)], [items[k].seconds for k in range(n)]


def summary(c) -> dict:
    """The I-V point of one instance after its steps: bias, power, anode currents."""
    a = c.get("anode", {})
    out = dict(index=int(c["index"]), ni=int(c["ni"]), nj=int(c["nj"]), V_bias=float(c["V_bias"]),
               Pmw=float(c["Pmw"]), itime=int(c["P"]["itime"]), I_Anode=float(a.get("I", 0.0)),
               Ii_Anode=float(a.get("Ii", 0.0)), Ie_Anode=float(a.get("Ie", 0.0)))
    if "mw_stats" in c:
        m = c["mw_stats"]
        out.update(mw_runs=int(m["runs"]), mw_power_before_rescale=float(m.get("power_sum", 0.0)))
    return out


def run_shard(specs, indices, runner):
    """Run this rank's share of the sweep: ``runner(selected_specs)`` returns one
    summary dict per spec (on a GPU: make_instances + batch_steps + summary)."""
    sel = [s for s in specs if s["index"] in set(indices)]
    return runner(sel)


def gather(local: list, world: int, group=None) -> list:
    """All instances' summaries on every rank, ordered by instance index: one
    all-gather of the per-rank lists (no collective while the instances run)."""
    if world == 1:
        allv = [local]
    else:
        import torch.distributed as dist
        allv = [None] * world
        dist.all_gather_object(allv, local, group=group)
    out = [x for part in allv for x in part]
    idx = [x["index"] for x in out]
    if len(set(idx)) != len(idx):
        raise RuntimeError("an instance was run on more than one rank")
    return sorted(out, key=lambda x: x["index"])


def gpu_runner(pkg, steps, device=0, nthreads=None, precision=1, microwave=False):
    """The runner of run_shard on one GPU: builds the specs' instances, advances
    them ``steps`` steps with cth_batch_steps and returns their summaries."""
    import os

    def run(sel):
        if not sel:
            return []
        cases = make_instances(pkg, sel, device=device, precision=precision, microwave=microwave)
        try:
            T = max(1, min(len(cases), nthreads or os.cpu_count() or 1))
            _, rc, _ = batch_steps(cases, steps=steps, nthreads=T)
            out = []
            for c, r in zip(cases, rc):
                d = summary(c)
                d["rc"] = int(r)
                out.append(d)
            return out
        finally:
            close(cases)
    return run


def sequential_steps(cases, steps: int):
    """The same steps one case after another on the caller's thread (host clock),
    with each case's microwave update where it has one."""
    import time
    import torch
    t0 = time.perf_counter()
    for c in cases:
        for _ in range(steps):
            r = c["fs"].fluid_step(c["gx"], c["gr"], c["P"])
            if r["solver_rc"] != 0:
                raise RuntimeError(f"solve did not converge: {r}")
            if c.get("mwu") is not None and c["mwu"].due(c["P"]["itime"]):
                c["mwu"].run(c["gx"], c["gr"])
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
        if c.get("mwu") is not None:
            c["mwu"].close()
            c["m3"].close()
        learned.close_case(c)
