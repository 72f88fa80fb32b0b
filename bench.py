#!/usr/bin/env python
"""Throughput of the implicit solve path on one B200 (or N replicas).

Workload: the two isolated 512 (r) x 1024 (z) systems of the cathode code.
  (a) potential: the reference's Poisson stencil with a 1:3.8 dielectric slab,
      Dirichlet electrodes at z = 0 / z = L, axis at r = 0, seeded space charge;
  (b) microwave Er: the reference's Er equation with B = 0 (cold-plasma
      conductivity from seeded n_e, nu), port excitation, open and Gauss
      boundaries; assembled on the device.
Both are solved from a zero guess to ||b-Ax||_2/||b||_2 < 1e-10.  One step =
solve (a) + assemble and solve (b).

Reported line (rank 0):
  value        steps/s with (a) on the mixed-precision path (FP32 multigrid
               + FP64 defect correction) and (b) in complex FP64 (BiCGStab +
               complex multigrid), inputs resident in HBM, L2 flushed
               (256 MiB memset) before every step, CUDA events on the stream
  fp64         the same with (a) on the plain FP64 multigrid
  e2e          steps/s through the public API with pinned host inputs: (a)
               via the host C ABI (cth_smg_solve: H2D of six arrays, D2H of
               the solution), (b) H2D of n_e, nu, epsr, device assembly and
               solve, D2H of the complex Er plane
  roofline     finest-level z-line relaxation kernel: algorithmic bytes /
               CUDA-event time vs the measured HBM copy bandwidth
  cpu_baseline the CPU restatement (oracle, OpenMP) on a bounded sample

--impl reference times the CPU restatement of the reference path (the
reference itself needs HYPRE/MPI/Eigen/yaml-cpp, which are not installed)
on the same workload and prints the same metric: (a) by the CPU
semicoarsening multigrid (OpenMP), (b) by a sparse direct LU (SuperLU, the
family of the reference's Eigen SparseLU) after the same assembly.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "steps/s at 512x1024 r-z: learned+mixed vs plain FP64 GPU at 1e-8 residual"
UNIT = "steps/s"
NI, NJ = 1024, 512
TOL = 1e-10
MAXIT = 30


def workload_config(extra=None):
    c = {
        "workload": "isolated 512 (r) x 1024 (z) systems: (a) potential (slab epsr 3.8, electrodes 0/20 V, axis) "
                    "+ (b) microwave Er (B=0 cold plasma, n_e 1e15-1e18, nu 1e8-1e10, port/open/Gauss); "
                    "one step = solve (a) + assemble and solve (b), each to 1e-10 relative residual",
        "ni_z": NI, "nj_r": NJ, "tol": TOL, "maxit": MAXIT,
        "l2": "256 MiB memset between timed steps (working set < L2)",
        "method": "(a) semicoarsening MG (z-line zebra smoother, Galerkin), FP32 cycles + FP64 defect "
                  "correction; (b) complex FP64 BiCGStab preconditioned by one complex semicoarsening V-cycle",
    }
    if extra:
        c.update(extra)
    return c


def env_rank():
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


# --------------------------------------------------------------------------
# clocks sampled during the timed region
# --------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.dev = device_index
        self.proc = None
        self.path = os.path.join("/tmp", f"cathode_clocks_{os.getpid()}.csv")

    def start(self):
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.dev}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "20"],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.close()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            p = [x.strip() for x in line.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                smax.append(float(p[2]))
            except ValueError:
                continue
            for n, v in zip(names, p[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "samples": len(sm), "reasons": sorted(reasons)}


def measured_peaks():
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        return None


def ncu_traffic():
    """DRAM bytes per launch of the finest-level relaxation from the committed ncu summary."""
    try:
        d = json.load(open(os.path.join(ROOT, "profiles", "traffic.json")))
        return d.get("relax0_dram_bytes_per_launch")
    except Exception:
        return None


# --------------------------------------------------------------------------
# CPU legs (oracle = test infrastructure, timed as the CPU baseline only)
# --------------------------------------------------------------------------
def cpu_step(sa, wb):
    """One step on the CPU restatement: (a) multigrid, (b) assembly + sparse LU."""
    import oracle
    from oracle import microwave as mw
    _, rc, it, rel = oracle.smg_solve(sa, MAXIT, TOL)
    p = mw.er_rect_params(NI, NJ)
    sysb = mw.er_rect_system(wb["ne"], wb["nu"], wb["epsr"], p)
    mw.solve_c5_direct(sysb)
    return rel


def cpu_sample(sa, wb, budget_s=25.0, max_steps=20):
    import oracle
    oracle.build()
    n = 0
    t0 = time.perf_counter()
    while True:
        cpu_step(sa, wb)
        n += 1
        el = time.perf_counter() - t0
        if el > budget_s or n >= max_steps:
            break
    return n / el, n, el


def run_reference(args, rank, world):
    if rank != 0:
        return 0
    import __graft_entry__
    pkg = __graft_entry__.load_package()
    import oracle
    oracle.build()
    sa = pkg.workloads.poisson_slab(NI, NJ, seed=1)
    wb = pkg.workloads.mw_er_rect(NI, NJ, seed=2)
    threads = os.cpu_count()
    # bounded sample: each CPU step takes ~10-20 s; keep the whole run to a few minutes
    t0 = time.perf_counter()
    cpu_step(sa, wb)
    t_first = time.perf_counter() - t0
    steps = max(1, min(args.steps, int(150.0 / max(t_first, 1e-3))))
    times = []
    for _ in range(steps):
        t0 = time.perf_counter()
        cpu_step(sa, wb)
        times.append(time.perf_counter() - t0)
    tot = sum(times)
    v = steps / tot
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
        "steps": steps, "warmup": 1, "ms_per_step": 1e3 * tot / steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded)", "config": workload_config({"parallelism": "host threads"}),
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": f"{steps} full steps after 1 warm-up (requested {args.steps}/{args.warmup}; "
                                   f"capped to ~150 s): (a) CPU restatement of solver_SMG (semicoarsening MG, "
                                   f"OpenMP over {threads} threads), (b) assembly + SuperLU direct solve "
                                   f"(single thread), as the reference's SparseLU; the reference's own build "
                                   f"needs HYPRE/MPI/Eigen/yaml-cpp, not installable here"},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# --------------------------------------------------------------------------
def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="cathode", choices=["cathode", "reference"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    args = ap.parse_args()
    rank, world, local = env_rank()
    if args.impl == "reference":
        return run_reference(args, rank, world)

    import numpy as np
    import torch
    import torch.distributed as dist
    import __graft_entry__
    pkg = __graft_entry__.load_package()
    capi = pkg.capi

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=dev)

    # independent instance per rank (replicas: the path has no exchange step)
    sa = pkg.workloads.poisson_slab(NI, NJ, seed=1 + rank)
    wb = pkg.workloads.mw_er_rect(NI, NJ, seed=2 + rank)
    g = pkg.Grid(NI, NJ, sa["i_bl"], sa["j_bl"], device=local)
    gb = pkg.Grid(NI, NJ, wb["i_bl"], wb["j_bl"], device=local)
    planes = [g.to_device(sa[k]) for k in ("aP", "aE", "aW", "aN", "aS", "b")]
    fields = [gb.to_device(wb[k]) for k in ("ne", "nu", "epsr")]
    x = g.device_plane(1)[0]
    eb = torch.zeros((NJ + 2, gb.ld), dtype=torch.complex128, device=dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream(dev)

    def solve_a(prec):
        return g.smg_solve_dev(*planes, x, maxITR=MAXIT, error_cnv=TOL, precision=prec, stream=stream)

    def solve_b():
        pb = gb.mw_er_assemble_dev(*fields, wb["params"], stream=stream)
        return gb.c5_solve_dev(*pb, eb, maxITR=200, error_cnv=TOL, stream=stream), pb

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize(dev)

    def timed(prec, steps, profile=False):
        if profile:
            g.profile(True)
        ms = ms_a = 0.0
        its = []
        l0 = g.launch_count() + gb.launch_count()
        for _ in range(steps):
            flush.zero_()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e2 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            st = solve_a(prec)
            e1.record(stream)
            stb, _ = solve_b()
            e2.record(stream)
            e2.synchronize()
            ms += e0.elapsed_time(e2)
            ms_a += e0.elapsed_time(e1)
            its.append((st.iterations, stb.iterations))
            if not (st.converged and stb.converged):
                raise RuntimeError(f"solve did not converge: {st.as_dict()} {stb.as_dict()}")
        launches = g.launch_count() + gb.launch_count() - l0
        prof = None
        if profile:
            prof = {c: g.profile_read(c) for c in (capi.CTH_PROF_RELAX0, capi.CTH_PROF_UPDATE,
                                                   capi.CTH_PROF_RESTRICT0, capi.CTH_PROF_SETUP)}
            g.profile(False)
        t = torch.tensor([ms, ms_a], dtype=torch.float64, device=dev)
        if world > 1:
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t[0].item()), float(t[1].item()), its, launches, prof

    # warm-up (both precisions)
    for _ in range(max(args.warmup, 3)):
        solve_a(capi.CTH_PREC_MIXED)
        solve_a(capi.CTH_PREC_FP64)
        solve_b()
    barrier()

    clk = ClockSampler(local)
    clk.start()
    barrier()
    ms_mixed, ms_a_mixed, its_mixed, launches, _ = timed(capi.CTH_PREC_MIXED, args.steps)
    barrier()
    ms_fp64, ms_a_fp64, its_fp64, _, _ = timed(capi.CTH_PREC_FP64, args.steps)
    barrier()
    clocks = clk.stop()
    # kernel-level profile pass (events around kernels of (a); not part of value)
    nprof = max(3, args.steps // 2)
    _, _, _, _, prof = timed(capi.CTH_PREC_MIXED, nprof, profile=True)
    barrier()

    # solution checks of the last solves (FP64 residuals on the device / host)
    solve_a(capi.CTH_PREC_MIXED)
    rn, bn = g.residual_dev(*planes, x)
    stb, pb = solve_b()
    relres_b = stb.residual

    # end-to-end through the public API with pinned host buffers
    pin = {k: torch.from_numpy(sa[k]).pin_memory().numpy() for k in ("aP", "aE", "aW", "aN", "aS", "b")}
    pinb = {k: torch.from_numpy(wb[k]).pin_memory() for k in ("ne", "nu", "epsr")}
    xs = torch.zeros((NI + 2, NJ + 2), dtype=torch.float64).pin_memory().numpy()
    eb_host = torch.empty((NJ + 2, gb.ld), dtype=torch.complex128).pin_memory()
    dfields = [torch.empty((NI + 2, NJ + 2), dtype=torch.float64, device=dev) for _ in range(3)]

    def e2e_step():
        pkg.solver_SMG(pin["aP"], pin["aE"], pin["aW"], pin["aN"], pin["aS"], pin["b"], sa["i_bl"],
                       sa["j_bl"], 1, MAXIT, TOL, 0, xs, precision=capi.CTH_PREC_MIXED, device=local)
        for d, k in zip(dfields, ("ne", "nu", "epsr")):
            d.copy_(pinb[k], non_blocking=True)
        dev_fields = []
        for d in dfields:
            plane = gb.device_plane(1)[0]
            capi.check(gb._L.cth_to_device_layout(gb._h, d.data_ptr(), plane.data_ptr(), stream.cuda_stream),
                       allow_positive=False)
            dev_fields.append(plane)
        pbx = gb.mw_er_assemble_dev(*dev_fields, wb["params"], stream=stream)
        gb.c5_solve_dev(*pbx, eb, maxITR=200, error_cnv=TOL, stream=stream)
        eb_host.copy_(eb, non_blocking=True)
        torch.cuda.synchronize(dev)

    for _ in range(2):
        e2e_step()
    barrier()
    e2e_steps = max(3, args.steps // 2)
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        flush.zero_()
        torch.cuda.synchronize(dev)
        e2e_step()
    e2e_s = time.perf_counter() - t0
    te = torch.tensor([e2e_s], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(te, op=dist.ReduceOp.MAX)
    e2e_s = float(te.item())

    if world > 1:
        dist.destroy_process_group()
    if rank != 0:
        return 0

    nbytes_ij = (NI + 2) * (NJ + 2) * 8
    value = world * args.steps / (ms_mixed / 1e3)
    fp64_value = world * args.steps / (ms_fp64 / 1e3)
    peaks = measured_peaks()
    peak = peaks["hbm_gbs"] if peaks else 6650.0
    r_ms, r_n, r_bytes = prof[capi.CTH_PROF_RELAX0]
    achieved = (r_bytes / r_n) / (r_ms / r_n / 1e3) / 1e9 if r_n else None
    u_ms, u_n, u_bytes = prof[capi.CTH_PROF_UPDATE]
    upd = (u_bytes / u_n) / (u_ms / u_n / 1e3) / 1e9 if u_n else None
    traffic = ncu_traffic()

    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_mixed / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64 (a), complex f64 (b)",
        "data": "synthetic (seeded)",
        "config": workload_config({"parallelism": f"replicas x{world}" if world > 1 else "single GPU"}),
        "poisson_ms": ms_a_mixed / args.steps, "helmholtz_ms": (ms_mixed - ms_a_mixed) / args.steps,
        "fp64": {"value": fp64_value, "unit": UNIT, "ms_per_step": ms_fp64 / args.steps,
                 "poisson_ms": ms_a_fp64 / args.steps},
        "mixed_over_fp64": value / fp64_value,
        "poisson_mixed_over_fp64": ms_a_fp64 / ms_a_mixed,
        "cycles_poisson": its_mixed[-1][0], "iterations_helmholtz": its_mixed[-1][1],
        "final_relres": {"poisson": rn / bn, "helmholtz": relres_b},
        "gpu_launches": launches,
        "e2e": {"value": world * e2e_steps / e2e_s, "unit": UNIT,
                "h2d_bytes_per_step": 6 * nbytes_ij + 3 * nbytes_ij,
                "d2h_bytes_per_step": nbytes_ij + (NJ + 2) * gb.ld * 16,
                "timing": "host wall clock around the synchronous public-API calls"},
        "roofline": {"bound": "hbm", "kernel": "k_relax<float,5,0> (finest-level z-line relaxation of (a))",
                     "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": (achieved / peak) if achieved else None,
                     "traffic": traffic,
                     "peak_source": "MEASURED_PEAKS.json hbm_gbs (measured)" if peaks else "fallback 6650",
                     "launch_us": 1e3 * r_ms / r_n if r_n else None,
                     "algorithmic_bytes_per_launch": r_bytes / r_n if r_n else None},
        "kernels": {
            "update_fp64_residual": {"GB/s": upd, "launch_us": 1e3 * u_ms / u_n if u_n else None},
            "setup_ms_per_solve": prof[capi.CTH_PROF_SETUP][0] / max(1, prof[capi.CTH_PROF_SETUP][1]),
            "relax0_share_of_step": (r_ms / nprof) / (ms_mixed / args.steps),
        },
        "clocks": clocks,
    }
    if world == 1 and not args.no_cpu:
        v, n, el = cpu_sample(sa, wb)
        line["cpu_baseline"] = {"value": v, "unit": UNIT, "cores": os.cpu_count(), "kind": "port",
                                "sample": f"{n} full steps in {el:.1f} s: (a) CPU restatement of solver_SMG "
                                          f"(OpenMP over {os.cpu_count()} threads), (b) assembly + SuperLU "
                                          f"direct solve (single thread)"}
    print(json.dumps(line), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
