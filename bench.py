#!/usr/bin/env python
"""Throughput of the implicit 5-point solve path on one B200 (or N replicas).

Workload: the isolated 512 (r) x 1024 (z) potential system of the
cathode fluid code (the reference's Poisson stencil with a 1:3.8 dielectric
slab, Dirichlet electrodes at z = 0 / z = L, axis at r = 0; seeded synthetic
space charge), solved from a zero guess to ||b-Ax||_2/||b||_2 < 1e-10.
One step = one complete solve (set-up + cycles + FP64 residual checks).

Reported line (rank 0):
  value        solves/s of the mixed-precision path (FP32 multigrid + FP64
               defect correction), inputs resident in HBM, L2 flushed
               (256 MiB memset) before every step, CUDA events on the stream
  fp64         the same for the plain FP64 multigrid
  e2e          solves/s through the host C ABI (cth_smg_solve) with pinned
               host inputs: H2D of the six input arrays and D2H of the
               solution inside every step
  roofline     finest-level z-line relaxation kernel: algorithmic bytes /
               CUDA-event time vs the measured HBM copy bandwidth
  cpu_baseline the CPU restatement (oracle, OpenMP) on a bounded sample

--impl reference times the CPU restatement of the reference path (the
reference itself needs HYPRE/MPI/Eigen/yaml-cpp, which are not installed)
on the same workload and prints the same metric.
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
        "workload": "isolated potential system, 512 (r) x 1024 (z) cells, slab epsr 3.8, "
                    "Dirichlet electrodes 0/20 V, axis; one step = one solve to 1e-10 relative residual",
        "ni_z": NI, "nj_r": NJ, "tol": TOL, "maxit": MAXIT,
        "l2": "256 MiB memset between timed steps (working set < L2)",
        "method": "semicoarsening MG (z-line zebra smoother, Galerkin), FP32 cycles + FP64 defect correction",
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
                                          "--format=csv,noheader,nounits", "-lms", "100"],
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
def cpu_solves(s, budget_s=12.0, max_solves=40):
    import oracle
    oracle.build()
    n = 0
    t0 = time.perf_counter()
    while True:
        _, rc, it, rel = oracle.smg_solve(s, MAXIT, TOL)
        n += 1
        el = time.perf_counter() - t0
        if el > budget_s or n >= max_solves:
            break
    return n / el, n, el, rel


def run_reference(args, rank, world):
    if rank != 0:
        return 0
    import __graft_entry__
    pkg = __graft_entry__.load_package()
    import oracle
    oracle.build()
    s = pkg.workloads.poisson_slab(NI, NJ, seed=1)
    threads = os.cpu_count()
    for _ in range(args.warmup):
        oracle.smg_solve(s, MAXIT, TOL)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        _, rc, it, rel = oracle.smg_solve(s, MAXIT, TOL)
        times.append(time.perf_counter() - t0)
    tot = sum(times)
    v = args.steps / tot
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * tot / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded)", "config": workload_config({"parallelism": "host threads"}),
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": f"{args.steps} full 512x1024 solves to 1e-10 (CPU restatement of "
                                   f"solver_SMG: semicoarsening MG, OpenMP); the reference's HYPRE build is "
                                   f"not installable here"},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "last_relres": rel,
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
    s = pkg.workloads.poisson_slab(NI, NJ, seed=1 + rank)
    g = pkg.Grid(NI, NJ, s["i_bl"], s["j_bl"], device=local)
    planes = [g.to_device(s[k]) for k in ("aP", "aE", "aW", "aN", "aS", "b")]
    x = g.device_plane(1)[0]
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream(dev)

    def solve(prec):
        return g.smg_solve_dev(*planes, x, maxITR=MAXIT, error_cnv=TOL, precision=prec, stream=stream)

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize(dev)

    def timed(prec, steps, profile=False):
        if profile:
            g.profile(True)
        ms = 0.0
        iters = []
        l0 = g.launch_count()
        for _ in range(steps):
            flush.zero_()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            st = solve(prec)
            e1.record(stream)
            e1.synchronize()
            ms += e0.elapsed_time(e1)
            iters.append(st.iterations)
            if not st.converged:
                raise RuntimeError(f"solve did not converge: {st.as_dict()}")
        launches = g.launch_count() - l0
        prof = None
        if profile:
            prof = {c: g.profile_read(c) for c in (capi.CTH_PROF_RELAX0, capi.CTH_PROF_UPDATE,
                                                   capi.CTH_PROF_RESTRICT0, capi.CTH_PROF_SETUP)}
            g.profile(False)
        t = torch.tensor([ms], dtype=torch.float64, device=dev)
        if world > 1:
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item()), iters, launches, prof

    # warm-up (both precisions)
    for _ in range(max(args.warmup, 3)):
        solve(capi.CTH_PREC_MIXED)
        solve(capi.CTH_PREC_FP64)
    barrier()

    clk = ClockSampler(local)
    clk.start()
    barrier()
    ms_mixed, it_mixed, launches, _ = timed(capi.CTH_PREC_MIXED, args.steps)
    barrier()
    clocks = clk.stop()
    ms_fp64, it_fp64, _, _ = timed(capi.CTH_PREC_FP64, args.steps)
    barrier()
    # kernel-level profile pass (events around kernels; not part of value)
    _, _, _, prof = timed(capi.CTH_PREC_MIXED, max(3, args.steps // 2), profile=True)
    barrier()

    # solution check of the last solve (FP64 residual on the device)
    solve(capi.CTH_PREC_MIXED)
    rn, bn = g.residual_dev(*planes, x)

    # end-to-end through the host C ABI with pinned host buffers
    pin = {k: torch.from_numpy(s[k]).pin_memory().numpy() for k in ("aP", "aE", "aW", "aN", "aS", "b")}
    xs = torch.zeros((NI + 2, NJ + 2), dtype=torch.float64).pin_memory().numpy()
    for _ in range(2):
        pkg.solver_SMG(pin["aP"], pin["aE"], pin["aW"], pin["aN"], pin["aS"], pin["b"], s["i_bl"],
                       s["j_bl"], 1, MAXIT, TOL, 0, xs, precision=capi.CTH_PREC_MIXED, device=local)
    barrier()
    t0 = time.perf_counter()
    e2e_steps = max(3, args.steps // 2)
    for _ in range(e2e_steps):
        flush.zero_()
        torch.cuda.synchronize(dev)
        pkg.solver_SMG(pin["aP"], pin["aE"], pin["aW"], pin["aN"], pin["aS"], pin["b"], s["i_bl"],
                       s["j_bl"], 1, MAXIT, TOL, 0, xs, precision=capi.CTH_PREC_MIXED, device=local)
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
        "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64", "data": "synthetic (seeded)",
        "config": workload_config({"parallelism": f"replicas x{world}" if world > 1 else "single GPU"}),
        "fp64": {"value": fp64_value, "unit": UNIT, "ms_per_step": ms_fp64 / args.steps,
                 "cycles": it_fp64[-1]},
        "mixed_over_fp64": value / fp64_value,
        "cycles": it_mixed[-1],
        "final_relres": rn / bn,
        "gpu_launches": launches,
        "e2e": {"value": world * e2e_steps / e2e_s, "unit": UNIT, "h2d_bytes_per_step": 6 * nbytes_ij,
                "d2h_bytes_per_step": nbytes_ij, "timing": "host wall clock around the synchronous C-ABI call"},
        "roofline": {"bound": "hbm", "kernel": "k_relax<float,5> (finest-level z-line relaxation)",
                     "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": (achieved / peak) if achieved else None,
                     "traffic": traffic,
                     "peak_source": "MEASURED_PEAKS.json hbm_gbs (measured)" if peaks else "fallback 6650",
                     "launch_us": 1e3 * r_ms / r_n if r_n else None,
                     "algorithmic_bytes_per_launch": r_bytes / r_n if r_n else None},
        "kernels": {
            "update_fp64_residual": {"GB/s": upd, "launch_us": 1e3 * u_ms / u_n if u_n else None},
            "setup_ms_per_solve": prof[capi.CTH_PROF_SETUP][0] / max(1, prof[capi.CTH_PROF_SETUP][1]),
            "relax0_share_of_step": (r_ms / (max(3, args.steps // 2))) / (ms_mixed / args.steps),
        },
        "clocks": clocks,
    }
    if world == 1 and not args.no_cpu:
        v, n, el, rel = cpu_solves(s)
        line["cpu_baseline"] = {"value": v, "unit": UNIT, "cores": os.cpu_count(), "kind": "port",
                                "sample": f"{n} full 512x1024 solves in {el:.1f} s (CPU restatement of "
                                          f"solver_SMG, OpenMP over {os.cpu_count()} host threads)"}
    print(json.dumps(line), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
