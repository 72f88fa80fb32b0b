"""Fixture of the small FP64 discharge: the r-z rectangle of 100 (r, 0-5 mm) x
200 (z, 0-10 mm) cells, seeded Gaussian plasma, cusp field, 20 V bias, Pmw = 8 W,
the reference's loop with the microwave update every 100 steps
(src/main.cpp:170-257), run for 1000 steps by the restated time step
(oracle/discharge.py, whose FluidModule part equals the reference's own code
bit for bit on the cathode geometry; tests/test_ref_pin.py) with exact solves
(what HYPRE SMG converges to).

Writes beside this script:
* config0_rect_100x200.npz -- phi, rhoe, rhoi, Te, Ex, Er after steps 100, 150
  and 1000 as ``s0100_phi`` etc.;
* config0_sensitivity.json -- the same loop started from n_e (= n_i) changed by
  a relative 1e-12 (seeded): rel-L2 between the two runs per field after
  steps 100, 150, 200, 500, 1000, and the largest Te of the unperturbed run.
  After the first microwave update the absorbed 8 W heats the electrons of
  this small volume to hundreds of eV and the loop amplifies differences of
  1e-12 to O(1e-3) within a hundred steps, so a comparison with any other
  implementation is meaningful up to step ~150 only.

The two runs go in two processes (about 50 minutes on 16 host threads).

    python tests/golden/make_config0.py
"""
import json
import multiprocessing as mp
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
NI, NJ = 200, 100
SAVE = (100, 150, 200, 500, 1000)
FIXTURE_STEPS = (100, 150, 1000)
KEYS = ("phi", "rhoe", "rhoi", "Te", "Ex", "Er")


def run(perturb: bool) -> dict:
    sys.path.insert(0, ROOT)
    import __graft_entry__
    pkg = __graft_entry__.load_package()
    from oracle import discharge
    geo = pkg.fluid.rectangle_geometry(NI, NJ, width_neutIn=2.03e-3)
    ds = pkg.workloads.discharge_state(NI, NJ, seed=0)
    cfg = pkg.workloads.discharge_params(geo, ds["dr"], 5e-3)
    st = {k: np.zeros((NI + 2, NJ + 2)) for k in pkg.discharge.FIELDS}
    st.update(ds["fields"])
    if perturb:
        eps = 1e-12 * np.random.default_rng(77).standard_normal((NI + 2, NJ + 2))
        st["rhoe"] = st["rhoe"] * (1.0 + eps)
        st["rhoi"] = st["rhoi"] * (1.0 + eps)
    st["rhoe_old"] = st["rhoe"].copy()
    ch = discharge.RectangleChain(st, cfg, geo, NI, NJ)
    out = {}
    t0 = time.time()
    for n in range(1, max(SAVE) + 1):
        ch.step()
        if n in SAVE:
            out[n] = {k: np.array(ch.s[k], dtype=np.float64) for k in KEYS}
            print("perturbed" if perturb else "reference", "step", n, f"{time.time() - t0:.0f} s", flush=True)
    return out


def rel_l2(a, b):
    m = np.zeros(a.shape, bool)
    m[1:NI + 1, 1:NJ + 1] = True
    return float(np.linalg.norm((a - b)[m]) / np.linalg.norm(b[m]))


def main():
    sys.path.insert(0, ROOT)
    import oracle
    oracle.build()                      # once, before the two runs start
    with mp.get_context("spawn").Pool(2) as pool:
        ref, per = pool.map(run, [False, True])
    np.savez_compressed(os.path.join(HERE, "config0_rect_100x200.npz"),
                        **{f"s{n:04d}_{k}": ref[n][k] for n in FIXTURE_STEPS for k in KEYS})
    sens = {"perturbation": "n_e = n_i times (1 + 1e-12 N(0,1)), seed 77", "steps": {}}
    for n in SAVE:
        sens["steps"][str(n)] = dict({k: rel_l2(per[n][k], ref[n][k]) for k in ("phi", "rhoe", "rhoi", "Te")},
                                     max_Te_K=float(np.max(ref[n]["Te"])))
    with open(os.path.join(HERE, "config0_sensitivity.json"), "w") as f:
        json.dump(sens, f, indent=1)


if __name__ == "__main__":
    main()
