"""The batched I-V sweep split over ranks (one process per GPU, no collective
while the instances run, one all-gather of the per-instance I-V points at the
end): the partition balanced by cells x steps, and the sharded run over two
gloo ranks on the CPU giving the same table as one rank.  The CPU runner
advances each instance with the oracle's whole time step (test
infrastructure) on a small grid; on GPUs the runner is batch.gpu_runner."""
import os
import socket

import numpy as np
import pytest

SIZES = ((8, 12), (10, 16), (12, 20))   # (r cells, z cells): small enough for the oracle


def _pkg():
    import __graft_entry__
    return __graft_entry__.load_package()


def cpu_runner(sel):
    """One oracle time step per instance (rectangle, the spec's bias); returns summaries."""
    import oracle
    from oracle import fluid
    pkg = _pkg()
    out = []
    for sp in sel:
        ni, nj = sp["ni"], sp["nj"]
        geo = pkg.fluid.rectangle_geometry(ni, nj, width_neutIn=2.03e-3)
        og = fluid.rectangle_geometry(ni, nj)
        ds = pkg.workloads.discharge_state(ni, nj, seed=sp["seed"] % 1000)
        cfg = pkg.workloads.discharge_params(geo, ds["dr"], 5e-3)
        P = cfg["params"]
        P["phi"]["V_bias"] = sp["V_bias"]
        P["neutral"].update(xL=geo["xL"], x6=geo["x6"], width_neutIn=geo["width_neutIn"])
        st = {k: np.zeros((ni + 2, nj + 2)) for k in ("phi", "Ex", "Er", "nUex", "nUer", "Uix", "Uir", "Uip",
                                                       "rhoUix", "rhoUir", "rhoUix_wall", "rhoUir_wall", "rhoUex",
                                                       "rhoUer", "rhoUex_wall", "rhoUer_wall", "Gx", "Gr", "Gx_wall",
                                                       "Gr_wall", "rhoUnx", "rhoUnr", "rhoUnx_wall", "rhoUnr_wall",
                                                       "rhoUmx", "rhoUmr", "rhoUmx_wall", "rhoUmr_wall", "nu_ano",
                                                       "nu_ano_IAT", "Pabs")}
        st.update(ds["fields"])
        st["rhoe_old"] = st["rhoe"].copy()
        see = (cfg["see"]["coefEISEE_eb_table"], cfg["see"]["coefEISEE_rd_table"], cfg["see"]["coefEISEE_ts_table"],
               P["phi"]["dTe_SEE"])

        def solve(aP, aE, aW, aN, aS, b, ib, jb):
            return oracle.direct_solve(dict(ni=ni, nj=nj, i_bl=ib, j_bl=jb, aP=aP, aE=aE, aW=aW, aN=aN, aS=aS, b=b))

        so = fluid.update_transport_coef(st, cfg["tables"], P["transport"], og["flags"])
        so = fluid.fluid_step(so, P, og, see, cfg["tables"], solve)
        out.append(dict(index=sp["index"], ni=ni, nj=nj, V_bias=sp["V_bias"], Pmw=sp["Pmw"], itime=P["itime"],
                        I_Anode=float(so["I_Anode"]), Ii_Anode=float(so["Ii_Anode"]), Ie_Anode=float(so["Ie_Anode"]),
                        rc=0))
    return out


def test_partition_balances_cells_times_steps():
    B = _pkg().batch
    specs = B.instance_specs(64, seed=3)
    cost = {s["index"]: s["ni"] * s["nj"] for s in specs}
    biggest = max(cost.values())
    for world in (1, 2, 3, 4, 8):
        parts = B.partition(specs, world, steps=2000)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(64)), world
        loads = [sum(cost[i] for i in p) for p in parts]
        # largest-first greedy: no rank exceeds another by more than one instance
        assert max(loads) - min(loads) <= biggest, (world, loads)
        assert parts == B.partition(specs, world, steps=2000)   # every rank computes the same split
    # per-instance step counts enter the cost
    steps = [10] * 63 + [10 ** 6]
    parts = B.partition(specs, 2, steps=steps)
    heavy = [p for p in parts if 63 in p][0]
    assert heavy == [63]


def test_instance_specs_independent_of_split():
    B = _pkg().batch
    a = B.instance_specs(16, seed=5)
    b = B.instance_specs(16, seed=5)
    assert a == b
    # the sweep's draws are those of sweep_instances before the split existed: sizes from SIZES
    assert all((s["nj"], s["ni"]) in B.SIZES for s in a)
    assert all(-10.0 <= s["V_bias"] <= 60.0 and 2.0 <= s["Pmw"] <= 16.0 for s in a)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, n, q):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        B = _pkg().batch
        specs = B.instance_specs(n, seed=7, sizes=SIZES)
        mine = B.partition(specs, world, steps=1)[rank]
        local = B.run_shard(specs, mine, cpu_runner)
        table = B.gather(local, world)
        q.put((rank, mine, table))
    finally:
        dist.destroy_process_group()


def test_sharded_sweep_two_gloo_ranks_equals_one_rank():
    import multiprocessing as mp
    B = _pkg().batch
    n = 6
    specs = B.instance_specs(n, seed=7, sizes=SIZES)
    serial = B.gather(B.run_shard(specs, list(range(n)), cpu_runner), 1)
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, n, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=300) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    mine = {r: m for r, m, _ in res}
    assert sorted(mine[0] + mine[1]) == list(range(n)) and not set(mine[0]) & set(mine[1])
    for _, _, table in res:
        assert [t["index"] for t in table] == list(range(n))
        for a, b in zip(table, serial):
            assert a == b   # the same I-V points, bit for bit, whichever rank ran the instance
    assert any(abs(t["I_Anode"]) > 0 for t in serial)
