"""The multi-rank paths on CPU: two gloo ranks (world size 2).

bench.py shards by specimen: every rank builds its own specimens from
rank-dependent seeds and runs them with no data-path collective; the only
collectives are the timing barrier and the max / sum of scalars over ranks
(Dist, over gloo).  Checked here without a GPU: the barrier and the
reductions give the max-over-ranks time and the whole-job sum, and the
per-rank workload seeds differ (no two ranks run the same specimen).

A calibration sweep is split into contiguous blocks of cases (sweep.shard)
and its per-case macro properties are exchanged afterwards
(sweep.gather_results, one all_gather).  Checked with a real solve on each
rank: every case of a six-case sweep (micro-parameters from the sweep's
Latin hypercube, small reference-mode cylinders) is loaded by the oracle's
whole loading test on the rank that owns it; after the exchange both ranks
hold all six results in case order, identical to one process solving the
whole sweep, and a case claimed by two ranks is an error.
"""
from __future__ import annotations

import importlib
import multiprocessing as mp
import os
import socket
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank: int, ws: int, port: int, q) -> None:
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(ws), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    sys.path.insert(0, str(ROOT))
    import bench

    ws_, rank_, local = bench.dist_env()
    D = bench.Dist(ws_)
    D.barrier()
    ms = 10.0 + rank_                      # a per-rank device time
    out = dict(rank=rank_, ws=ws_, local=local, max=D.max(ms), sum=D.sum(100.0 * (rank_ + 1)),
               sizes=bench.sweep_sizes(16, 11 + rank_),
               seeds=[1 + rank_ * 2 + k for k in range(2)])   # the default bench's specimen seeds
    D.barrier()
    D.close()
    q.put(out)


N_CASES = 6


def _solve_case(k: int) -> dict:
    """Case k of the sweep, solved by the oracle: a reference-mode cylinder
    (specimen k mod 2) with the case's bond modulus and strengths, uniaxial
    loading for at most 600 steps."""
    import dem_testlib as T
    import numpy as np
    from oracle import drive, sim

    sweep = importlib.import_module("dem-rock-calibration_b200.sweep")
    p = sweep.latin_hypercube(N_CASES, 3)[k]
    c = T.ref_case(seed=1 + k % 2, lsi=(0.003, 0.003, 0.004), space=(0.006, 0.006, 0.008), E=p["E_bond"] * 1e9,
                   Ec=p["strength"] * 1e9, Gc=p["strength"] * 1e9, velocity_si=-0.5, maxstrain=0.004,
                   lattice_gap=0.5, jitter_frac=0.1)
    st = sim.RefState.empty(c.N)
    st.R[:] = c.R
    sim.oracle_setup_bonds(st, c.sc)
    bonds0 = int(np.count_nonzero(st.ILtype == 1)) // 2
    o = drive.loading_run(st, c.sc, brazil=False, size_real=list(c.smp.size_real),
                          center_real=list(c.smp.center_real), p_r=c.pot.p_r, min_stress=c.cmp.MinStress,
                          max_strain=c.cmp.MaxStrain, cond_fracture=c.cmp.ConditionFracture, velocity=c.sc.wall_V,
                          dt=c.sc.dt, dNsave=20, max_steps=600)
    E, _ = drive.chord_moduli(o["rec"], None)
    sig = 0.5 * (np.abs(o["rec"][:, 1]) + np.abs(o["rec"][:, 2]))
    return dict(FractureStress=o["FractureStress"], FractureStrain=o["FractureStrain"], E_chord=E, nu=0.0,
                Strain=o["Strain"], Stress=float(sig[-1]), Destruction=0.0, dt=c.sc.dt, steps=o["steps"],
                bonds_initial=bonds0, bonds_now=int(np.count_nonzero(st.ILtype == 1)) // 2,
                fracture=int(o["fracture"]), done=1, numeric=0)


def _sweep_rank(rank: int, ws: int, port: int, q) -> None:
    # one host thread per rank: the oracle's OpenMP loops and torch's thread
    # pool would otherwise oversubscribe the cores between the two ranks
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(ws), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port), OMP_NUM_THREADS="1")
    sys.path[:0] = [str(ROOT), str(ROOT / "tests")]
    import datetime

    import torch.distributed as td

    sweep = importlib.import_module("dem-rock-calibration_b200.sweep")
    td.init_process_group("gloo", timeout=datetime.timedelta(seconds=120))
    mine = list(sweep.shard(N_CASES, rank, ws))
    whole = sweep.gather_results({k: _solve_case(k) for k in mine}, N_CASES)
    # a case claimed by both ranks is refused on every rank
    dup = None
    try:
        sweep.gather_results({0: _solve_case(0)}, N_CASES)
    except RuntimeError as e:
        dup = str(e)
    td.destroy_process_group()
    q.put(dict(rank=rank, mine=mine, whole=whole, dup=dup))


def test_sharded_sweep_gathers_every_case_in_order():
    sys.path[:0] = [str(ROOT), str(ROOT / "tests")]
    sweep = importlib.import_module("dem-rock-calibration_b200.sweep")
    assert [list(sweep.shard(7, r, 3)) for r in range(3)] == [[0, 1], [2, 3], [4, 5, 6]]
    assert [len(sweep.shard(100, r, 8)) for r in range(8)] == [12, 13, 12, 13, 12, 13, 12, 13]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_sweep_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    outs = sorted((q.get(timeout=300) for _ in procs), key=lambda d: d["rank"])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert outs[0]["mine"] == [0, 1, 2] and outs[1]["mine"] == [3, 4, 5]
    # one process solving the whole sweep
    want = [_solve_case(k) for k in range(N_CASES)]
    for o in outs:
        assert len(o["whole"]) == N_CASES
        for k in range(N_CASES):
            for f in sweep.MACRO_FIELDS:
                assert o["whole"][k][f] == want[k][f], (o["rank"], k, f)
        assert o["dup"] is not None and "two ranks" in o["dup"]
    # the sweep is not degenerate: the cases differ
    assert len({round(w["E_chord"], 9) for w in want}) == N_CASES
    assert all(w["steps"] > 0 and w["FractureStress"] > 0 for w in want)


def test_two_gloo_ranks_time_and_sum_over_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    outs = sorted((q.get(timeout=120) for _ in procs), key=lambda d: d["rank"])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [o["ws"] for o in outs] == [2, 2]
    assert all(o["max"] == 11.0 for o in outs)          # the slowest rank's time
    assert all(o["sum"] == 300.0 for o in outs)         # whole-job throughput = sum over ranks
    assert outs[0]["sizes"] != outs[1]["sizes"]         # different sweep specimens per rank
    assert not set(outs[0]["seeds"]) & set(outs[1]["seeds"])
