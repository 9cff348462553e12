"""The multi-rank path of bench.py on CPU: two gloo ranks (world size 2).

bench.py shards by specimen: every rank builds its own specimens from
rank-dependent seeds and runs them with no data-path collective; the only
collectives are the timing barrier and the max / sum of scalars over ranks
(Dist, over gloo).  Checked here without a GPU: the barrier and the
reductions give the max-over-ranks time and the whole-job sum, and the
per-rank workload seeds differ (no two ranks run the same specimen).
"""
from __future__ import annotations

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
