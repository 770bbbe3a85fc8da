"""The multi-GPU host logic of bench.py on two CPU ranks (gloo): every rank
renders its own frame with its own seed (weak scaling, no data-path
collective), the job's time is the slowest rank's and its work the sum of the
ranks'.  The ranks rendezvous on 127.0.0.1."""
import os
import socket
import sys
from pathlib import Path

import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parent.parent


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank: int, world: int, port: int, out):
    import datetime

    import torch.distributed as dist

    sys.path.insert(0, str(ROOT))
    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        assert bench.dist_env() == (world, rank, rank)
        elapsed = 100.0 + 25.0 * rank          # rank 1 is the slow one
        units = 1e6 * (rank + 1)
        t, u = bench.combine_ranks(dist, elapsed, units, "cpu")
        out.put((rank, t, u, bench.rank_seed(rank)))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_ranks_combine_max_time_and_summed_work():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=10) for _ in range(2))
    for rank, t, u, seed in got:
        assert t == 125.0 and u == 3e6
    assert got[0][3] != got[1][3]  # each rank traces its own samples


def test_one_rank_needs_no_process_group():
    sys.path.insert(0, str(ROOT))
    import bench

    assert bench.combine_ranks(None, 7.0, 9.0, "cpu") == (7.0, 9.0)
