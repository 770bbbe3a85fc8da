"""One frame split into bands over ranks (pfx_b200.shard): the band split and
the gather of the bands into the frame, on two and three CPU ranks (gloo),
rendezvous on 127.0.0.1."""
import os
import socket
import sys
from pathlib import Path

import pytest
import torch.multiprocessing as mp

from pfx_b200 import shard

ROOT = Path(__file__).resolve().parent.parent


def test_bands_cover_the_frame():
    for height in (1, 7, 23, 2160):
        for ranks in (1, 2, 3, 8):
            if height < ranks:
                with pytest.raises(ValueError):
                    shard.band(height, 0, ranks)
                continue
            rows = [shard.band(height, r, ranks) for r in range(ranks)]
            assert rows[0][0] == 0 and sum(n for _, n in rows) == height
            assert all(a + n == b for (a, n), (b, _) in zip(rows, rows[1:]))
            assert max(n for _, n in rows) - min(n for _, n in rows) <= 1


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, height, width, out):
    import datetime

    import torch
    import torch.distributed as dist

    sys.path.insert(0, str(ROOT))
    from pfx_b200 import shard

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        first, rows = shard.band(height, rank, world)
        # each pixel of the band holds (row, column, rank, 1)
        y = torch.arange(first, first + rows, dtype=torch.float32)[:, None].expand(rows, width)
        x = torch.arange(width, dtype=torch.float32)[None, :].expand(rows, width)
        film = torch.stack([y, x, torch.full_like(x, float(rank)), torch.ones_like(x)], -1)
        frame = shard.gather_frame(dist, film, first, rows, width, height)
        out.put((rank, frame.numpy()))
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world, height", [(2, 9), (3, 10)])
def test_gather_assembles_the_frame(world, height):
    import numpy as np

    width = 5
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, height, width, q)) for r in range(world)]
    for p in procs:
        p.start()
    got = dict(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for r in range(world):
        frame = got[r]
        assert frame.shape == (height, width, 4)
        assert np.array_equal(frame[:, :, 0], np.arange(height, dtype=np.float32)[:, None].repeat(width, 1))
        assert np.array_equal(frame[:, :, 1], np.arange(width, dtype=np.float32)[None, :].repeat(height, 0))
        owners = [shard.band(height, k, world) for k in range(world)]
        for k, (first, rows) in enumerate(owners):
            assert np.all(frame[first:first + rows, :, 2] == k)
