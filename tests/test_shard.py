"""One frame over ranks (pfx_b200.shard): the golden-ratio strips and their
halo rows, contiguous bands and the gathers, and an adaptive render whose
strips are sampled by two and three CPU ranks (gloo, the oracle renderer)
equal to one renderer's; rendezvous on 127.0.0.1."""
import os
import socket
import sys
from pathlib import Path

import numpy as np
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


# ------------------------------------------------------------ strips
def test_strips_are_dealt_in_golden_ratio_order():
    # block_stride (gpu.rs:1198-1207): nearest blocks*(1-1/phi), coprime
    assert shard.block_stride(2) == 1 and shard.block_stride(1) == 1
    assert shard.block_stride(270) == 103  # the 4K frame's 8-row strips
    assert shard.block_stride(10) == 7     # round(3.82) = 4 is not coprime with 10: the search goes upwards
    for height in (8, 23, 40, 2160):
        blocks = -(-height // 8)
        for ranks in (1, 2, 3, 8):
            if blocks < ranks:
                with pytest.raises(ValueError):
                    shard.strips(height, 0, ranks)
                continue
            mine = [shard.strips(height, r, ranks) for r in range(ranks)]
            assert sorted(b for m in mine for b in m) == list(range(blocks))
            assert max(map(len, mine)) - min(map(len, mine)) <= 1
            rows = np.concatenate([shard.strip_rows(height, m) for m in mine])
            assert sorted(rows.tolist()) == list(range(height))
    # on the 4K frame every one of 8 ranks gets strips from the whole height
    for r in range(8):
        b = shard.strips(2160, r, 8)
        assert min(b) < 60 and max(b) > 210


def test_halo_rows_are_the_neighbours_edge_rows():
    height, ranks = 61, 3
    for r in range(ranks):
        mine = shard.strips(height, r, ranks)
        own = set(shard.strip_rows(height, mine).tolist())
        halo = shard.halo_rows(height, mine)
        for y in own:
            for dy in (-1, 1):
                if 0 <= y + dy < height and y + dy not in own:
                    assert y + dy in halo
        others = set()
        for k in range(ranks):
            if k != r:
                others |= set(shard.edge_rows(height, shard.strips(height, k, ranks)).tolist())
        assert set(halo.tolist()) <= others


class OracleStrips:
    """shard.StripTracer's interface over the CPU oracle: a full-frame
    accumulation of which only this rank's strips are sampled."""

    def __init__(self, w, rank, ranks):
        import oracle
        self.width, self.height, self.rank, self.ranks = w.width, w.height, rank, ranks
        self.blocks = shard.strips(w.height, rank, ranks)
        self.mask = shard.strip_mask(w.width, w.height, self.blocks)
        buffers = oracle.scene_buffers(w.scene, w.settings)
        self.r = oracle.Renderer(buffers, w.settings)
        self.frame = oracle.frame_of(w.scene, w.width, w.height, buffers.buffers.triangle_count)
        self.accum = np.zeros((w.height, w.width, 12), np.float32)
        self.snaps = np.zeros((w.height, w.width, 8), np.float32)
        self.samples = 0

    def rows(self):
        return shard.strip_rows(self.height, self.blocks)

    def sample(self, count, seed):
        self.r.render(self.frame, self.accum, self.samples, count, seed, mask=self.mask)
        self.samples += count

    def measure(self, first):
        if first:
            self.snaps[:] = 0.0
        self.r.measure(self.accum, self.snaps)

    def errors(self, rows):
        import torch
        return torch.from_numpy(self.snaps[rows, :, 5].copy())

    def set_errors(self, rows, values):
        self.snaps[rows, :, 5] = values.numpy()

    def mark(self, min_samples, threshold):
        return self.r.mark(self.accum, self.snaps, min_samples, threshold)

    def device(self):
        import torch
        return torch.device("cpu")


def _adaptive_scene():
    from pfx_b200 import synth
    from pfx_b200.trace import Adaptive, Settings
    w = synth.small("instanced_1080", (40, 30), sampler="sobol")
    w.settings = Settings.deep(8, sampler="sobol", sobol_samples=64)
    return w, Adaptive(threshold=0.05, min_samples=8, max_samples=32, growth=1.5)


def _strip_rank(rank, world, port, out):
    import datetime

    import torch
    import torch.distributed as dist

    sys.path.insert(0, str(ROOT))
    sys.path.insert(0, str(ROOT / "tests"))
    from pfx_b200 import shard
    from test_shard import OracleStrips, _adaptive_scene

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        w, adaptive = _adaptive_scene()
        tracer = OracleStrips(w, rank, world)
        rounds = shard.sample_adaptive(dist, tracer, adaptive, 11)
        accum = shard.gather_rows(dist, torch.from_numpy(tracer.accum), tracer.rows(), w.height)
        out.put((rank, rounds, accum.numpy()))
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_strips_over_ranks_render_the_one_rank_adaptive_frame(world):
    """Each rank samples its golden-ratio strips with the CPU oracle, exchanges
    the one-row error halo every round and sums the running counts; the rounds
    and the gathered accumulation equal one renderer's of the whole frame bit
    for bit.  (Host logic on gloo ranks; unmeasured on GPUs.)"""
    import oracle

    w, adaptive = _adaptive_scene()
    buffers = oracle.scene_buffers(w.scene, w.settings)
    r = oracle.Renderer(buffers, w.settings)
    frame = oracle.frame_of(w.scene, w.width, w.height, buffers.buffers.triangle_count)
    want_rounds, want_accum, _ = r.sample_adaptive(frame, w.width, w.height, adaptive, 11)
    assert len(want_rounds) >= 3 and 0 < want_rounds[-1][1] < w.width * w.height or want_rounds[-1][1] == 0

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_strip_rank, args=(k, world, port, q)) for k in range(world)]
    for p in procs:
        p.start()
    got = dict((k, (rounds, accum)) for k, rounds, accum in (q.get(timeout=300) for _ in range(world)))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for k in range(world):
        rounds, accum = got[k]
        assert [tuple(x) for x in rounds] == [tuple(x) for x in want_rounds]
        assert np.array_equal(accum.view(np.uint32), want_accum.view(np.uint32))


def test_the_halo_decides_pixels_at_strip_edges():
    """Without the halo rows, mark at a strip's edge sees fewer neighbours and
    stops pixels the whole-frame render keeps running: the exchange matters on
    this scene (three strip owners simulated in one process)."""
    w, adaptive = _adaptive_scene()

    def run(halo):
        ts = [OracleStrips(w, r, 3) for r in range(3)]
        samples, rounds = 0, []
        for step, target in enumerate(adaptive.rounds()):
            count = max(target - samples, 0)
            for t in ts:
                if count:
                    t.sample(count, 11)
            samples += count
            for t in ts:
                t.measure(step == 0)
            if step == 0:
                continue
            if halo:
                for t in ts:
                    for o in ts:
                        if o is not t:
                            rows = np.intersect1d(shard.halo_rows(w.height, t.blocks), o.rows())
                            t.snaps[rows, :, 5] = o.snaps[rows, :, 5]
            rounds.append(sum(t.mark(adaptive.min_samples, adaptive.threshold) for t in ts))
        return rounds

    with_halo, without = run(True), run(False)
    assert with_halo != without
    assert all(a >= b for a, b in zip(with_halo, without))
