"""One frame rendered by several ranks (one process per GPU).

Pixels are independent: a pixel's samples depend only on its full-frame
position, the sample index and the seed.  So the frame is cut into the
reference's 8-row strips and every rank samples its own strips with its own
tracer, with nothing exchanged while it samples.

Which strips a rank takes: the strips in the order the reference dispatches
them, block j -> (j * stride) mod blocks with the golden-ratio stride of
gpu.rs:1198-1214, dealt to the ranks in contiguous runs of that order.  The
order scatters a run over the whole height, so every rank gets some of the
ceiling, the shelves and the floor instead of one band of them.

Adaptive sampling (adaptive.rs:136-325) adds one exchange per round: mark's
3x3 maximum of the errors (converge.wgsl:32-51) reads the row above and the
row below each strip, which other ranks may own.  After measure, every rank
publishes the errors of its strips' first and last rows (one all-gather) and
writes the rows next to its own strips into its snapshots, then marks; the
round's active count is the sum over ranks (one all-reduce).  The rounds and
every pixel's accumulation are then those of one tracer of the whole frame.

The finished strips come together with one all-gather of equal-sized (padded)
row blocks, on NCCL between GPUs or gloo on the host.

    rank, ranks = dist.get_rank(), dist.get_world_size()
    trace = StripTracer(Trace(scene, settings, width, height), rank, ranks)
    conv = sample_adaptive(dist, trace, adaptive, seed)          # or trace.sample(spp, seed)
    frame = gather_rows(dist, trace.films()[0], trace.rows(), height)   # on every rank
"""
from __future__ import annotations

import math

import numpy as np

from .trace import SceneDesc, Settings, Trace

STRIP_ROWS = 8  # the reference's strips (gpu.rs:3188-3231 dispatches 8x8 groups in 8-row strips)


def coprime(a: int, b: int) -> bool:
    return math.gcd(a, b) == 1


def block_stride(blocks: int) -> int:
    """gpu.rs:1198-1207: the stride nearest blocks x (1 - 1/phi) that is coprime
    with `blocks`, searched upwards then from 1."""
    if blocks <= 2:
        return 1
    golden = int(math.floor(blocks * 0.38196601125 + 0.5))
    for stride in list(range(golden, blocks)) + list(range(1, golden)):
        if coprime(stride, blocks):
            return stride
    return 1


def strips(height: int, rank: int, ranks: int, rows: int = STRIP_ROWS) -> list:
    """The strips (block indices, ascending) of `rank`: the golden-ratio order
    of the frame's blocks dealt in contiguous runs, the first blocks % ranks
    ranks taking one block more."""
    blocks = -(-height // rows)
    if not (0 <= rank < ranks) or blocks < ranks:
        raise ValueError("every rank needs at least one strip")
    stride = block_stride(blocks)
    order = [(j * stride) % blocks for j in range(blocks)]
    base, extra = divmod(blocks, ranks)
    first = rank * base + min(rank, extra)
    return sorted(order[first:first + base + (1 if rank < extra else 0)])


def strip_rows(height: int, blocks, rows: int = STRIP_ROWS) -> np.ndarray:
    """Row indices of the given strips, ascending."""
    out = [np.arange(b * rows, min((b + 1) * rows, height)) for b in sorted(blocks)]
    return np.concatenate(out) if out else np.zeros(0, np.int64)


def edge_rows(height: int, blocks, rows: int = STRIP_ROWS) -> np.ndarray:
    """The first and last row of each strip: the rows neighbours may read."""
    out = set()
    for b in blocks:
        out.add(b * rows)
        out.add(min((b + 1) * rows, height) - 1)
    return np.array(sorted(out), np.int64)


def halo_rows(height: int, blocks, rows: int = STRIP_ROWS) -> np.ndarray:
    """Rows next to the strips (above the first, below the last row) that
    belong to other strips."""
    own = set(strip_rows(height, blocks, rows).tolist())
    out = set()
    for b in blocks:
        for y in (b * rows - 1, min((b + 1) * rows, height)):
            if 0 <= y < height and y not in own:
                out.add(y)
    return np.array(sorted(out), np.int64)


def strip_mask(width: int, height: int, blocks, rows: int = STRIP_ROWS) -> np.ndarray:
    m = np.zeros((height, width), bool)
    m[strip_rows(height, blocks, rows)] = True
    return m


class StripTracer:
    """A full-frame tracer that samples only `rank`'s strips (pfxt_set_pixel_mask),
    with the adaptive steps a sharded render needs."""

    def __init__(self, trace: Trace, rank: int, ranks: int):
        self.trace, self.rank, self.ranks = trace, rank, ranks
        self.width, self.height = trace.width, trace.height
        self.blocks = strips(self.height, rank, ranks)
        trace.set_pixel_mask(strip_mask(self.width, self.height, self.blocks))

    def rows(self) -> np.ndarray:
        return strip_rows(self.height, self.blocks)

    def sample(self, count: int, seed: int) -> None:
        self.trace.sample(count, seed)

    def measure(self, first: bool) -> None:
        self.trace.adaptive_measure(first)

    def errors(self, rows):
        """(len(rows), width) errors of those rows (a CUDA tensor)."""
        import torch
        return self.trace.adaptive_snaps_device()[torch.as_tensor(rows, device="cuda"), :, 5].contiguous()

    def set_errors(self, rows, values) -> None:
        import torch
        snaps = self.trace.adaptive_snaps_device()
        snaps[torch.as_tensor(rows, device="cuda"), :, 5] = values.to(snaps.device)
        # the write runs on torch's stream, mark on the tracer's: finish it first
        torch.cuda.current_stream().synchronize()

    def mark(self, min_samples: int, threshold: float) -> int:
        return self.trace.adaptive_mark(min_samples, threshold)

    def films(self):
        return self.trace.films_device()

    def device(self):
        import torch
        return torch.device("cuda", torch.cuda.current_device())


def _all_gather_rows(dist, local, counts, group=None):
    """All-gather of per-rank row blocks of different heights: pads to the
    tallest, gathers once, returns the list of every rank's rows."""
    import torch
    tallest = max(counts)
    padded = torch.zeros((tallest,) + tuple(local.shape[1:]), dtype=local.dtype, device=local.device)
    padded[:len(local)] = local
    out = torch.empty((len(counts) * tallest,) + tuple(local.shape[1:]), dtype=local.dtype, device=local.device)
    dist.all_gather_into_tensor(out, padded, group=group)
    return [out[r * tallest:r * tallest + counts[r]] for r in range(len(counts))]


def exchange_halo(dist, tracer, group=None) -> None:
    """Write into `tracer`'s snapshots the errors of the rows next to its strips
    that other ranks own (their strips' edge rows), after measure."""
    import torch
    ranks, height = tracer.ranks, tracer.height
    edges = [edge_rows(height, strips(height, r, ranks)) for r in range(ranks)]
    mine = torch.as_tensor(tracer.errors(edges[tracer.rank]))
    gathered = _all_gather_rows(dist, mine, [len(e) for e in edges], group)
    need = halo_rows(height, tracer.blocks)
    if len(need) == 0:
        return
    owner_rows, values = [], []
    for r in range(ranks):
        if r == tracer.rank:
            continue
        pick = np.isin(edges[r], need)
        if pick.any():
            owner_rows.append(edges[r][pick])
            values.append(gathered[r][torch.as_tensor(np.flatnonzero(pick), device=gathered[r].device)])
    rows = np.concatenate(owner_rows)
    assert np.array_equal(np.sort(rows), need), "every halo row is an edge row of its owner"
    tracer.set_errors(rows, torch.cat(values))


def sample_adaptive(dist, tracer, adaptive, seed: int, group=None):
    """Trace::sample_adaptive (adaptive.rs:136-325) over the strips of every
    rank; returns the rounds [(samples, active)] of the whole frame, the same
    on every rank."""
    import torch
    rounds, samples = [], 0
    for step, target in enumerate(adaptive.rounds()):
        count = max(target - samples, 0)
        if count:
            tracer.sample(count, seed)
        samples += count
        tracer.measure(step == 0)
        if step == 0:
            active = tracer.width * tracer.height
        else:
            exchange_halo(dist, tracer, group)
            running = torch.tensor([tracer.mark(adaptive.min_samples, adaptive.threshold)], dtype=torch.int64,
                                   device=tracer.device())
            dist.all_reduce(running, group=group)
            active = int(running.item())
        rounds.append((target, active))
        if active == 0:
            break
    return rounds


def gather_rows(dist, local_frame, rows, height: int, group=None):
    """Assemble the full frame from every rank's strip rows: `local_frame` is
    this rank's full-size (height, width, C) tensor of which only `rows` are
    its own; returns the (height, width, C) frame on every rank."""
    import torch
    ranks = dist.get_world_size(group)
    all_rows = [strip_rows(height, strips(height, r, ranks)) for r in range(ranks)]
    mine = local_frame[torch.as_tensor(rows, device=local_frame.device)]
    parts = _all_gather_rows(dist, mine, [len(x) for x in all_rows], group)
    out = torch.empty((height,) + tuple(local_frame.shape[1:]), dtype=local_frame.dtype, device=local_frame.device)
    for r in range(ranks):
        out[torch.as_tensor(all_rows[r], device=out.device)] = parts[r]
    return out


def render_strips(scene: SceneDesc, settings: Settings, width: int, height: int, rank: int, ranks: int, spp: int,
                  seed: int) -> StripTracer:
    """`spp` samples of `rank`'s strips of the width x height frame."""
    t = StripTracer(Trace(scene, settings, width, height), rank, ranks)
    t.sample(spp, seed)
    return t


# ------------------------------------------------------------ contiguous bands
def band(height: int, rank: int, ranks: int) -> tuple:
    """(first row, rows) of `rank`'s band of contiguous rows (a tracer of the
    band's size through Trace::set_window, gpu.rs:2836): the first
    height % ranks ranks take one row more."""
    if not (0 <= rank < ranks) or height < ranks:
        raise ValueError("every rank needs at least one row")
    base, extra = divmod(height, ranks)
    rows = base + (1 if rank < extra else 0)
    first = rank * base + min(rank, extra)
    return first, rows


def render_band(scene: SceneDesc, settings: Settings, width: int, height: int, rank: int, ranks: int, spp: int,
                seed: int, trace: Trace | None = None):
    """Trace `spp` samples of `rank`'s band of the width x height frame; returns
    the tracer (its films are the band) and (first row, rows)."""
    first, rows = band(height, rank, ranks)
    if trace is None:
        trace = Trace(scene, settings, width, rows)
    elif (trace.width, trace.height) != (width, rows):
        raise ValueError("the tracer does not have the band's size")
    trace.set_window((width, height), (0, first))
    trace.sample(spp, seed)
    return trace, (first, rows)


def gather_frame(dist, film, first: int, rows: int, width: int, height: int, group=None):
    """Assemble the full frame from every rank's band: `film` is this rank's
    (rows, width, 4) float32 tensor; returns the (height, width, 4) frame."""
    import torch

    ranks = dist.get_world_size(group)
    tallest = -(-height // ranks)
    padded = torch.zeros((tallest, width, 4), dtype=torch.float32, device=film.device)
    padded[:rows] = film.reshape(rows, width, 4)
    out = torch.empty((ranks * tallest, width, 4), dtype=torch.float32, device=film.device)
    dist.all_gather_into_tensor(out, padded, group=group)
    parts = []
    for r in range(ranks):
        _, n = band(height, r, ranks)
        parts.append(out[r * tallest:r * tallest + n])
    return torch.cat(parts, 0)
