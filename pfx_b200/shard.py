"""One frame rendered by several ranks (one process per GPU).

Pixels are independent: a pixel's samples depend only on its full-frame
position, the sample index and the seed (Trace::set_window, gpu.rs:2836, keeps
the full-frame coordinates of a tile's pixels).  So each rank traces one band
of rows of the frame with its own tracer, with no exchange while it samples.
The only collective is the gather of the finished bands into the full frame:
one all-gather of equal-sized (padded) RGBA32F bands, on NCCL between GPUs or
gloo on the host.

    rank, ranks = dist.get_rank(), dist.get_world_size()
    trace, (y0, rows) = render_band(scene, settings, width, height, rank, ranks, spp=16, seed=0)
    frame = gather_frame(dist, trace.films_device()[0], y0, rows, width, height)   # on every rank
"""
from __future__ import annotations

from .trace import SceneDesc, Settings, Trace


def band(height: int, rank: int, ranks: int) -> tuple:
    """(first row, rows) of `rank`'s band: the first height % ranks ranks take
    one row more, so bands differ by at most one row."""
    if not (0 <= rank < ranks) or height < ranks:
        raise ValueError("every rank needs at least one row")
    base, extra = divmod(height, ranks)
    rows = base + (1 if rank < extra else 0)
    first = rank * base + min(rank, extra)
    return first, rows


def render_band(scene: SceneDesc, settings: Settings, width: int, height: int, rank: int, ranks: int, spp: int,
                seed: int, trace: Trace | None = None):
    """Trace `spp` samples of `rank`'s band of the width x height frame; returns
    the tracer (its films are the band) and (first row, rows).  A tracer of the
    band's size may be passed in to be reused."""
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
    (rows, width, 4) float32 tensor (on the rank's GPU for NCCL, on the host for
    gloo); returns the (height, width, 4) frame on every rank."""
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
