"""Splitting one DEM's computable grid across ranks (one process per GPU).

Every (point of view, direction, sector) band is independent, so a row range
of the computable grid is a complete unit of work: rank r sweeps rows
shard_rows(...)[r] for all 180 sectors (tvs_params.tvs_row_begin/end), each
point keeps the reference's per-point f32 summation order, and the only
exchange is gathering the finished rows (no collective on the data path).
"""

import numpy as np


def shard_rows(tvs_height, rank, world):
    """Contiguous, balanced [begin, end) rows of the computable grid for `rank`."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("rank outside [0, world)")
    base, extra = divmod(tvs_height, world)
    begin = rank * base + min(rank, extra)
    return begin, begin + base + (1 if rank < extra else 0)


def gather_rows(rows, tvs_width, tvs_height, world, group=None):
    """All-gather every rank's finished rows (float32 [n_rows * tvs_width]) into
    the full grid (float32 [tvs_height * tvs_width]) on every rank."""
    import torch
    import torch.distributed as dist
    counts = [(e - b) * tvs_width for b, e in (shard_rows(tvs_height, r, world)
                                               for r in range(world))]
    longest = max(counts)
    src = rows if isinstance(rows, torch.Tensor) else torch.as_tensor(np.asarray(rows, np.float32))
    t = torch.zeros(longest, dtype=torch.float32, device=src.device)
    t[:src.numel()] = src.reshape(-1)
    parts = [torch.zeros_like(t) for _ in range(world)]
    dist.all_gather(parts, t, group=group)
    return torch.cat([p[:c] for p, c in zip(parts, counts)]).cpu().numpy()


def max_over_ranks(value, device="cpu", group=None):
    """The largest of every rank's `value` (timings are reported as the max)."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())
