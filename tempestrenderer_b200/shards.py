"""Texel sharding across GPUs: one process per GPU, contiguous texel ranges.

The svbrdffit texel loop (PusherThread::execute, tools/svbrdf-fitting/
svbrdf-fitting.cc:86-121) hands texels of one W x H region to worker threads
through an atomic counter; every texel is fitted independently.  Across GPUs the
same independence means no data-path collective: each rank fits a contiguous
range of texels in its own HBM.  torch.distributed (NCCL between GPUs, gloo on
CPU) is used only for

  * agreeing that every rank's shard succeeded (check_all_ranks), so that all
    ranks take the same collective steps and a failure on one rank surfaces as
    a ShardError on every rank instead of a hang,
  * the max-over-ranks device time of a timed region (max_over_ranks),
  * the optional all-gather of the output maps (gather_maps; 48-64 bytes per
    texel).

The fitter itself is a callable, so the host logic runs on CPU ranks in the
tests; on GPUs it is Context.fit_texels on the rank's range.
"""
from __future__ import annotations

from typing import Callable, Mapping, Sequence

import numpy as np


class ShardError(RuntimeError):
    """A shard failed on at least one rank; raised on every rank."""

    def __init__(self, failed_ranks: Sequence[int], message: str):
        super().__init__(message)
        self.failed_ranks = list(failed_ranks)


def shard_range(total: int, rank: int, world: int) -> tuple[int, int]:
    """Contiguous range (first, count) of `total` texels for `rank` of `world`;
    the first total % world ranks get one texel more."""
    if world < 1 or not 0 <= rank < world or total < 0:
        raise ValueError(f"bad shard request: total={total} rank={rank} world={world}")
    base, extra = divmod(total, world)
    first = rank * base + min(rank, extra)
    return first, base + (1 if rank < extra else 0)


def weighted_shards(costs: Sequence[float], world: int) -> list[tuple[int, int]]:
    """Contiguous ranges over items with per-item costs (e.g. texels x pairs of a
    batch of BTFs with different direction layouts), cut at the item boundary
    nearest to k/world of the total cost, so that every rank's cost is within one
    item's cost of the even share.  Returns (first, count) per rank."""
    if world < 1:
        raise ValueError("world must be >= 1")
    c = np.asarray(costs, np.float64)
    if c.ndim != 1 or np.any(c < 0):
        raise ValueError("costs must be a 1-D array of non-negative numbers")
    n = c.shape[0]
    total = float(c.sum())
    if n == 0 or total == 0.0:
        return [shard_range(n, r, world) for r in range(world)]
    prefix = np.concatenate([[0.0], np.cumsum(c)])
    cuts = [0]
    for k in range(1, world):
        target = total * k / world
        i = int(np.searchsorted(prefix, target, side="left"))   # first prefix >= target
        if i > 0 and (i > n or target - prefix[i - 1] <= prefix[i] - target):
            i -= 1
        cuts.append(max(cuts[-1], min(i, n)))
    cuts.append(n)
    cuts = [min(x, n) for x in cuts]
    return [(cuts[r], cuts[r + 1] - cuts[r]) for r in range(world)]


def _dist():
    import torch.distributed as dist

    return dist if dist.is_available() and dist.is_initialized() else None


def _flag_device(group=None):
    """Device of the tensors handed to collectives: CUDA for NCCL groups."""
    import torch

    dist = _dist()
    if dist is not None and dist.get_backend(group) == "nccl":
        return torch.device("cuda", torch.cuda.current_device())
    return torch.device("cpu")


def check_all_ranks(ok: bool, message: str = "", group=None) -> None:
    """Collective: every rank reports whether its shard succeeded; if any failed,
    every rank raises ShardError naming the failed ranks.  Without an initialised
    process group it raises locally when ok is False."""
    import torch

    dist = _dist()
    if dist is None:
        if not ok:
            raise ShardError([0], message or "shard failed")
        return
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    flags = torch.zeros(world, dtype=torch.int32, device=_flag_device(group))
    flags[rank] = 0 if ok else 1
    dist.all_reduce(flags, op=dist.ReduceOp.SUM, group=group)
    failed = [r for r in range(world) if int(flags[r].item()) != 0]
    if failed:
        detail = f"; this rank: {message}" if not ok and message else ""
        raise ShardError(failed, f"texel shards failed on ranks {failed}{detail}")


def max_over_ranks(value: float, group=None) -> float:
    """Collective: the maximum of a per-rank number (device time of a timed region)."""
    import torch

    dist = _dist()
    if dist is None:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=_flag_device(group))
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())


def gather_maps(local: Mapping[str, "torch.Tensor"], counts: Sequence[int], group=None) -> dict:
    """Collective: all-gathers per-rank map arrays ([count_r][...] each, in rank
    order of contiguous ranges) into full arrays on every rank.  Shards of
    unequal size are padded to the largest for the exchange."""
    import torch

    dist = _dist()
    if dist is None:
        return {k: v for k, v in local.items()}
    world = dist.get_world_size(group)
    if len(counts) != world:
        raise ValueError("one count per rank")
    rank = dist.get_rank(group)
    width = max(counts) if counts else 0
    dev = _flag_device(group)
    out = {}
    for key in sorted(local):   # same order on every rank
        v = local[key]
        if v.shape[0] != counts[rank]:
            raise ValueError(f"map {key}: {v.shape[0]} rows, expected {counts[rank]}")
        padded = torch.zeros((width, *v.shape[1:]), dtype=v.dtype, device=dev)
        padded[: v.shape[0]] = v.to(dev)
        parts = [torch.empty_like(padded) for _ in range(world)]
        dist.all_gather(parts, padded, group=group)
        out[key] = torch.cat([parts[r][: counts[r]] for r in range(world)], dim=0)
    return out


def fit_sharded(fit_fn: Callable[[int, int], Mapping[str, "torch.Tensor"]], total: int, group=None,
                gather: bool = True):
    """Fits this rank's contiguous range of `total` texels with fit_fn(first,
    count) -> {map name: tensor [count][...]} and, with gather, returns the full
    maps on every rank (else this rank's maps).  A fit_fn that raises on any rank
    becomes a ShardError on every rank, after the same collective steps."""
    dist = _dist()
    world = dist.get_world_size(group) if dist else 1
    rank = dist.get_rank(group) if dist else 0
    first, count = shard_range(total, rank, world)
    maps, err = None, ""
    try:
        maps = fit_fn(first, count)
    except Exception as e:   # reported to every rank by check_all_ranks
        err = f"{type(e).__name__}: {e}"
    check_all_ranks(maps is not None, err, group=group)
    if not gather:
        return maps, (first, count)
    counts = [shard_range(total, r, world)[1] for r in range(world)]
    return gather_maps(maps, counts, group=group), (first, count)
