"""Texel sharding across ranks (tempestrenderer_b200.shards): the partition, and
the collective host logic on world_size-2 gloo process groups on CPU, with
failures made on the host (a rank whose fitter raises, a rank that leaves before
the collective)."""
import datetime
import multiprocessing as mp
import os
import socket
import traceback

import numpy as np
import pytest

from tempestrenderer_b200 import shards


def test_shard_range_covers_exactly():
    for total in (0, 1, 7, 160000, 160001):
        for world in (1, 2, 3, 8):
            ranges = [shards.shard_range(total, r, world) for r in range(world)]
            assert ranges[0][0] == 0
            for (f0, c0), (f1, _) in zip(ranges, ranges[1:]):
                assert f0 + c0 == f1
            assert sum(c for _, c in ranges) == total
            assert max(c for _, c in ranges) - min(c for _, c in ranges) <= 1


def test_shard_range_rejects_bad_requests():
    with pytest.raises(ValueError):
        shards.shard_range(10, 2, 2)
    with pytest.raises(ValueError):
        shards.shard_range(10, 0, 0)


def test_weighted_shards_balance_cost():
    # a batch of BTFs: 4096 texels at 81 directions then 4096 at 151 directions
    costs = np.r_[np.full(4096, 81 ** 2), np.full(4096, 151 ** 2)]
    for world in (1, 2, 4, 8):
        parts = shards.weighted_shards(costs, world)
        assert parts[0][0] == 0 and sum(c for _, c in parts) == costs.size
        for (f0, c0), (f1, _) in zip(parts, parts[1:]):
            assert f0 + c0 == f1
        loads = np.array([costs[f:f + c].sum() for f, c in parts], np.float64)
        assert np.all(np.abs(loads - costs.sum() / world) <= costs.max())
    assert shards.weighted_shards([], 3) == [(0, 0)] * 3


def test_single_process_fallbacks():
    with pytest.raises(shards.ShardError):
        shards.check_all_ranks(False, "x")
    assert shards.max_over_ranks(2.5) == 2.5


def _fake_maps(first, count):
    """Deterministic per-texel maps standing in for a GPU fit of texels
    [first, first + count)."""
    import torch

    t = torch.arange(first, first + count, dtype=torch.float32)
    return {"rmse": t * 0.5, "sigma": torch.stack([t, -t], dim=1), "params": t[:, None].repeat(1, 7) + 0.25}


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, case, q):
    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    try:
        dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=10))
        if case == "gather":
            maps, rng = shards.fit_sharded(_fake_maps, 7)
            full = _fake_maps(0, 7)
            ok = all(np.array_equal(maps[k].numpy(), full[k].numpy()) for k in full)
            q.put((rank, "ok" if ok else "mismatch", rng))
        elif case == "raise":
            def fit(first, count):
                if rank == 1:
                    raise RuntimeError("slab did not arrive")
                return _fake_maps(first, count)

            try:
                shards.fit_sharded(fit, 9)
                q.put((rank, "no error", None))
            except shards.ShardError as e:
                q.put((rank, "shard error", (e.failed_ranks, str(e))))
        elif case == "max":
            q.put((rank, "max", shards.max_over_ranks(1.0 + 3.0 * rank)))
        elif case == "leave":
            if rank == 1:
                # leaves between steps, with no collective in flight
                q.put((rank, "left", None))
                q.close()
                q.join_thread()   # the message is flushed before the process ends
                os._exit(0)
            try:
                shards.check_all_ranks(True)
                q.put((rank, "no error", None))
            except Exception as e:  # the peer's departure ends the collective with an error
                q.put((rank, "error", type(e).__name__))
        dist.destroy_process_group()
    except Exception:
        q.put((rank, "crash", traceback.format_exc()))


def _run(case, world=2, timeout=90):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, case, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = {}
    try:
        for _ in range(world):
            rank, status, info = q.get(timeout=timeout)
            out[rank] = (status, info)
    finally:
        for p in procs:
            p.join(timeout=30)
            if p.is_alive():
                p.kill()
    return out


def test_gloo_gather_matches_single_process():
    out = _run("gather")
    assert out[0][0] == "ok" and out[1][0] == "ok", out
    assert out[0][1] == (0, 4) and out[1][1] == (4, 3)


def test_gloo_failure_on_one_rank_raises_everywhere():
    out = _run("raise")
    for r in (0, 1):
        status, info = out[r]
        assert status == "shard error", out
        assert info[0] == [1]
    assert "slab did not arrive" in out[1][1][1]


def test_gloo_max_over_ranks():
    out = _run("max")
    assert out[0] == ("max", 4.0) and out[1] == ("max", 4.0)


def test_gloo_rank_that_leaves_ends_the_collective_with_an_error():
    out = _run("leave")
    assert out[1][0] == "left"
    assert out[0][0] == "error", out
