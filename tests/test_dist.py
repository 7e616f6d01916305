"""Multi-process coordination on CPU: two gloo ranks exercise the replica
collectives (max of the timed region, sums, gathers of per-scene metrics)
and the scene sharding of batches."""
import os
import socket

import pytest

from gpufluid_b200.dist import shard_scenes


def test_shard_scenes_balances_and_covers():
    counts = [500, 100, 400, 300, 300, 200, 100, 50]
    shards = shard_scenes(counts, 3)
    flat = sorted(i for s in shards for i in s)
    assert flat == list(range(len(counts)))
    loads = [sum(counts[i] for i in s) for s in shards]
    assert max(loads) - min(loads) <= max(counts)
    assert all(s == sorted(s) for s in shards)
    assert shard_scenes(counts, 1) == [list(range(len(counts)))]
    assert shard_scenes([], 2) == [[], []]
    with pytest.raises(ValueError):
        shard_scenes(counts, 0)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    os.environ.update({"RANK": str(rank), "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    from gpufluid_b200.dist import Ranks
    r = Ranks(backend="gloo", timeout_s=60)
    r.barrier()
    res = {
        "max": r.max(10.0 + rank),
        "sum": r.sum(1.0 + rank),
        "gather": r.gather([rank, 2.0 * rank]),
        "shard": shard_scenes([5, 4, 3, 3, 1], r.world)[r.rank],
    }
    r.close()
    out.put((rank, res))


def test_two_gloo_ranks():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    results = dict(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank in (0, 1):
        assert results[rank]["max"] == 11.0
        assert results[rank]["sum"] == 3.0
        assert results[rank]["gather"] == [[0.0, 0.0], [1.0, 2.0]]
    assert sorted(results[0]["shard"] + results[1]["shard"]) == [0, 1, 2, 3, 4]
