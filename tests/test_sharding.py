"""Multi-rank logic on CPU: two gloo ranks partition the batched workload's scenes, reduce
timings, route serving requests and gather their reports the way bench.py does on GPUs (no GPU
involved)."""
import os
import socket

import numpy as np
import torch.multiprocessing as mp

from yarnball_b200 import scenes, sharding


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, sizes, out):
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    parts = sharding.partition_scenes(sizes, world)
    mine = parts[rank]
    verts = int(sum(sizes[i] for i in mine))
    ms, total = sharding.reduce_timing(10.0 + rank, verts)
    stats = sharding.reduce_stats([1.0, float(verts)])
    routed = sharding.route_requests(list(range(101)), world, rank)
    gathered = sharding.gather_to_rank0({"rank": rank, "requests": routed})
    out[rank] = (mine, ms, total, stats.tolist(), routed, gathered)
    dist.barrier()
    dist.destroy_process_group()


def test_partition_is_complete_disjoint_and_balanced():
    yarns, lens, _ = scenes.batched_spec()
    sizes = [int(l.sum()) for l in lens]
    for world in (1, 2, 4, 8):
        parts = sharding.partition_scenes(sizes, world)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(sizes)))
        loads = [sum(sizes[i] for i in p) for p in parts]
        # greedy longest-first: the spread is at most the largest scene
        assert max(loads) - min(loads) <= max(sizes)
    assert sharding.partition_scenes(sizes, 3) == sharding.partition_scenes(sizes, 3)


def test_two_gloo_ranks_agree_on_partition_and_reduce():
    yarns, lens, _ = scenes.batched_spec(num_scenes=40, cap=1_000_000)
    sizes = [int(l.sum()) for l in lens]
    world = 2
    port = _free_port()
    with mp.Manager() as mgr:
        out = mgr.dict()
        mp.spawn(_worker, args=(world, port, sizes, out), nprocs=world, join=True)
        res = dict(out)
    parts = sharding.partition_scenes(sizes, world)
    for r in range(world):
        mine, ms, total, stats, routed, gathered = res[r]
        assert mine == parts[r]
        assert ms == 11.0  # max over ranks
        assert total == float(sum(sizes))
        assert stats[0] == 2.0 and stats[1] == float(sum(sizes))
    assert sorted(res[0][0] + res[1][0]) == list(range(len(sizes)))
    np.testing.assert_equal(len(set(res[0][0]) & set(res[1][0])), 0)
    # serving: each request goes to exactly one rank; rank 0 receives every rank's report
    assert sorted(res[0][4] + res[1][4]) == list(range(101))
    assert abs(len(res[0][4]) - len(res[1][4])) <= 1
    assert [g["rank"] for g in res[0][5]] == [0, 1] and res[0][5][1]["requests"] == res[1][4]
    assert res[1][5] is None


def test_rank_subsets_hold_the_one_gpu_geometry():
    """Each rank of a multi-GPU run builds its scenes of the one batch: their geometry equals
    those scenes' slices of the 1-GPU batch, and the ranks together hold every scene once."""
    spec = scenes.batched_spec(seed=7, num_scenes=30, cap=600_000)
    full = scenes.batched_positions(7, spec)
    sizes = [int(l.sum()) for l in spec[1]]
    parts = sharding.partition_scenes(sizes, 4)
    seen = []
    for p in parts:
        sub = scenes.batched_positions(7, spec, p)
        for i, pos in zip(p, sub):
            assert np.array_equal(pos, full[i])
        seen += p
    assert sorted(seen) == list(range(len(sizes)))
