"""Placing independent scenes on several GPUs (one process per GPU).

Scenes never interact, so the batched and serving workloads shard with no collective on the
data path: each rank simulates its own scenes.  A single scene is not split (that would need
a halo exchange every Jacobi iteration and a distributed BVH); it runs as a replica.
torch.distributed (NCCL on GPUs, gloo in the CPU tests) is used only for barriers and for
reducing timings and statistics.
"""
import heapq

import numpy as np


def partition_scenes(sizes, world):
    """Greedy longest-first bin packing of scene vertex counts onto `world` ranks.
    Deterministic (ties broken by rank, then scene index); returns one sorted index list
    per rank."""
    order = sorted(range(len(sizes)), key=lambda i: (-int(sizes[i]), i))
    heap = [(0, r) for r in range(world)]
    heapq.heapify(heap)
    parts = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        parts[r].append(i)
        heapq.heappush(heap, (load + int(sizes[i]), r))
    return [sorted(p) for p in parts]


def subset_spec(spec, indices):
    yarns, lens, kbend = spec
    return [yarns[i] for i in indices], [lens[i] for i in indices], [kbend[i] for i in indices]


def reduce_timing(ms, vertices, device=None):
    """(max over ranks of ms, sum over ranks of vertices); plain values without a process group."""
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()):
        return float(ms), float(vertices)
    t = torch.tensor([float(ms), float(vertices)], dtype=torch.float64, device=device)
    tmax = t.clone()
    dist.all_reduce(tmax, op=dist.ReduceOp.MAX)
    tsum = t.clone()
    dist.all_reduce(tsum, op=dist.ReduceOp.SUM)
    return float(tmax[0]), float(tsum[1])


def reduce_stats(values, device=None):
    """Sum of FP64 statistics (energies, counts) over ranks."""
    import torch
    import torch.distributed as dist

    v = np.asarray(values, np.float64)
    if not (dist.is_available() and dist.is_initialized()):
        return v
    t = torch.tensor(v, dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return t.cpu().numpy()


def route_requests(request_ids, world, rank):
    """Requests of a serving stream handled by `rank` of `world` GPUs, each running its own
    server: round-robin on the request id (arrival order), so every rank sees the same arrival
    process thinned by `world` and each request goes to exactly one rank."""
    return [i for i in request_ids if i % world == rank]


def gather_to_rank0(obj):
    """Every rank's object, gathered on rank 0 (a list in rank order; None elsewhere); without a
    process group the object alone, as a one-element list."""
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()):
        return [obj]
    out = [None] * dist.get_world_size() if dist.get_rank() == 0 else None
    dist.gather_object(obj, out, dst=0)
    return out
