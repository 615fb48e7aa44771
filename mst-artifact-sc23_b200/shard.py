"""Batched mode across GPUs: one process per GPU, graphs sharded by size.

A batch's graphs are independent, so several GPUs share a batch with no
data-path collective: every rank computes the same partition from the same
per-graph costs (directed CSR entries), solves its own graphs, and the
per-graph results (forest weight and size) are gathered once at the end.
"""
import heapq


def partition_by_cost(costs, world):
    """Greedy longest-processing-time partition of graph ids over `world`
    ranks: graphs in decreasing cost (ties by id) each go to the least-loaded
    rank (ties by rank). Deterministic, so every rank computes the same answer.
    Returns one sorted id list per rank."""
    if world < 1:
        raise ValueError("world must be >= 1")
    heap = [(0, r) for r in range(world)]
    shards = [[] for _ in range(world)]
    for gid in sorted(range(len(costs)), key=lambda i: (-int(costs[i]), i)):
        load, r = heapq.heappop(heap)
        shards[r].append(gid)
        heapq.heappush(heap, (load + int(costs[gid]), r))
    return [sorted(s) for s in shards]


def gather_results(local, dist=None):
    """Union of every rank's {graph id: result} (all_gather_object over the
    default process group); `local` alone when not distributed."""
    if dist is None or not dist.is_available() or not dist.is_initialized():
        return dict(local)
    parts = [None] * dist.get_world_size()
    dist.all_gather_object(parts, local)
    merged = {}
    for p in parts:
        for k, v in p.items():
            if k in merged:
                raise ValueError(f"graph {k} solved by two ranks")
            merged[k] = v
    return merged
