"""Multi-GPU plumbing for the k-NN path: one process per GPU.

The reference is single-device (code/knncuda.cu:296).  Exact k-NN shards in
two ways, neither needing a collective inside the hot path:

* query sharding (what ``bench.py --gpus N`` does): every rank holds a replica
  of the reference set and answers a contiguous slice of the queries;
  ``shard_range`` assigns the slices and ``gather_query_shards`` reassembles
  the k x Q result on one rank.
* reference sharding: every rank holds a contiguous slice of the reference
  set and returns its local top-k with global indices; one exchange of
  Q*k (distance, index) pairs per rank and ``merge_ref_shards`` give the
  global top-k.  Ordering by (distance, global index) keeps the reference's
  tie rule (equal distances: lower index first, code/knncuda.cu:172, :178),
  so the merged answer equals a single-device run bit for bit.

``compute`` callables take (ref, query, k) numpy arrays (dim x n) and return
(dist, index) k x n arrays -- the CUDA entry points on a GPU rank, or the CPU
oracle in tests.
"""
from __future__ import annotations

import numpy as np


def shard_range(n: int, world: int, rank: int) -> tuple:
    """Contiguous [start, stop) slice of n items for `rank` of `world`."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("bad world/rank")
    return n * rank // world, n * (rank + 1) // world


def merge_ref_shards(parts, k: int):
    """Merge per-reference-shard top-k lists.

    parts: list of (dist, index, offset) with dist/index k_s x Q arrays from a
    shard starting at global reference `offset` (index is shard-local).
    Returns (dist, index) k x Q ordered by (distance, global index)."""
    dists = np.concatenate([p[0] for p in parts], axis=0)
    idxs = np.concatenate([p[1].astype(np.int64) + p[2] for p in parts], axis=0)
    if dists.shape[0] < k:
        raise ValueError("shards hold fewer than k candidates")
    # lexicographic sort per query column: primary distance, secondary index
    order = np.lexsort((idxs, dists), axis=0)
    top = order[:k]
    return (np.take_along_axis(dists, top, axis=0),
            np.take_along_axis(idxs, top, axis=0).astype(np.int32))


def gather_query_shards(local_dist, local_idx, total_q: int, group=None, dst: int = 0):
    """Collect per-rank query-shard results (k x q_r) on rank `dst` as k x total_q
    (torch.distributed; any backend).  Non-destination ranks return None."""
    import torch.distributed as dist

    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    objs = [None] * world if rank == dst else None
    dist.gather_object((np.asarray(local_dist), np.asarray(local_idx)), objs, dst=dst,
                       group=group)
    if rank != dst:
        return None
    d = np.concatenate([o[0] for o in objs], axis=1)
    i = np.concatenate([o[1] for o in objs], axis=1)
    assert d.shape[1] == total_q
    return d, i


def query_sharded_knn(ref, query, k, compute, group=None, dst: int = 0):
    """Every rank answers its slice of the queries; the result lands on `dst`."""
    import torch.distributed as dist

    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    q0, q1 = shard_range(query.shape[1], world, rank)
    d, i = compute(ref, np.ascontiguousarray(query[:, q0:q1]), k)
    return gather_query_shards(d, i, query.shape[1], group, dst)


def ref_sharded_knn(ref, query, k, compute, group=None, dst: int = 0):
    """Every rank searches its slice of the reference set; one gather of the
    per-shard top-k lists and a (distance, global index) merge on `dst`."""
    import torch.distributed as dist

    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    r0, r1 = shard_range(ref.shape[1], world, rank)
    k_local = min(k, r1 - r0)
    d, i = compute(np.ascontiguousarray(ref[:, r0:r1]), query, k_local)
    objs = [None] * world if rank == dst else None
    dist.gather_object((d, i, r0), objs, dst=dst, group=group)
    if rank != dst:
        return None
    return merge_ref_shards(objs, k)
