"""The neighbour search split across ranks (one process per GPU).

The only stage of the pipeline that shards: every rank holds the whole data,
computes its shard of the exact kNN (umapb_knn_shard: a balanced range of the
search's tree-ordered query tiles), and one all-gather of the shards' rows
gives every rank the full neighbour lists, from which each rank can continue
with initialize_knn_matrix (the later stages replicate: every SGD step gathers
random embedding rows).  The collective is torch.distributed's all_gather --
NCCL between GPUs, gloo on CPUs -- over tensors padded to the largest shard.
"""
from __future__ import annotations

from typing import Callable, Optional

import numpy as np


def gather_shards(rows: np.ndarray, indices: np.ndarray, distances: np.ndarray, num_obs: int, group=None,
                  device=None):
    """All-gather every rank's (rows, indices, distances) block and assemble
    the (num_obs, k) lists on every rank.  Raises if the ranks' rows do not
    partition range(num_obs)."""
    import torch
    import torch.distributed as dist

    world = dist.get_world_size(group)
    if device is None:
        device = torch.device("cuda", torch.cuda.current_device()) if dist.get_backend(group) == "nccl" \
            else torch.device("cpu")
    k = indices.shape[1]
    count = torch.tensor([len(rows)], dtype=torch.int64, device=device)
    counts = [torch.zeros_like(count) for _ in range(world)]
    dist.all_gather(counts, count, group=group)
    counts = [int(c.item()) for c in counts]
    m = max(counts + [1])

    def padded(a, shape, dtype):
        t = torch.zeros(shape, dtype=dtype, device=device)
        if len(a):
            t[:len(a)] = torch.as_tensor(np.ascontiguousarray(a), device=device)
        return t

    blocks = []
    for a, shape, dtype in ((rows, (m,), torch.int32), (indices, (m, k), torch.int32),
                            (distances, (m, k), torch.float64 if distances.dtype == np.float64 else torch.float32)):
        mine = padded(a, shape, dtype)
        parts = [torch.empty_like(mine) for _ in range(world)]
        dist.all_gather(parts, mine, group=group)
        blocks.append([p.cpu().numpy() for p in parts])
    out_idx = np.full((num_obs, k), -1, dtype=np.int32)
    out_dist = np.zeros((num_obs, k), dtype=distances.dtype)
    seen = np.zeros(num_obs, dtype=np.int64)
    for r in range(world):
        c = counts[r]
        rr = blocks[0][r][:c].astype(np.int64)
        out_idx[rr] = blocks[1][r][:c]
        out_dist[rr] = blocks[2][r][:c]
        np.add.at(seen, rr, 1)
    if not np.all(seen == 1):
        raise RuntimeError("the ranks' shards do not partition the observations")
    return out_idx, out_dist


def knn_sharded(data: np.ndarray, k: int, group=None, local: Optional[Callable] = None, device=None):
    """Exact kNN of 'data' split over the ranks of 'group': this rank's shard by
    'local(data, k, rank, world)' (default: umappp_b200.knn_shard on the current
    GPU), then gather_shards.  Returns (indices, distances) of shape (n, k) on
    every rank."""
    import torch.distributed as dist

    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    if local is None:
        from . import knn_shard as local_shard

        def local(x, kk, r, w):
            return local_shard(x, kk, r, w)
    rows, idx, dst = local(data, k, rank, world)
    return gather_shards(rows, idx, dst, data.shape[0], group=group, device=device)
