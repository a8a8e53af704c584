"""Work split across ranks (one process per GPU): the neighbour search of one
data set, and the instances of a batch (at the end of this file).

The search is the only stage of a single run that shards: every rank holds the whole data,
computes its shard of the exact kNN (umapb_knn_shard: a balanced range of the
search's tree-ordered query tiles), and one all-gather of the shards' rows
gives every rank the full neighbour lists, from which each rank can continue
with initialize_knn_matrix (the later stages replicate: every SGD step gathers
random embedding rows).  The collectives are torch.distributed's -- NCCL
between GPUs, gloo on CPUs: one all-reduce of a failure flag (a search that
raises on one rank raises on all) and one all_gather of the rows, indices and
distances, padded to the largest shard.
"""
from __future__ import annotations

from typing import Callable, Optional

import numpy as np


def _collective_device(group, device):
    import torch
    import torch.distributed as dist

    if device is not None:
        return device
    return torch.device("cuda", torch.cuda.current_device()) if dist.get_backend(group) == "nccl" \
        else torch.device("cpu")


def agree_on_failure(error: Optional[BaseException], group=None, device=None) -> None:
    """One all-reduce of a failure flag over the ranks of 'group', taken by
    every rank whether or not its own step failed, so that no rank is left
    waiting in a later collective: if any rank failed, every rank raises --
    the failing rank its own error, the others a RuntimeError."""
    import torch
    import torch.distributed as dist

    if dist.get_world_size(group) <= 1:
        if error is not None:
            raise error
        return
    failed = torch.tensor([1 if error is not None else 0], dtype=torch.int32, device=_collective_device(group, device))
    dist.all_reduce(failed, op=dist.ReduceOp.MAX, group=group)
    if int(failed.item()):
        if error is not None:
            raise error
        raise RuntimeError("another rank's step failed")


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
    error = None
    try:
        rows, idx, dst = local(data, k, rank, world)
    except Exception as e:  # reported after every rank has learnt of it
        error = e
    agree_on_failure(error, group, device)
    return gather_shards(rows, idx, dst, data.shape[0], group=group, device=device)


def initialize_sharded(data, num_dim: int, embedding, options=None, group=None, local: Optional[Callable] = None,
                       init: Optional[Callable] = None, device=None):
    """initialize(data, builder, ...) of one data set with the neighbour
    search split over the ranks of 'group': knn_sharded for
    options.num_neighbors neighbours, then, on every rank, the rest of the
    pipeline from the gathered lists by 'init(indices, distances, num_dim,
    embedding, options)' (default: initialize_knn_matrix on the current GPU).
    Every rank returns its own Status over the same graph; the stages after
    the search replicate (each SGD step gathers random embedding rows)."""
    from . import Options
    from . import initialize_knn_matrix

    options = options or Options()
    idx, dst = knn_sharded(data, options.num_neighbors, group=group, local=local, device=device)
    return (init or initialize_knn_matrix)(idx, dst, num_dim, embedding, options)


# ------------------------------------------------- batched instances ---
#
# The batched mode's instances are independent runs, so a batch splits over
# ranks with nothing exchanged while it runs: each rank runs a balanced subset
# of the instances in one batch_run of its own, and an optional all-gather
# afterwards gives every rank every instance's layout.


def partition_instances(sizes, world: int) -> list:
    """Instances of a batch dealt to 'world' ranks: the largest first, each to
    the rank with the fewest observations so far (ties: the lower rank), so
    that the ranks' shares of the observations -- and of the edges the epochs
    process, k per observation -- are balanced.  Returns one ascending int64
    array of instance numbers per rank; the arrays partition range(len(sizes)).
    The same on every rank (no randomness, no communication)."""
    sizes = np.asarray(sizes, dtype=np.int64)
    if world < 1:
        raise ValueError("world must be at least 1")
    if sizes.ndim != 1 or np.any(sizes < 0):
        raise ValueError("sizes must be a 1-d array of non-negative counts")
    load = np.zeros(world, dtype=np.int64)
    owner = np.empty(len(sizes), dtype=np.int64)
    for i in sorted(range(len(sizes)), key=lambda j: (-int(sizes[j]), j)):
        r = int(np.argmin(load))
        owner[i] = r
        load[r] += sizes[i]
    return [np.nonzero(owner == r)[0].astype(np.int64) for r in range(world)]


def _take_rows(a, offs, inst):
    """Rows of instances 'inst' of 'a' (numpy array or torch tensor), concatenated in order."""
    parts = [a[int(offs[i]):int(offs[i + 1])] for i in inst]
    if isinstance(a, np.ndarray):
        return np.ascontiguousarray(np.concatenate(parts) if parts else a[:0])
    import torch

    return torch.cat(parts).contiguous() if parts else a[:0].contiguous()


def batch_sharded(data, sizes, num_dim: int, embedding, options=None, group=None, run: Optional[Callable] = None,
                  gather: bool = True, device=None) -> dict:
    """A batch of independent UMAP runs (batch_run's arguments: instance i is
    the next sizes[i] rows of 'data' and of 'embedding') split over the ranks
    of 'group'.  Every rank holds the whole batch's data; this rank runs the
    instances partition_instances gives it, in one call of
    'run(data, sizes, num_dim, embedding, options)' (default: batch_run on the
    current GPU) over their rows, and writes their layouts into 'embedding'.
    With 'gather', one all-gather of the ranks' layouts (padded to the largest
    share) then fills every instance's rows on every rank; without it only this
    rank's instances are written.  Returns {"instances": this rank's instance
    numbers, "stage_ms": run's result (None for a rank with no instances)}.
    If any rank's run raises, every rank raises (that rank its own error, the
    others a RuntimeError) after one all-reduce of a failure flag, so that no
    rank is left waiting in the gather."""
    import torch
    import torch.distributed as dist

    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    sizes = np.asarray(sizes, dtype=np.int64)
    offs = np.concatenate([[0], np.cumsum(sizes)])
    if int(data.shape[0]) != int(offs[-1]) or int(embedding.shape[0]) != int(offs[-1]):
        raise ValueError("data and embedding must have sum(sizes) rows")
    shares = partition_instances(sizes, world)
    mine = shares[rank]
    if run is None:
        from . import batch_run as run
    stage_ms = None
    local = None
    error = None
    if len(mine):
        try:
            sub_data = _take_rows(data, offs, mine)
            local = _take_rows(embedding, offs, mine)
            stage_ms = run(sub_data, sizes[mine], num_dim, local, options)
            pos = 0
            for i in mine:
                m = int(sizes[i])
                embedding[int(offs[i]):int(offs[i]) + m] = local[pos:pos + m]
                pos += m
        except Exception as e:  # reported after every rank has learnt of it
            error = e
    agree_on_failure(error, group, device)
    if gather and world > 1:
        device = _collective_device(group, device)
        rows = [int(sizes[s].sum()) for s in shares]
        m = max(rows + [1])
        is_np = isinstance(embedding, np.ndarray)
        tdtype = torch.from_numpy(np.zeros(1, dtype=embedding.dtype)).dtype if is_np else embedding.dtype
        buf = torch.zeros((m, num_dim), dtype=tdtype, device=device)
        if local is not None and rows[rank]:
            buf[:rows[rank]] = torch.as_tensor(local, device=device).reshape(rows[rank], num_dim)
        parts = [torch.empty_like(buf) for _ in range(world)]
        dist.all_gather(parts, buf, group=group)
        for r in range(world):
            if r == rank:
                continue
            blk = parts[r].cpu().numpy() if is_np else parts[r].to(embedding.device)
            pos = 0
            for i in shares[r]:
                n_i = int(sizes[i])
                embedding[int(offs[i]):int(offs[i]) + n_i] = blk[pos:pos + n_i]
                pos += n_i
    return {"instances": mine, "stage_ms": stage_ms}
