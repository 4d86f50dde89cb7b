"""Sharded exact k-NN over several GPUs: every rank holds a contiguous range
of the collection's rows as its own index, answers every query of a batch on
it, and one all-gather of the k (distance, id) pairs per query (NCCL between
GPUs, gloo on the host) is followed by a deterministic merge.

Exact k-NN is partition-invariant: the k nearest rows of the whole collection
are the k nearest of the union of every shard's k nearest.  The merge keeps
the reference's rule for the answer list (queue_bounded_sorted_insert,
hercules_query_engine.c:4034-4082: k distinct distances) with this library's
tie rule (the lowest dataset id for a distance), so a sharded answer equals
the single-index answer bit for bit.
"""
import numpy as np


def shard_range(n, world, rank):
    """Rows [start, start + count) of rank's shard: contiguous, sizes differing
    by at most one."""
    if world <= 0 or not 0 <= rank < world:
        raise ValueError("rank %d outside a world of %d" % (rank, world))
    base, extra = divmod(int(n), int(world))
    start = rank * base + min(rank, extra)
    return start, base + (1 if rank < extra else 0)


def merge_topk(dist, ids, k):
    """Merge candidate lists into the k smallest distinct distances, lowest id
    per distance.  dist, ids: [nq, m] (float32, int64; empty slots +inf / -1),
    m the concatenated lists of every shard.  Returns ([nq, k], [nq, k])."""
    dist = np.asarray(dist, np.float32)
    ids = np.asarray(ids, np.int64)
    nq, m = dist.shape
    out_d = np.full((nq, k), np.inf, np.float32)
    out_i = np.full((nq, k), -1, np.int64)
    for j in range(nq):
        d, i = dist[j], ids[j]
        ok = i >= 0
        d, i = d[ok], i[ok]
        order = np.lexsort((i, d))  # by distance, then id
        d, i = d[order], i[order]
        if d.size:
            first = np.ones(d.size, bool)
            first[1:] = d[1:] != d[:-1]  # one entry per distance: its lowest id
            d, i = d[first], i[first]
        c = min(k, d.size)
        out_d[j, :c] = d[:c]
        out_i[j, :c] = i[:c]
    return out_d, out_i


def merge_topk_torch(dist, ids, k):
    """merge_topk on device tensors (one sort per query row, no host copy)."""
    import torch
    inf = torch.tensor(float("inf"), dtype=dist.dtype, device=dist.device)
    d = torch.where(ids >= 0, dist, inf)
    # sort by id, then stably by distance: (distance, id) order
    oi = torch.argsort(ids, dim=1, stable=True)
    d, i = torch.gather(d, 1, oi), torch.gather(ids, 1, oi)
    od = torch.argsort(d, dim=1, stable=True)
    d, i = torch.gather(d, 1, od), torch.gather(i, 1, od)
    dup = torch.zeros_like(d, dtype=torch.bool)
    dup[:, 1:] = d[:, 1:] == d[:, :-1]
    d = torch.where(dup, inf, d)
    i = torch.where(dup, torch.full_like(i, -1), i)
    od = torch.argsort(d, dim=1, stable=True)[:, :k]
    d, i = torch.gather(d, 1, od), torch.gather(i, 1, od)
    i = torch.where(torch.isinf(d), torch.full_like(i, -1), i)
    return d, i


def allgather_knn(dist, ids, k, group=None):
    """All-gather every rank's [nq, kmax] answers (device or host tensors,
    the ids already global) and merge them into the k nearest of the whole
    collection, on every rank."""
    import torch
    import torch.distributed as dist_
    world = dist_.get_world_size(group)
    dl = [torch.empty_like(dist) for _ in range(world)]
    il = [torch.empty_like(ids) for _ in range(world)]
    dist_.all_gather(dl, dist.contiguous(), group=group)
    dist_.all_gather(il, ids.contiguous(), group=group)
    return merge_topk_torch(torch.cat(dl, 1), torch.cat(il, 1), k)


def sharded_batch_answers(dist, ids, first, ks, kmax, group=None):
    """One batch answered on a row-range shard -> the answers of the whole
    collection, on every rank.  dist, ids: this shard's [nq, kmax] answers
    with ids local to the shard (row i of the shard is global row first + i;
    -1 marks an empty entry); ks: each query's k.  The ids are made global,
    every rank's lists are all-gathered and merged, and each query's entries
    past its own k are cleared (+inf / -1), as a single index returns them."""
    import torch
    gi = torch.where(ids >= 0, ids + int(first), torch.full_like(ids, -1))
    md, mi = allgather_knn(dist, gi, kmax, group=group)
    kq = torch.as_tensor(np.asarray(ks, np.int64), device=dist.device)
    beyond = torch.arange(kmax, device=dist.device)[None, :] >= kq[:, None]
    return md.masked_fill(beyond, float("inf")), mi.masked_fill(beyond, -1)
