"""Sharded exact k-NN on the GPU, both shards in one process: an index per
contiguous row range, the batched path on each, the ids made global and the
lists merged (hercules_b200/shard.py) give the single index's answers."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def bits(x):
    return np.asarray(x, np.float32).view(np.uint32)


@pytest.mark.parametrize("world", [2, 3])
def test_sharded_batch_equals_single_index(hg, gpu_available, world):
    import torch
    from hercules_b200.shard import merge_topk, merge_topk_torch, shard_range
    X = hg.generate_walks(1184, 120_000, 256)
    X[100_000] = X[5]  # the same row in two shards
    Q = np.concatenate([hg.generate_queries(14784, X, np.array([0.01, 0.1, 1.0] * 20)), X[5:6]])
    ks = np.array([1, 10, 100, 10] * (len(Q) // 4) + [10] * (len(Q) % 4), np.uint32)
    full = hg.HerculesIndex.build(X, 5_000)
    want_d, want_i = full.knn_batch(Q, ks)
    parts_d, parts_i = [], []
    for r in range(world):
        s, c = shard_range(X.shape[0], world, r)
        ix = hg.HerculesIndex.build(X[s:s + c], 5_000)
        d, i = ix.knn_batch(Q, ks)
        parts_d.append(d)
        parts_i.append(np.where(i >= 0, i + s, -1))
        ix.close()
    d, i = np.concatenate(parts_d, 1), np.concatenate(parts_i, 1)
    md, mi = merge_topk(d, i, int(ks.max()))
    td, ti = merge_topk_torch(torch.from_numpy(d).cuda(), torch.from_numpy(i).cuda(), int(ks.max()))
    for j, k in enumerate(ks):
        assert np.array_equal(bits(md[j, :k]), bits(want_d[j, :k])), j
        assert np.array_equal(mi[j, :k], want_i[j, :k]), j
    assert np.array_equal(bits(td.cpu().numpy()), bits(md)) and np.array_equal(ti.cpu().numpy(), mi)
