"""Edge cases of the C ABI on the GPU path: empty calls, a one-node index, capacity
exhaustion that leaves the index usable, and invalid search parameters."""
import numpy as np
import pytest

from vann import workload

pytestmark = pytest.mark.gpu


def _index(vann_mod, n=1500, capacity=None, stores=("f32", "u8")):
    import torch

    base = workload.mixture(n, 128, 15, seed=101)
    idx = vann_mod.Index(128, 32, 48, 1.2, capacity=capacity or n, stores=stores)
    idx.build(torch.from_numpy(base).cuda(), batch=0, seed=2)
    return idx, base


def test_empty_calls_are_no_ops(vann_mod):
    import torch

    idx, base = _index(vann_mod)
    before = idx.get_graph()
    empty_q = torch.empty((0, 128), dtype=torch.float32, device="cuda")
    ids, d = idx.search(empty_q, k=10, L=32)
    assert ids.shape == (0, 10)
    ids, d = idx.search_staged(empty_q, L=32)
    assert ids.shape == (0, 32)
    assert idx.insert(empty_q).numel() == 0
    idx.delete(torch.empty(0, dtype=torch.int32, device="cuda"))
    idx.stage_insert(empty_q)
    idx.consolidate()  # nothing deleted
    idx.sync()
    after = idx.get_graph()
    assert all(np.array_equal(x, y) for x, y in zip(before, after))
    assert idx.info()["free_ids"] == 0 and idx.info()["staged"] == 0


def test_one_node_index(vann_mod):
    import torch

    row = workload.mixture(1, 128, 1, seed=102)
    idx = vann_mod.Index(128, 32, 16, 1.2, capacity=4, stores=("f32", "u8"))
    idx.build(torch.from_numpy(row).cuda(), batch=0, seed=1)
    assert idx.info()["entry"] == 0
    q = torch.from_numpy(workload.mixture(3, 128, 1, seed=103)).cuda()
    ids, d = idx.search(q, k=4, L=8)
    ids, d = ids.cpu().numpy().view(np.uint32), d.cpu().numpy()
    for row, dist in zip(ids, d):  # the node, possibly again as its own neighbour, then padding
        valid = row != 0xFFFFFFFF
        assert valid[0] and (row[valid] == 0).all() and np.isinf(dist[~valid]).all()
    new = idx.insert(torch.from_numpy(workload.mixture(3, 128, 1, seed=104)).cuda()).cpu().tolist()
    assert new == [1, 2, 3]


def test_capacity_exhausted_leaves_the_index_usable(vann_mod):
    import torch

    idx, base = _index(vann_mod, n=1000, capacity=1050)
    extra = torch.from_numpy(workload.mixture(100, 128, 15, seed=105)).cuda()
    with pytest.raises(vann_mod.VannError) as e:
        idx.insert(extra)  # 100 > 50 free slots
    assert e.value.status == vann_mod.ERR_CAPACITY
    assert idx.info()["size"] == 1000
    assert idx.insert(extra[:50]).cpu().tolist() == list(range(1000, 1050))
    ids, _ = idx.search(extra[:20], k=1, L=48)
    assert (ids.cpu().numpy()[:, 0] == np.arange(1000, 1020)).mean() >= 0.95


def test_invalid_search_parameters(vann_mod):
    import torch

    idx, base = _index(vann_mod)
    q = torch.from_numpy(base[:4]).cuda()
    for k, L in ((0, 8), (16, 8), (10, 2000)):
        with pytest.raises(vann_mod.VannError) as e:
            idx.search(q, k=k, L=L)
        assert e.value.status == vann_mod.ERR_INVALID
    with pytest.raises(vann_mod.VannError) as e:
        idx.search(q, k=10, L=32, store="bf16")  # copy not enabled at create
    assert e.value.status == vann_mod.ERR_UNSUPPORTED
    ids, _ = idx.search(q, k=1, L=64)  # the index still answers
    assert (ids.cpu().numpy()[:, 0] == np.arange(4)).mean() >= 0.75
