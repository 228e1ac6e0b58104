"""searchPoints2 (vann_search_staged): graph results merged with the insert list under
the reference's replace-the-farthest rule, bit for bit against the oracle; patchGraph
(vann_patch_graph) moves the list into the graph."""
import numpy as np
import pytest

from vann import workload

pytestmark = pytest.mark.gpu


def _graph(oracle, vann_mod, n=3000, seed=71, integer=True):
    import torch

    kw = {} if integer else {"sigma": 0.05, "integer": False, "unit_norm": True}
    base = workload.mixture(n, 128, 30, seed=seed, **kw)
    og, entry = oracle.build_index(base, R=32, L=64, alpha=1.2, seed=seed, skip_mode=2,
                                   bloom_mode=oracle.BLOOM_SNAPSHOT)
    idx = vann_mod.Index(128, 32, 64, 1.2, capacity=n + 2000)
    idx.set_graph(base, og.deg, og.adj, entry, consistent=True)
    return base, og, entry, idx, torch


@pytest.mark.parametrize("L", [16, 75])
def test_search_staged_matches_oracle(oracle, vann_mod, L):
    base, og, entry, idx, torch = _graph(oracle, vann_mod)
    il = workload.mixture(500, 128, 30, seed=72)
    q = workload.mixture(150, 128, 30, seed=73)
    idx.stage_insert(torch.from_numpy(il[:200]).cuda())
    idx.stage_insert(torch.from_numpy(il[200:]).cuda())  # grows the list, keeps the rows
    assert idx.info()["staged"] == 500
    ids, d, rows = idx.search_staged(torch.from_numpy(q).cuda(), L=L, with_vecs=True)
    ids = ids.cpu().numpy().view(np.uint32)
    d = d.cpu().numpy()
    # oracle: GreedySearch worklist (all L entries, in order), then the merge
    st, wids, _, _, _ = og.search(q, L, L, entry, bloom_mode=oracle.BLOOM_SNAPSHOT)
    assert st == 0
    oids, od = oracle.merge_rerank(base, q, wids, il)
    assert np.array_equal(ids, oids)
    assert np.array_equal(d, od)
    assert (ids >= oracle.STAGED).any()  # staged rows made it into results
    # the rows returned are the rows named
    rows = rows.cpu().numpy()
    for qi in range(0, 150, 7):
        for t in range(L):
            i = ids[qi, t]
            want = il[i & 0x7FFFFFFF] if i & oracle.STAGED else base[i]
            assert np.array_equal(rows[qi, t], want)


def test_float_rows_merge_bit_exact(oracle, vann_mod):
    """Distances are sequential fused multiply-adds as in l2_distance_sq, so float
    rows merge bit for bit too (given the same graph worklist)."""
    base, og, entry, idx, torch = _graph(oracle, vann_mod, integer=False)
    il = workload.mixture(300, 128, 30, seed=74, sigma=0.05, integer=False, unit_norm=True)
    q = workload.mixture(100, 128, 30, seed=75, sigma=0.05, integer=False, unit_norm=True)
    idx.stage_insert(torch.from_numpy(il).cuda())
    qd = torch.from_numpy(q).cuda()
    ids, d = idx.search_staged(qd, L=32)
    wids, _ = idx.search(qd, k=32, L=32)
    oids, od = oracle.merge_rerank(base, q, wids.cpu().numpy().view(np.uint32), il)
    assert np.array_equal(ids.cpu().numpy().view(np.uint32), oids)
    assert np.array_equal(d.cpu().numpy(), od)


def test_patch_graph_moves_the_list_into_the_graph(oracle, vann_mod):
    base, og, entry, idx, torch = _graph(oracle, vann_mod, seed=76)
    il = workload.mixture(400, 128, 30, seed=77)
    idx.stage_insert(torch.from_numpy(il).cuda())
    new = idx.patch_graph().cpu().numpy()
    assert new.tolist() == list(range(3000, 3400))
    assert idx.info()["staged"] == 0 and idx.info()["size"] == 3400
    # an empty list merges nothing: search_staged equals the plain worklist search
    q = torch.from_numpy(il[:50]).cuda()
    ids, _ = idx.search_staged(q, L=32)
    assert (ids.cpu().numpy().view(np.uint32) < oracle.STAGED).all()
    got = ids.cpu().numpy().view(np.uint32)[:, 0]
    assert (got == new[:50]).mean() >= 0.95  # each inserted row finds itself


def test_vamana_mirror_search_points2(vann_mod):
    import torch

    base = workload.mixture(2000, 128, 20, seed=78)
    v = vann_mod.Vamana(torch.from_numpy(base).cuda(), R=32, L=40, alpha=1.2)
    extra = workload.mixture(100, 128, 20, seed=79)
    v.insertPoints(torch.from_numpy(extra).cuda())
    rows = v.searchPoints2(torch.from_numpy(extra[:10]).cuda()).cpu().numpy()
    assert rows.shape == (10, 40, 128)
    for i in range(10):  # each staged row is its own nearest neighbour
        assert np.array_equal(rows[i, 0], extra[i])
    v.patchGraph()
    assert v.index.info()["staged"] == 0 and v.index.info()["size"] == 2100
