"""The CPU-runnable configuration exactly as stated: 10,000 x 128 integer-valued
rows (100-cluster clipped Gaussian mixture, seeds 1 / 2), 100 queries, build
R=32, L=75, alpha=1.2 from the medoid, search k=10, L=75.

The GPU build (one batch over the seeded random start graph, as runVamana,
vamana/include/vamana_impl.cuh:289-360) must equal the oracle's row for row, on
the CUDA-core prune and on the tensor-core prune; the search must equal the
oracle's GreedySearch (vamana/include/search.cuh:226-367) in ids, distances, hop
and distance-evaluation counts; recall@10 is measured against FP64 brute force.
"""
import numpy as np
import pytest

from vann import workload

pytestmark = pytest.mark.gpu

N, DIM, R, L, ALPHA, K, SEED = 10_000, 128, 32, 75, 1.2, 10, 11


@pytest.fixture(scope="module")
def c1(oracle):
    base, q = workload.config1()
    g, entry = oracle.build_index(base, R=R, L=L, alpha=ALPHA, seed=SEED, skip_mode=2,
                                  bloom_mode=oracle.BLOOM_SNAPSHOT)
    return base, q, g, entry


@pytest.mark.parametrize("stores", [("f32",), ("f32", "u8")], ids=["cuda_cores", "tensor_cores"])
def test_c1_build_and_search_bit_exact(oracle, vann_mod, c1, stores):
    import torch

    base, q, g, entry = c1
    assert entry == oracle.medoid(base)
    idx = vann_mod.Index(DIM, R, L, ALPHA, capacity=N, stores=stores)
    idx.build(torch.from_numpy(base).cuda(), batch=0, seed=SEED)
    assert idx.info()["entry"] == entry
    _, deg, adj = idx.get_graph()
    diff = [i for i in range(N) if not np.array_equal(adj[i, :deg[i]], g.adj[i, :g.deg[i]])]
    assert diff == []
    if "u8" in stores:
        assert idx.info()["pruned_tc"] > 0

    st, oids, od, oh, oe = g.search(q, L, K, entry, bloom_mode=oracle.BLOOM_SNAPSHOT)
    assert st == 0
    for store in stores:
        ids, d, stats = idx.search_stats(torch.from_numpy(q).cuda(), k=K, L=L, store=store)
        idx.sync()
        assert np.array_equal(ids.cpu().numpy().view(np.uint32), oids), store
        assert np.array_equal(d.cpu().numpy(), od), store
        s = stats.cpu().numpy()
        assert np.array_equal(s[0], oh) and np.array_equal(s[1], oe), store

    truth, _ = oracle.bruteforce_knn(base, q, K)
    rec = oracle.recall_at_k(oids, truth, K)
    assert rec >= 0.95, rec
