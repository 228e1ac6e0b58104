"""GPU build / insert / delete / consolidate vs the CPU oracle."""
import numpy as np
import pytest

from vann import workload

pytestmark = pytest.mark.gpu


def _rows_equal(deg_a, adj_a, deg_b, adj_b):
    return [i for i in range(len(deg_a)) if not np.array_equal(adj_a[i, :deg_a[i]], adj_b[i, :deg_b[i]])]


@pytest.mark.parametrize("R,L,quirk", [(32, 75, 1), (64, 64, 0)])
def test_one_batch_build_bit_exact(oracle, vann_mod, R, L, quirk):
    import torch

    base = workload.mixture(3000, 128, 30, seed=31)
    og, entry = oracle.build_index(base, R=R, L=L, alpha=1.2, seed=7, skip_mode=1 if quirk else 2,
                                   bloom_mode=oracle.BLOOM_SNAPSHOT)
    idx = vann_mod.Index(128, R, L, 1.2, capacity=3000, quirks=quirk)
    idx.build(torch.from_numpy(base).cuda(), batch=0, seed=7)
    assert idx.info()["entry"] == entry
    _, deg, adj = idx.get_graph()
    assert _rows_equal(deg, adj, og.deg, og.adj) == []


def test_batched_build_bit_exact(oracle, vann_mod):
    import torch

    n, B, R, L = 4000, 1000, 32, 64
    base = workload.mixture(n, 128, 30, seed=32)
    deg0, adj0 = oracle.random_graph(B, R, 11)
    deg = np.zeros(n, np.uint32)
    adj = np.zeros((n, R), np.uint32)
    deg[:B], adj[:B] = deg0, adj0
    og = oracle.Graph(base, deg, adj)
    entry = oracle.medoid(base[:B])
    assert og.vamana_batch(0, B, L, 1.2, entry, skip_mode=2) == 0
    for s in range(B, n, B):
        assert og.vamana_batch(s, B, L, 1.2, entry, skip_mode=0) == 0
    idx = vann_mod.Index(128, R, L, 1.2, capacity=n)
    idx.build(torch.from_numpy(base).cuda(), batch=B, seed=11)
    _, gdeg, gadj = idx.get_graph()
    assert _rows_equal(gdeg, gadj, og.deg, og.adj) == []


def test_insert_matches_reference_patch(oracle, vann_mod):
    import torch

    n0, n1, R, L = 3000, 700, 32, 64
    base = workload.mixture(n0 + n1, 128, 30, seed=33)
    og, entry = oracle.build_index(base[:n0], R=R, L=L, alpha=1.2, seed=5, skip_mode=2)
    idx = vann_mod.Index(128, R, L, 1.2, capacity=n0 + n1)
    idx.build(torch.from_numpy(base[:n0]).cuda(), batch=0, seed=5)
    new_ids = idx.insert(torch.from_numpy(base[n0:]).cuda())
    assert new_ids.cpu().tolist() == list(range(n0, n0 + n1))
    # oracle: patchGraph semantics on the same graph
    deg = np.zeros(n0 + n1, np.uint32)
    adj = np.zeros((n0 + n1, R), np.uint32)
    deg[:n0], adj[:n0] = og.deg, og.adj
    g2 = oracle.Graph(base, deg, adj)
    assert g2.vamana_batch(n0, n1, L, 1.2, entry, skip_mode=0) == 0
    _, gdeg, gadj = idx.get_graph()
    assert _rows_equal(gdeg, gadj, g2.deg, g2.adj) == []


@pytest.mark.parametrize("stores", [("f32",), ("f32", "u8")], ids=["cuda_cores", "tensor_cores"])
def test_insert_over_lists_out_of_order(oracle, vann_mod, stores):
    """The reverse re-prune merges a node's new sources into its list when the list is in
    RobustPrune order (nondecreasing distance) and sorts the candidates otherwise.  A
    graph set from outside with every other list reversed takes both paths in one insert
    batch.  Every row the batch touches (the new rows and the targets of their edges)
    must equal the oracle's.  The oracle re-prunes every node, as the reference does, so
    it also puts the untouched reversed lists back in order; the engine, told the lists
    are consistent, re-prunes only the targets and leaves the other rows as they were."""
    import torch

    n0, n1, R, L = 3000, 300, 32, 64
    base = workload.mixture(n0 + n1, 128, 30, seed=36)
    og, entry = oracle.build_index(base[:n0], R=R, L=L, alpha=1.2, seed=6, skip_mode=2)
    deg = np.zeros(n0 + n1, np.uint32)
    adj = np.zeros((n0 + n1, R), np.uint32)
    deg[:n0] = og.deg
    for i in range(n0):
        row = og.adj[i, :og.deg[i]]
        adj[i, :og.deg[i]] = row[::-1] if i % 2 == 0 else row
    idx = vann_mod.Index(128, R, L, 1.2, capacity=n0 + n1, stores=stores)
    idx.set_graph(base[:n0], deg[:n0], adj[:n0], entry, consistent=True)
    new_ids = idx.insert(torch.from_numpy(base[n0:]).cuda())
    assert new_ids.cpu().tolist() == list(range(n0, n0 + n1))
    g2 = oracle.Graph(base, deg.copy(), adj.copy())
    assert g2.vamana_batch(n0, n1, L, 1.2, entry, skip_mode=0) == 0
    _, gdeg, gadj = idx.get_graph()
    live = np.arange(R)[None, :] < g2.deg[n0:, None]
    touched = np.zeros(n0 + n1, bool)
    touched[n0:] = True
    touched[np.unique(g2.adj[n0:][live])] = True
    want_deg = np.where(touched, g2.deg, deg)
    want_adj = np.where(touched[:, None], g2.adj, adj)
    assert _rows_equal(gdeg, gadj, want_deg, want_adj) == []
    assert 0 < touched[:n0].sum() < n0  # both kinds of old rows occur


def test_delete_consolidate_and_reuse(oracle, vann_mod):
    import torch

    n, R, L = 4000, 32, 64
    base = workload.mixture(n, 128, 30, seed=34)
    q = workload.mixture(200, 128, 30, seed=35)
    idx = vann_mod.Index(128, R, L, 1.2, capacity=n)
    idx.build(torch.from_numpy(base).cuda(), batch=0, seed=5)
    rng = np.random.default_rng(0)
    dead = rng.choice(n, 400, replace=False).astype(np.int32)
    idx.delete(torch.from_numpy(dead).cuda())
    qd = torch.from_numpy(q).cuda()
    ids, _ = idx.search(qd, k=10, L=64)
    got = set(ids.cpu().numpy().ravel().tolist())
    entry = idx.info()["entry"]
    assert not (got & (set(dead.tolist()) - {entry}))
    idx.consolidate()
    info = idx.info()
    assert info["free_ids"] == 400 and info["entry"] not in set(dead.tolist())
    _, deg, adj = idx.get_graph()
    dead_set = set(dead.tolist())
    for i in range(n):
        if i in dead_set:
            assert deg[i] == 0
        else:
            assert not (set(adj[i, :deg[i]].tolist()) & dead_set)
    live = np.array(sorted(set(range(n)) - dead_set))
    truth, _ = oracle.bruteforce_knn(base[live], q, 10)
    ids, _ = idx.search(qd, k=10, L=64)
    assert oracle.recall_at_k(ids.cpu().numpy(), live[truth], 10) >= 0.93
    # inserts reuse the freed ids
    extra = workload.mixture(100, 128, 30, seed=36)
    new = idx.insert(torch.from_numpy(extra).cuda()).cpu().numpy()
    assert set(new.tolist()) <= dead_set
    ids, d = idx.search(torch.from_numpy(extra[:20]).cuda(), k=1, L=64)
    assert (ids.cpu().numpy()[:, 0] == new[:20]).mean() >= 0.95


def test_delete_by_vector(vann_mod):
    import torch

    base = workload.mixture(2000, 128, 20, seed=37)
    idx = vann_mod.Index(128, 32, 64, 1.2, capacity=2000)
    idx.build(torch.from_numpy(base).cuda(), batch=0, seed=1)
    probe = np.concatenate([base[[5, 17, 1999]], np.full((1, 128), -1, np.float32)])
    out = idx.delete_by_vector(torch.from_numpy(probe).cuda()).cpu().numpy()
    assert out.tolist() == [5, 17, 1999, -1]


def test_save_load_roundtrip(vann_mod, tmp_path):
    import torch

    base = workload.mixture(1500, 128, 20, seed=38)
    idx = vann_mod.Index(128, 64, 64, 1.2, capacity=1500)
    idx.build(torch.from_numpy(base).cuda(), batch=0, seed=1)
    p = str(tmp_path / "g.bin")
    idx.save_graph(p)
    import os

    assert os.path.getsize(p) == 1500 * 772  # the reference's record layout
    idx2 = vann_mod.Index(128, 64, 64, 1.2, capacity=1500)
    idx2.load_graph(p, 1500, idx.info()["entry"])
    va, da, aa = idx.get_graph()
    vb, db, ab = idx2.get_graph()
    assert np.array_equal(va, vb) and np.array_equal(da, db)
    for i in range(1500):
        assert np.array_equal(aa[i, :da[i]], ab[i, :db[i]])


def test_build_over_loaded_start_graph(oracle, vann_mod):
    """runVamana over a start graph read from the caller (the reference reads one
    from sift10k_randomgraph.bin): the loaded adjacency, duplicates included, is
    the start graph."""
    import torch  # noqa: F401

    n, R, L = 3000, 64, 100
    base = workload.mixture(n, 128, 30, seed=39)
    rng = np.random.default_rng(5)
    adj = rng.integers(0, n, (n, R)).astype(np.uint32)  # with duplicates, like the reference's file
    deg = np.full(n, R, np.uint32)
    entry = 1500
    og = oracle.Graph(base, deg.copy(), adj.copy())
    assert og.vamana_batch(0, n, L, 1.5, entry, 600, 500, skip_mode=1,
                           bloom_mode=oracle.BLOOM_SNAPSHOT) == 0
    idx = vann_mod.Index(128, R, L, 1.5, capacity=n, quirks=vann_mod.QUIRK_SKIP_BATCH_INDEX)
    idx.set_graph(base, deg, adj, entry)
    idx.build_loaded()
    _, gdeg, gadj = idx.get_graph()
    assert _rows_equal(gdeg, gadj, og.deg, og.adj) == []
