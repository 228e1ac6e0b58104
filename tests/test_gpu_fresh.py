"""FreshVamana write paths against the oracle, bit for bit.

* Lazy delete: a search over a graph with tombstoned ids skips them before the
  bloom-filter test, as the reference skips ids found in its delete list
  (vamana/include/search.cuh:121-123, delete_list.cuh:108-115).  The engine keeps
  a tombstone bitmap instead of the list; the oracle searches with the same bitmap.
* Delete consolidation: FreshDiskANN's Algorithm 4, which the reference lacks
  (patchGraph, vamana_impl.cuh:182-265, consolidates inserts only).  The oracle's
  vo_consolidate restates it with the engine's candidate order; graph rows, the
  entry point and the freed ids must be identical, on the CUDA-core prune and on
  the tensor-core prune (uint8 copy).
"""
import numpy as np
import pytest

from vann import workload

pytestmark = pytest.mark.gpu


def _rows_equal(deg_a, adj_a, deg_b, adj_b):
    return [i for i in range(len(deg_a)) if not np.array_equal(adj_a[i, :deg_a[i]], adj_b[i, :deg_b[i]])]


@pytest.fixture(scope="module")
def fresh_graph(oracle):
    n, R, L = 4000, 64, 64
    base = workload.mixture(n, 128, 30, seed=81)
    g, entry = oracle.build_index(base, R=R, L=L, alpha=1.2, seed=9, skip_mode=2,
                                  bloom_mode=oracle.BLOOM_SNAPSHOT)
    return base, g, entry


def _index(vann, base, g, entry, stores):
    idx = vann.Index(base.shape[1], g.R, 64, 1.2, capacity=base.shape[0] + 200, stores=stores)
    idx.set_graph(base, g.deg, g.adj, entry, consistent=True)
    return idx


@pytest.mark.parametrize("with_entry", [False, True])
def test_search_over_tombstones_bit_exact(oracle, vann_mod, fresh_graph, with_entry):
    """8% of the ids deleted (with and without the entry point): every worklist
    kernel (L=48 in registers, L=100 in shared memory), both row formats, with and
    without the batch-index quirk, equals the oracle's search with the same
    tombstones."""
    import torch

    base, g, entry = fresh_graph
    n = base.shape[0]
    rng = np.random.default_rng(3)
    dead = rng.choice(n, n * 8 // 100, replace=False)
    if with_entry:
        dead = np.unique(np.append(dead, entry))
    else:
        dead = dead[dead != entry]
    og = oracle.Graph(g.vecs, g.deg.copy(), g.adj.copy(), tomb=oracle.tomb_bitmap(n, dead))
    q = workload.mixture(300, 128, 30, seed=82)
    qd = torch.from_numpy(q).cuda()
    idx = _index(vann_mod, base, g, entry, ("f32", "u8"))
    idx.delete(torch.from_numpy(dead.astype(np.int32)).cuda())
    dead_set = set(dead.tolist())
    for L in (48, 100):
        for quirk in (0, 1):
            st, oids, od, oh, oe = og.search(q, L, 10, entry, skip_mode=quirk, bloom_mode=oracle.BLOOM_SNAPSHOT)
            assert st == 0
            # no deleted id is ever found as a neighbour (the entry itself stays in the list)
            assert not (set(oids.ravel().tolist()) & (dead_set - {entry}))
            for store in ("f32", "u8"):
                ids, d, stats = idx.search_stats(qd, k=10, L=L, store=store, quirks=quirk)
                idx.sync()
                assert np.array_equal(ids.cpu().numpy().view(np.uint32), oids), (L, quirk, store)
                assert np.array_equal(d.cpu().numpy(), od), (L, quirk, store)
                s = stats.cpu().numpy()
                assert np.array_equal(s[0], oh) and np.array_equal(s[1], oe), (L, quirk, store)


@pytest.mark.parametrize("stores", [("f32",), ("f32", "u8")], ids=["cuda_cores", "tensor_cores"])
def test_consolidate_bit_exact(oracle, vann_mod, fresh_graph, stores):
    """Two rounds of delete + consolidate (the first deletes the entry point): the
    graph, the entry and the free ids equal the oracle's; freed ids are then reused
    last-freed first."""
    import torch

    base, g, entry = fresh_graph
    n = base.shape[0]
    idx = _index(vann_mod, base, g, entry, stores)
    og = oracle.Graph(g.vecs, g.deg.copy(), g.adj.copy(), tomb=np.zeros((n + 31) // 32, np.uint32))
    rng = np.random.default_rng(11)
    dead_all = np.zeros(0, np.int64)
    is_free = np.zeros(n, np.uint8)
    o_entry = entry
    freed_all = []
    for rnd, frac in enumerate((8, 5)):
        live = np.setdiff1d(np.arange(n), dead_all)
        dead = rng.choice(live, n * frac // 100, replace=False)
        if rnd == 0:
            dead = np.unique(np.append(dead, o_entry))
        dead_all = np.union1d(dead_all, dead)
        og.tomb = oracle.tomb_bitmap(n, dead_all)
        o_entry, freed = og.consolidate(1.2, 600, o_entry, is_free=is_free)
        is_free[freed] = 1
        freed_all.extend(freed.tolist())
        idx.delete(torch.from_numpy(dead.astype(np.int32)).cuda())
        idx.consolidate()
        info = idx.info()
        assert info["entry"] == o_entry, rnd
        assert info["free_ids"] == len(freed_all), rnd
        _, gdeg, gadj = idx.get_graph()
        assert _rows_equal(gdeg, gadj, og.deg, og.adj) == [], rnd
    info = idx.info()
    if "u8" in stores:
        assert info["pruned_tc"] > 0
    else:
        assert info["pruned_tc"] == 0 and info["pruned_cuda"] > 0
    # the free list is a stack: the last freed id (the largest of the last round) comes back first
    extra = workload.mixture(5, 128, 30, seed=83)
    new = idx.insert(torch.from_numpy(extra).cuda()).cpu().numpy().tolist()
    assert new == freed_all[::-1][:5]


@pytest.mark.parametrize("stores", [("f32",), ("f32", "u8")], ids=["cuda_cores", "tensor_cores"])
def test_churn_cycle_bit_exact(oracle, vann_mod, fresh_graph, stores):
    """The whole FreshVamana cycle, twice: lazy deletes, consolidation, then inserts in
    uneven batches into the freed ids (the free list is a stack, last freed first).
    After every insert batch the graph equals the oracle's, which runs the same batch
    over the same ids (vo_vamana_batch_ids: search from the entry, out-prune, reverse
    edges in batch order, re-prune)."""
    import torch

    base, g, entry = fresh_graph
    n = base.shape[0]
    idx = _index(vann_mod, base, g, entry, stores)
    vecs = g.vecs.copy()
    og = oracle.Graph(vecs, g.deg.copy(), g.adj.copy(), tomb=np.zeros((n + 31) // 32, np.uint32))
    rng = np.random.default_rng(21)
    dead_now = set()
    is_free = np.zeros(n, np.uint8)
    free_stack = []
    o_entry = entry
    for rnd in range(2):
        live = np.array(sorted(set(range(n)) - dead_now))
        dead = rng.choice(live, n * 6 // 100, replace=False)
        dead_now |= set(dead.tolist())
        og.tomb = oracle.tomb_bitmap(n, sorted(dead_now))
        o_entry, freed = og.consolidate(1.2, 600, o_entry, is_free=is_free)
        is_free[freed] = 1
        free_stack.extend(freed.tolist())
        idx.delete(torch.from_numpy(dead.astype(np.int32)).cuda())
        idx.consolidate()
        assert idx.info()["entry"] == o_entry, rnd
        newv = workload.mixture(len(dead), 128, 30, seed=700 + rnd)
        off = 0
        for size in (37, 5, len(dead) - 42):
            rows = newv[off:off + size]
            off += size
            want = [free_stack.pop() for _ in range(size)]
            got = idx.insert(torch.from_numpy(rows).cuda()).cpu().numpy().tolist()
            assert got == want, rnd
            ids = np.array(want, np.uint32)
            og.vecs[ids] = rows
            og.deg[ids] = 0
            for i in want:
                og.tomb[i >> 5] &= np.uint32(~(1 << (i & 31)) & 0xFFFFFFFF)
                is_free[i] = 0
                dead_now.discard(i)
            assert og.vamana_batch_ids(ids, 64, 1.2, o_entry, skip_mode=0) == 0
            _, gdeg, gadj = idx.get_graph()
            assert _rows_equal(gdeg, gadj, og.deg, og.adj) == [], (rnd, size)
