"""Properties of the CPU oracle on seeded synthetic data (no GPU, no reference files)."""
import numpy as np
import pytest

from vann import workload


@pytest.fixture(scope="module")
def small():
    base = workload.mixture(3000, 128, 30, seed=11)
    q = workload.mixture(50, 128, 30, seed=12)
    return base, q


def test_build_degrees_and_ids(oracle, small):
    base, _ = small
    g, entry = oracle.build_index(base, R=32, L=75, alpha=1.2, seed=5)
    assert g.deg.max() <= 32 and g.deg.min() >= 1
    for i in range(0, g.n, 97):
        row = g.adj[i, :g.deg[i]]
        assert (row < g.n).all()
        assert len(set(row.tolist())) == len(row)  # RobustPrune never keeps duplicates


def test_build_is_deterministic(oracle, small):
    base, _ = small
    a, _ = oracle.build_index(base, R=32, L=50, alpha=1.2, seed=5, threads=1)
    b, _ = oracle.build_index(base, R=32, L=50, alpha=1.2, seed=5, threads=8)
    assert np.array_equal(a.deg, b.deg)
    for i in range(a.n):
        assert np.array_equal(a.adj[i, :a.deg[i]], b.adj[i, :b.deg[i]])


def test_recall(oracle, small):
    base, q = small
    g, entry = oracle.build_index(base, R=32, L=75, alpha=1.2, seed=5)
    st, ids, d, hops, evals = g.search(q, 75, 10, entry)
    truth, td = oracle.bruteforce_knn(base, q, 10)
    assert st == 0
    assert oracle.recall_at_k(ids, truth, 10) >= 0.95
    # reported distances are the exact squared L2 of the reported ids
    for s in range(5):
        for t in range(10):
            exact = float(((base[ids[s, t]].astype(np.float64) - q[s]) ** 2).sum())
            assert d[s, t] == pytest.approx(exact, rel=0, abs=0)


def test_robust_prune_rule(oracle, small):
    base, _ = small
    g = oracle.Graph(base, np.zeros(len(base), np.uint32), np.zeros((len(base), 32), np.uint32))
    node = 7
    cand = np.array([i for i in range(100) if i != node], np.uint32)
    cd = np.array([((base[c] - base[node]) ** 2).sum() for c in cand], np.float32)
    order = np.argsort(cd, kind="stable")
    cand, cd = cand[order], cd[order]
    out = g.robust_prune(base[node], cand, cd, 1.2, 32)
    # restate the rule directly
    status = np.zeros(len(cand), int)
    chosen = []
    while len(chosen) < 32:
        idx = np.where(status == 0)[0]
        if len(idx) == 0:
            break
        f = idx[0]
        chosen.append(cand[f])
        status[f] = 2
        ps = base[cand[f]]
        for t in np.where(status == 0)[0]:
            dd = np.float32(((base[cand[t]] - ps) ** 2).sum())
            if np.float32(dd * np.float32(1.2)) <= cd[t]:
                status[t] = 1
    assert out.tolist() == [int(c) for c in chosen]


def test_hop_limit_status(oracle, small):
    base, q = small
    g, entry = oracle.build_index(base, R=32, L=50, alpha=1.2, seed=5)
    st, ids, d, hops, evals = g.search(q[:4], 50, 10, entry, max_hops=3)
    assert st == 5 and (hops <= 3).all()


def test_insert_batch_matches_full_rebuild_shape(oracle, small):
    base, q = small
    n0 = 2000
    deg, adj = oracle.random_graph(n0, 32, 9)
    deg_all = np.zeros(len(base), np.uint32)
    adj_all = np.zeros((len(base), 32), np.uint32)
    deg_all[:n0] = deg
    adj_all[:n0] = adj
    g = oracle.Graph(base, deg_all, adj_all)
    entry = oracle.medoid(base[:n0])
    assert g.vamana_batch(0, n0, 64, 1.2, entry, skip_mode=2) == 0
    assert g.vamana_batch(n0, 1000, 64, 1.2, entry, skip_mode=0) == 0
    assert (g.deg[n0:] > 0).all()
    st, ids, d, _, _ = g.search(q, 64, 10, entry)
    truth, _ = oracle.bruteforce_knn(base, q, 10)
    assert oracle.recall_at_k(ids, truth, 10) >= 0.9


def _merge_rerank_literal(vecs, q, graph_ids, il):
    """merge_and_rerank_kernel (vamana/include/utils.cuh:199-285) line by line, with
    the FP32 arithmetic of l2_distance_sq (:150-158) done exactly (integer rows)."""
    nq, L = graph_ids.shape
    out_i = np.full((nq, L), 0xFFFFFFFF, np.uint32)
    out_d = np.full((nq, L), np.inf, np.float32)
    for qi in range(nq):
        sd = [np.inf] * L
        si = [0xFFFFFFFF] * L
        cands = [(int(g), vecs[g]) for g in graph_ids[qi] if g != 0xFFFFFFFF]
        cands += [(0x80000000 | s, il[s]) for s in range(len(il))]
        for cid, row in cands:
            dist = float(((q[qi].astype(np.float64) - row) ** 2).sum())
            max_d, max_k = -1.0, 0
            for k in range(L):
                if sd[k] > max_d:
                    max_d, max_k = sd[k], k
            if dist < max_d:
                sd[max_k], si[max_k] = dist, cid
        for i in range(L - 1):
            for j in range(L - i - 1):
                if sd[j] > sd[j + 1]:
                    sd[j], sd[j + 1] = sd[j + 1], sd[j]
                    si[j], si[j + 1] = si[j + 1], si[j]
        out_i[qi], out_d[qi] = si, sd
    return out_i, out_d


def test_merge_rerank_matches_the_reference_loop(oracle):
    """The oracle's searchPoints2 merge against a literal port of the reference's
    loop, on small integer rows chosen to tie often (first-slot eviction matters)."""
    rng = np.random.default_rng(12)
    n, D, L = 300, 16, 12
    vecs = rng.integers(0, 3, (n, D)).astype(np.float32)
    il = rng.integers(0, 3, (40, D)).astype(np.float32)
    q = rng.integers(0, 3, (25, D)).astype(np.float32)
    gids = rng.integers(0, n, (25, L)).astype(np.uint32)
    gids[:, -2:] = 0xFFFFFFFF  # padded worklist slots
    gids[3, 1] = gids[3, 0]    # a duplicate, as the entry point gives
    ids, d = oracle.merge_rerank(vecs, q, gids, il)
    ri, rd = _merge_rerank_literal(vecs, q, gids, il)
    assert np.array_equal(ids, ri)
    assert np.array_equal(d, rd)
    assert (ids >= oracle.STAGED).any() and (ids < oracle.STAGED).any()


def test_consolidate_properties(oracle, small):
    """The oracle's delete consolidation (FreshDiskANN Algorithm 4): no live node
    keeps a deleted neighbour, every list stays a RobustPrune output (no repeats,
    degree <= R), the deleted ids are freed with degree 0, a deleted entry moves to
    a live node, the result does not depend on the thread count, and the lists of
    nodes without a deleted neighbour are untouched.  Recall over the live rows
    stays high."""
    base, q = small
    n = base.shape[0]
    g0, entry = oracle.build_index(base, R=32, L=75, alpha=1.2, seed=5)
    rng = np.random.default_rng(4)
    dead = np.unique(np.append(rng.choice(n, 300, replace=False), entry))
    tomb = oracle.tomb_bitmap(n, dead)
    a = oracle.Graph(base, g0.deg.copy(), g0.adj.copy(), tomb=tomb)
    b = oracle.Graph(base, g0.deg.copy(), g0.adj.copy(), tomb=tomb.copy())
    ea, fa = a.consolidate(1.2, 600, entry, threads=1)
    eb, fb = b.consolidate(1.2, 600, entry, threads=8)
    assert ea == eb and np.array_equal(fa, fb) and np.array_equal(a.deg, b.deg)
    assert np.array_equal(fa, np.sort(dead).astype(np.uint32))
    dead_set = set(dead.tolist())
    assert ea not in dead_set
    for i in range(n):
        row = a.adj[i, :a.deg[i]]
        assert np.array_equal(a.adj[i, :a.deg[i]], b.adj[i, :b.deg[i]])
        if i in dead_set:
            assert a.deg[i] == 0
            continue
        assert not (set(row.tolist()) & dead_set) and len(set(row.tolist())) == len(row) and len(row) <= 32
        if not (set(g0.adj[i, :g0.deg[i]].tolist()) & dead_set):
            assert np.array_equal(row, g0.adj[i, :g0.deg[i]])
    live = np.array(sorted(set(range(n)) - dead_set))
    truth, _ = oracle.bruteforce_knn(base[live], q, 10)
    st, ids, _, _, _ = a.search(q, 75, 10, ea)
    assert st == 0 and oracle.recall_at_k(ids, live[truth], 10) >= 0.95
