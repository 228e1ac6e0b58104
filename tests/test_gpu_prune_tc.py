"""Tensor-core RobustPrune (prune_tc.cu): with an exact uint8 copy the Gram matrix
of each node's candidates comes from tcgen05.mma, and every graph it builds must be
bit-identical to the CUDA-core path and to the CPU oracle."""
import numpy as np
import pytest

from vann import workload

pytestmark = pytest.mark.gpu


def _rows_equal(deg_a, adj_a, deg_b, adj_b):
    return [i for i in range(len(deg_a)) if not np.array_equal(adj_a[i, :deg_a[i]], adj_b[i, :deg_b[i]])]


def _build(vann_mod, base, R, L, stores, batch=0, seed=7, quirks=0, alpha=1.2):
    import torch

    idx = vann_mod.Index(base.shape[1], R, L, alpha, capacity=len(base) + 1000, stores=stores, quirks=quirks)
    idx.build(torch.from_numpy(base).cuda(), batch=batch, seed=seed)
    return idx


@pytest.mark.parametrize("R,L", [(32, 75), (64, 100)])
def test_one_batch_build_matches_oracle(oracle, vann_mod, R, L):
    base = workload.mixture(3000, 128, 30, seed=41)
    og, entry = oracle.build_index(base, R=R, L=L, alpha=1.2, seed=7, skip_mode=2,
                                   bloom_mode=oracle.BLOOM_SNAPSHOT)
    idx = _build(vann_mod, base, R, L, ("f32", "u8"))
    info = idx.info()
    assert info["entry"] == entry
    assert info["pruned_tc"] > 0
    _, deg, adj = idx.get_graph()
    assert _rows_equal(deg, adj, og.deg, og.adj) == []


@pytest.mark.parametrize("stores", [("f32", "u8"), ("f32",)])
def test_large_batch_build_matches_oracle(oracle, vann_mod, stores):
    """One batch of 6,000 rows: its search is ordered on the device and its first run
    times the launch-bound variants; the graph is still the oracle's, row for row."""
    base = workload.mixture(6000, 128, 40, seed=141)
    og, entry = oracle.build_index(base, R=32, L=64, alpha=1.2, seed=7, skip_mode=2,
                                   bloom_mode=oracle.BLOOM_SNAPSHOT)
    idx = _build(vann_mod, base, 32, 64, stores)
    assert idx.info()["entry"] == entry
    _, deg, adj = idx.get_graph()
    assert _rows_equal(deg, adj, og.deg, og.adj) == []


def test_batched_build_and_insert_equal_cuda_core_path(vann_mod):
    import torch

    base = workload.mixture(6000, 128, 40, seed=42)
    extra = workload.mixture(700, 128, 40, seed=43)
    tc = _build(vann_mod, base, 64, 100, ("f32", "u8"), batch=1000, seed=3)
    cc = _build(vann_mod, base, 64, 100, ("f32",), batch=1000, seed=3)
    assert tc.info()["pruned_tc"] > 0 and cc.info()["pruned_tc"] == 0
    for idx in (tc, cc):
        for s in range(0, 700, 233):  # uneven insert batches
            idx.insert(torch.from_numpy(extra[s:s + 233]).cuda())
    _, da, aa = tc.get_graph()
    _, db, ab = cc.get_graph()
    assert _rows_equal(da, aa, db, ab) == []


def test_loaded_start_graph_two_tiles(oracle, vann_mod):
    """runVamana over a loaded R=64 start graph: expansion lists of ~L plus 64
    out-neighbours give 129..256 candidates, i.e. two 128-row tiles."""
    n, R, L = 3000, 64, 150
    base = workload.mixture(n, 128, 30, seed=44)
    rng = np.random.default_rng(6)
    adj = rng.integers(0, n, (n, R)).astype(np.uint32)
    deg = np.full(n, R, np.uint32)
    entry = 1200
    og = oracle.Graph(base, deg.copy(), adj.copy())
    assert og.vamana_batch(0, n, L, 1.5, entry, 600, 500, skip_mode=1, bloom_mode=oracle.BLOOM_SNAPSHOT) == 0
    idx = vann_mod.Index(128, R, L, 1.5, capacity=n, quirks=vann_mod.QUIRK_SKIP_BATCH_INDEX, stores=("f32", "u8"))
    idx.set_graph(base, deg, adj, entry)
    idx.build_loaded()
    assert idx.info()["pruned_tc"] > 0
    _, gdeg, gadj = idx.get_graph()
    assert _rows_equal(gdeg, gadj, og.deg, og.adj) == []


@pytest.mark.parametrize("L,max_visited,cuda_share", [(300, 600, False), (600, 800, False), (900, 1100, True)])
def test_large_candidate_lists(oracle, vann_mod, L, max_visited, cuda_share):
    """257..512 candidates (expansion lists at L=300) take the second tensor-core
    pass, up to 768 (L=600) the third; more (L=900) are handed to the CUDA-core
    kernel.  Every way the graph is the oracle's."""
    import torch

    base = workload.mixture(2500, 128, 20, seed=45)
    og, entry = oracle.build_index(base, R=32, L=L, alpha=1.2, seed=9, skip_mode=2,
                                   bloom_mode=oracle.BLOOM_SNAPSHOT, max_visited=max_visited)
    idx = vann_mod.Index(128, 32, L, 1.2, capacity=2500, max_visited=max_visited, stores=("f32", "u8"))
    idx.build(torch.from_numpy(base).cuda(), batch=0, seed=9)
    info = idx.info()
    assert info["pruned_tc"] > 0
    if cuda_share:
        assert info["pruned_cuda"] > 0
    _, deg, adj = idx.get_graph()
    assert _rows_equal(deg, adj, og.deg, og.adj) == []


def test_float_rows_stand_the_tensor_core_pass_down(vann_mod):
    """Rows that are not integers in [0, 255] set the inexact flag: the uint8 copy
    still serves searches, but every prune runs on the CUDA cores."""
    base = workload.mixture(2000, 128, 20, seed=46, sigma=0.05, integer=False, unit_norm=True)
    idx = _build(vann_mod, base, 32, 64, ("f32", "u8"))
    ref = _build(vann_mod, base, 32, 64, ("f32",))
    info = idx.info()
    assert info["pruned_tc"] == 0 and info["pruned_cuda"] > 0
    _, da, aa = idx.get_graph()
    _, db, ab = ref.get_graph()
    assert _rows_equal(da, aa, db, ab) == []


def test_consolidate_equals_cuda_core_path(vann_mod):
    import torch

    base = workload.mixture(5000, 128, 30, seed=47)
    tc = _build(vann_mod, base, 32, 64, ("f32", "u8"), seed=5)
    cc = _build(vann_mod, base, 32, 64, ("f32",), seed=5)
    dead = np.random.default_rng(2).choice(5000, 600, replace=False).astype(np.int32)
    extra = workload.mixture(300, 128, 30, seed=48)
    for idx in (tc, cc):
        idx.delete(torch.from_numpy(dead).cuda())
        idx.consolidate()
        idx.insert(torch.from_numpy(extra).cuda())
    assert tc.info()["entry"] == cc.info()["entry"]
    _, da, aa = tc.get_graph()
    _, db, ab = cc.get_graph()
    assert _rows_equal(da, aa, db, ab) == []


@pytest.mark.parametrize("D", [64, 256])
def test_other_dims_match_oracle(oracle, vann_mod, D):
    """D=64 (two K steps per Gram tile) and D=256 (eight K steps, 256-byte rows, the
    wide warp layouts): batched build and insert, every prune path, against the oracle."""
    import torch

    n, B, R, L = 3000, 1000, 32, 64
    base = workload.mixture(n + 300, D, 30, seed=49)
    deg0, adj0 = oracle.random_graph(B, R, 13)
    deg = np.zeros(n + 300, np.uint32)
    adj = np.zeros((n + 300, R), np.uint32)
    deg[:B], adj[:B] = deg0, adj0
    og = oracle.Graph(base, deg, adj)
    entry = oracle.medoid(base[:B])
    assert og.vamana_batch(0, B, L, 1.2, entry, skip_mode=2) == 0
    for s in range(B, n, B):
        assert og.vamana_batch(s, B, L, 1.2, entry, skip_mode=0) == 0
    assert og.vamana_batch(n, 300, L, 1.2, entry, skip_mode=0) == 0
    idx = vann_mod.Index(D, R, L, 1.2, capacity=n + 300, stores=("f32", "u8"))
    idx.build(torch.from_numpy(base[:n]).cuda(), batch=B, seed=13)
    idx.insert(torch.from_numpy(base[n:]).cuda())
    info = idx.info()
    assert info["pruned_tc"] > 0 and info["pruned_cuda"] > 0
    _, gdeg, gadj = idx.get_graph()
    assert _rows_equal(gdeg, gadj, og.deg, og.adj) == []
    q = workload.mixture(100, D, 30, seed=50)
    ids, d = idx.search(torch.from_numpy(q).cuda(), k=10, L=48, store="u8")
    st, oids, od, _, _ = og.search(q, 48, 10, entry, bloom_mode=oracle.BLOOM_SNAPSHOT)
    assert np.array_equal(ids.cpu().numpy().view(np.uint32), oids)
    assert np.array_equal(d.cpu().numpy(), od)
