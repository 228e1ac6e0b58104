"""GPU search kernel vs the CPU oracle (bit-exact on integer-valued data)."""
import numpy as np
import pytest

from vann import workload

pytestmark = pytest.mark.gpu


def _oracle_graph(oracle, n, R, L, seed=3, clusters=40, dim=128):
    base = workload.mixture(n, dim, clusters, seed=seed)
    g, entry = oracle.build_index(base, R=R, L=L, alpha=1.2, seed=seed)
    return base, g, entry


@pytest.fixture(scope="module")
def graph64(oracle):
    return _oracle_graph(oracle, 4000, 64, 64)


@pytest.fixture(scope="module")
def graph32(oracle):
    return _oracle_graph(oracle, 3000, 32, 75, seed=4)


def _gpu_index(vann, base, g, entry, stores=("f32",)):
    idx = vann.Index(base.shape[1], g.R, 64, 1.2, capacity=base.shape[0] + 100, stores=stores)
    idx.set_graph(base, g.deg, g.adj, entry, consistent=True)
    return idx


@pytest.mark.parametrize("L,k", [(10, 10), (64, 10), (150, 150)])
@pytest.mark.parametrize("quirk", [0, 1])
def test_search_bit_exact(oracle, vann_mod, graph64, L, k, quirk):
    import torch

    base, g, entry = graph64
    q = workload.mixture(300, 128, 40, seed=99)
    idx = _gpu_index(vann_mod, base, g, entry)
    ids, d = idx.search(torch.from_numpy(q).cuda(), k=k, L=L, quirks=quirk)
    idx.sync()
    st, oids, od, _, _ = g.search(q, L, k, entry, skip_mode=quirk, bloom_mode=oracle.BLOOM_SNAPSHOT)
    assert st == 0
    gi = ids.cpu().numpy().view(np.uint32)
    gd = d.cpu().numpy()
    assert np.array_equal(gi, oids)
    assert np.array_equal(gd, od)


def test_search_r32_and_padding(oracle, vann_mod, graph32):
    import torch

    base, g, entry = graph32
    q = workload.mixture(200, 128, 40, seed=98)
    idx = _gpu_index(vann_mod, base, g, entry)
    ids, d = idx.search(torch.from_numpy(q).cuda(), k=75, L=75, quirks=1)
    st, oids, od, _, _ = g.search(q, 75, 75, entry, skip_mode=1)
    assert np.array_equal(ids.cpu().numpy().view(np.uint32), oids)
    assert np.array_equal(d.cpu().numpy(), od)
    # a 2-node graph pads the tail with UINT32_MAX / +inf.  The entry sits in the
    # worklist but never in the bloom filter (search.cuh:30-58), so it is found
    # again as node 1's neighbour: 3 entries, the entry twice.
    tiny = vann_mod.Index(128, 32, 8, 1.2, capacity=4)
    adj = np.zeros((2, 32), np.uint32)
    adj[0, 0], adj[1, 0] = 1, 0
    tiny.set_graph(base[:2], np.array([1, 1], np.uint32), adj, 0)
    ids, d = tiny.search(torch.from_numpy(q[:3]).cuda(), k=5, L=8)
    ids = ids.cpu().numpy().view(np.uint32)
    assert (ids[:, 3:] == 0xFFFFFFFF).all() and np.isinf(d.cpu().numpy()[:, 3:]).all()
    for row in ids[:, :3]:
        assert sorted(row.tolist()) == [0, 0, 1]
    tg = oracle.Graph(base[:2], np.array([1, 1], np.uint32), adj)
    st, oids, _, _, _ = tg.search(q[:3], 8, 5, 0)
    assert np.array_equal(ids, oids)


def test_bf16_store_is_exact_on_integer_data(oracle, vann_mod, graph64):
    import torch

    base, g, entry = graph64
    q = workload.mixture(200, 128, 40, seed=97)
    idx = _gpu_index(vann_mod, base, g, entry, stores=("f32", "bf16", "u8"))
    qd = torch.from_numpy(q).cuda()
    a = idx.search(qd, k=10, L=64)
    for store in ("bf16", "u8"):
        b = idx.search(qd, k=10, L=64, store=store)
        assert torch.equal(a[0], b[0]) and torch.equal(a[1], b[1])


def test_fp8_rerank(oracle, vann_mod, graph64):
    import torch

    base, g, entry = graph64
    q = workload.mixture(300, 128, 40, seed=96)
    idx = _gpu_index(vann_mod, base, g, entry, stores=("f32", "fp8"))
    qd = torch.from_numpy(q).cuda()
    ids, d = idx.search(qd, k=10, L=64, store="fp8", rerank=True)
    truth, td = oracle.bruteforce_knn(base, q, 10)
    gi = ids.cpu().numpy().view(np.uint32)
    assert oracle.recall_at_k(gi, truth, 10) >= 0.95
    # reranked distances are exact FP32 squared L2 of the returned ids, ascending
    gd = d.cpu().numpy()
    for s in range(20):
        ex = ((base[gi[s]].astype(np.float64) - q[s]) ** 2).sum(1)
        assert np.allclose(gd[s], ex, rtol=0, atol=0)
        assert (np.diff(gd[s]) >= 0).all()


def test_float_data_within_tolerance(oracle, vann_mod):
    import torch

    base = workload.mixture(3000, 96, 30, seed=21, sigma=0.05, integer=False, unit_norm=True)
    g, entry = oracle.build_index(base, R=32, L=64, alpha=1.2, seed=21)
    q = workload.mixture(200, 96, 30, seed=22, sigma=0.05, integer=False, unit_norm=True)
    idx = vann_mod.Index(96, 32, 64, 1.2, capacity=3100)
    idx.set_graph(base, g.deg, g.adj, entry, consistent=True)
    ids, d = idx.search(torch.from_numpy(q).cuda(), k=10, L=64)
    st, oids, od, _, _ = g.search(q, 64, 10, entry)
    gi = ids.cpu().numpy().view(np.uint32)
    gd = d.cpu().numpy()
    # summation order differs (sequential vs warp tree): 1e-5 relative on distances,
    # and ids agree except where near-equal distances swap
    same = (gi == oids).mean()
    assert same >= 0.99
    m = gi == oids
    assert np.allclose(gd[m], od[m], rtol=1e-5, atol=1e-7)
    truth, _ = oracle.bruteforce_knn(base, q, 10)
    assert abs(oracle.recall_at_k(gi, truth, 10) - oracle.recall_at_k(oids, truth, 10)) < 0.01


def test_hop_limit_reported(oracle, vann_mod, graph64):
    import torch

    base, g, entry = graph64
    q = workload.mixture(16, 128, 40, seed=95)
    idx = _gpu_index(vann_mod, base, g, entry)
    idx.search(torch.from_numpy(q).cuda(), k=10, L=64, max_hops=3)
    with pytest.raises(vann_mod.VannError) as e:
        idx.sync()
    assert e.value.status == vann_mod.ERR_HOP_LIMIT
    idx.sync()  # cleared


def test_autotuned_variant_is_still_exact(oracle, vann_mod, graph64):
    import torch

    base, g, entry = graph64
    q = workload.mixture(256, 128, 40, seed=94)
    idx = _gpu_index(vann_mod, base, g, entry, stores=("f32", "u8"))
    qd = torch.from_numpy(q).cuda()
    st, oids, od, _, _ = g.search(q, 48, 10, entry)
    for store in ("f32", "u8"):
        idx.autotune(qd, k=10, L=48, store=store)
        ids, d = idx.search(qd, k=10, L=48, store=store)
        assert np.array_equal(ids.cpu().numpy().view(np.uint32), oids)
        assert np.array_equal(d.cpu().numpy(), od)


def test_uneven_batch_equals_separate_launches(oracle, vann_mod, graph64):
    """One launch with its own (k, L) per query gives, query by query, exactly the
    results of a separate search with that k and L (the rest of the row padded)."""
    import torch

    base, g, entry = graph64
    q = workload.mixture(96, 128, 40, seed=93)
    idx = _gpu_index(vann_mod, base, g, entry)
    rng = np.random.default_rng(1)
    ks = rng.choice([1, 10, 50], 96).astype(np.int32)
    Ls = np.maximum(ks, rng.integers(16, 200, 96)).astype(np.int32)
    qd = torch.from_numpy(q).cuda()
    ids, d = idx.search_uneven(qd, torch.from_numpy(Ls).cuda(), torch.from_numpy(ks).cuda())
    ids, d = ids.cpu().numpy().view(np.uint32), d.cpu().numpy()
    for i in range(96):
        a, b = idx.search(qd[i:i + 1].contiguous(), k=int(ks[i]), L=int(Ls[i]))
        assert np.array_equal(ids[i, :ks[i]], a.cpu().numpy().view(np.uint32)[0])
        assert np.array_equal(d[i, :ks[i]], b.cpu().numpy()[0])
        assert (ids[i, ks[i]:] == 0xFFFFFFFF).all()


@pytest.mark.parametrize("store", ["f32", "u8"])
def test_large_batch_in_any_order(oracle, vann_mod, graph64, store):
    """A batch larger than the resident warps is taken farthest-from-the-entry first
    (an order computed on the device); every query's result is still exactly the
    oracle's, and a shuffled copy of the batch gives the same rows shuffled."""
    import torch

    base, g, entry = graph64
    q = workload.mixture(6000, 128, 40, seed=91)
    idx = _gpu_index(vann_mod, base, g, entry, stores=("f32", "u8"))
    qd = torch.from_numpy(q).cuda()
    ids, d = idx.search(qd, k=10, L=48, store=store)
    st, oids, od, _, _ = g.search(q, 48, 10, entry, bloom_mode=oracle.BLOOM_SNAPSHOT)
    assert st == 0
    assert np.array_equal(ids.cpu().numpy().view(np.uint32), oids)
    assert np.array_equal(d.cpu().numpy(), od)
    perm = torch.from_numpy(np.random.default_rng(3).permutation(6000)).cuda()
    ids2, d2 = idx.search(qd[perm].contiguous(), k=10, L=48, store=store)
    assert torch.equal(ids2, ids[perm]) and torch.equal(d2, d[perm])


def test_large_batch_of_equal_distances(vann_mod, graph64):
    """A batch whose queries are all the same row puts every query in one order bucket
    (zero distance range): each is still searched once, with the same result."""
    import torch

    base, g, entry = graph64
    idx = _gpu_index(vann_mod, base, g, entry)
    one = torch.from_numpy(base[17:18]).cuda()
    ids, d = idx.search(one.repeat(5000, 1).contiguous(), k=10, L=32)
    ref, rd = idx.search(one, k=10, L=32)
    assert torch.equal(ids, ref.repeat(5000, 1)) and torch.equal(d, rd.repeat(5000, 1))
