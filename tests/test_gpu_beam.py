"""Two parents per hop (beam=2), the batched search form beside the reference's
GreedySearch: the kernel equals the plain-Python restatement in beam_restatement.py
(pinned to the oracle at beam 1 by test_beam_restatement.py) bit for bit on integer
data, keeps recall, halves the hops, and rejects what it does not cover."""
import numpy as np
import pytest

from beam_restatement import beam_search
from vann import workload

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def graph(oracle):
    base = workload.mixture(2000, 128, 20, seed=121)
    g, entry = oracle.build_index(base, R=32, L=64, alpha=1.2, seed=121)
    return base, g, entry


@pytest.mark.parametrize("L,store", [(16, "f32"), (32, "u8"), (64, "f32"), (48, "u8")])
def test_beam2_matches_restatement(oracle, vann_mod, graph, L, store):
    import torch

    base, g, entry = graph
    q = workload.mixture(40, 128, 20, seed=123)
    idx = vann_mod.Index(128, 32, 64, 1.2, capacity=2000, stores=("f32", "u8"))
    idx.set_graph(base, g.deg, g.adj, entry, consistent=True)
    ids, d = idx.search(torch.from_numpy(q).cuda(), k=10, L=L, store=store, beam=2)
    ids, d = ids.cpu().numpy().view(np.uint32), d.cpu().numpy()
    for i in range(len(q)):
        rid, rd = beam_search(oracle, base, g.deg, g.adj, q[i], L, 10, entry, 2)
        assert np.array_equal(ids[i], rid), i
        assert np.array_equal(d[i], rd), i


def test_beam2_recall_hops_and_limits(oracle, vann_mod):
    import torch

    base = workload.mixture(20000, 128, 40, seed=124)
    q = workload.mixture(500, 128, 40, seed=125)
    idx = vann_mod.Index(128, 64, 100, 1.2, capacity=20000, stores=("f32", "u8"))
    idx.build(torch.from_numpy(base).cuda(), batch=5000, seed=3)
    qd = torch.from_numpy(q).cuda()
    truth, _ = oracle.bruteforce_knn(base, q, 10)
    _, _, s1 = idx.search_stats(qd, k=10, L=32, store="u8")
    i2, d2, s2 = idx.search_stats(qd, k=10, L=32, store="u8", beam=2)
    i1, _ = idx.search(qd, k=10, L=32, store="u8")
    r1 = oracle.recall_at_k(i1.cpu().numpy(), truth, 10)
    r2 = oracle.recall_at_k(i2.cpu().numpy(), truth, 10)
    assert r2 >= r1 - 0.01, (r1, r2)
    h1, h2 = s1[0].float().mean().item(), s2[0].float().mean().item()
    assert h2 < 0.7 * h1, (h1, h2)  # about half the hops
    # the same two-parent search on the FP32 rows: exact integer distances, same results
    f2 = idx.search(qd, k=10, L=32, store="f32", beam=2)
    assert torch.equal(f2[0], i2) and torch.equal(f2[1], d2)
    # repeatable
    again = idx.search(qd, k=10, L=32, store="u8", beam=2)
    assert torch.equal(again[0], i2) and torch.equal(again[1], d2)
    with pytest.raises(vann_mod.VannError) as e:
        idx.search(qd, k=10, L=100, beam=2)  # beyond the register worklist
    assert e.value.status == vann_mod.ERR_UNSUPPORTED
    with pytest.raises(vann_mod.VannError) as e:
        idx.search(qd, k=10, L=32, beam=3)
    assert e.value.status == vann_mod.ERR_INVALID


def test_beam2_uneven_batch_equals_separate_launches(vann_mod, graph):
    """Per-query L and k with two parents per hop: each row is the separate search's."""
    import torch

    base, g, entry = graph
    q = workload.mixture(64, 128, 20, seed=126)
    idx = vann_mod.Index(128, 32, 64, 1.2, capacity=2000, stores=("f32", "u8"))
    idx.set_graph(base, g.deg, g.adj, entry, consistent=True)
    rng = np.random.default_rng(4)
    ks = rng.choice([1, 5, 10], 64).astype(np.int32)
    Ls = np.maximum(ks, rng.integers(8, 65, 64)).astype(np.int32)
    qd = torch.from_numpy(q).cuda()
    ids, d = idx.search_uneven(qd, torch.from_numpy(Ls).cuda(), torch.from_numpy(ks).cuda(), store="u8", beam=2)
    ids, d = ids.cpu().numpy().view(np.uint32), d.cpu().numpy()
    for i in range(64):
        a, b = idx.search(qd[i:i + 1].contiguous(), k=int(ks[i]), L=int(Ls[i]), store="u8", beam=2)
        assert np.array_equal(ids[i, :ks[i]], a.cpu().numpy().view(np.uint32)[0])
        assert np.array_equal(d[i, :ks[i]], b.cpu().numpy()[0])
