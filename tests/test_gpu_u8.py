"""uint8 traversal copy: exact integer distances (dp4a over the codes, rows of 128
bytes spread over 4 lanes) give the oracle's search bit for bit in every worklist
kernel, at 128 and 96 dimensions, and after inserts into consolidated ids."""
import numpy as np
import pytest

from vann import workload

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("L", [16, 32, 100])
@pytest.mark.parametrize("R,dim", [(32, 96), (64, 128)])
def test_u8_search_matches_oracle(oracle, vann_mod, L, R, dim):
    """L=16/32 take the one-register worklist, L=100 the shared-memory one; 96
    dimensions leave the last chunk of every 4-lane row group empty."""
    import torch

    base = workload.mixture(3000, dim, 30, seed=91)
    g, entry = oracle.build_index(base, R=R, L=64, alpha=1.2, seed=91)
    idx = vann_mod.Index(dim, R, 64, 1.2, capacity=3100, stores=("f32", "u8"))
    idx.set_graph(base, g.deg, g.adj, entry, consistent=True)
    q = workload.mixture(200, dim, 30, seed=92)
    ids, d = idx.search(torch.from_numpy(q).cuda(), k=10, L=L, store="u8")
    st, oids, od, _, _ = g.search(q, L, 10, entry, bloom_mode=oracle.BLOOM_SNAPSHOT)
    assert st == 0
    assert np.array_equal(ids.cpu().numpy().view(np.uint32), oids)
    assert np.array_equal(d.cpu().numpy(), od)


def test_u8_codes_of_reused_ids(vann_mod):
    """Rows inserted into consolidated ids rewrite their codes: the uint8 search
    still equals the FP32 search exactly on integer data."""
    import torch

    base = workload.mixture(4000, 128, 30, seed=93)
    idx = vann_mod.Index(128, 32, 64, 1.2, capacity=4000, stores=("f32", "u8"))
    idx.build(torch.from_numpy(base).cuda(), batch=1000, seed=4)
    dead = np.random.default_rng(5).choice(4000, 500, replace=False).astype(np.int32)
    idx.delete(torch.from_numpy(dead).cuda())
    idx.consolidate()
    fresh = workload.mixture(500, 128, 30, seed=94)
    new = idx.insert(torch.from_numpy(fresh).cuda()).cpu().numpy()
    assert sorted(new.tolist()) == sorted(dead.tolist())
    q = torch.from_numpy(np.concatenate([fresh[:100], workload.mixture(100, 128, 30, seed=95)])).cuda()
    a = idx.search(q, k=10, L=48, store="f32")
    b = idx.search(q, k=10, L=48, store="u8")
    assert torch.equal(a[0], b[0]) and torch.equal(a[1], b[1])
    assert (b[0][:100, 0].cpu().numpy() == new[:100]).mean() >= 0.95


def test_u8_store_with_float_queries(vann_mod):
    """Queries that are not integers in [0, 255] take the FP32 arithmetic over the
    widened codes: on integer rows that is the FP32 search up to summation order."""
    import torch

    base = workload.mixture(3000, 128, 30, seed=96)
    idx = vann_mod.Index(128, 32, 64, 1.2, capacity=3000, stores=("f32", "u8"))
    idx.build(torch.from_numpy(base).cuda(), batch=0, seed=6)
    q = workload.mixture(200, 128, 30, seed=97, integer=False)
    qd = torch.from_numpy(q).cuda()
    a = idx.search(qd, k=10, L=32, store="f32")
    b = idx.search(qd, k=10, L=32, store="u8")
    assert (a[0] == b[0]).float().mean().item() >= 0.98
    assert np.allclose(a[1].cpu().numpy(), b[1].cpu().numpy(), rtol=1e-5, atol=0)
