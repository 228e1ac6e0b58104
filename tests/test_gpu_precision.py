"""Reduced-precision traversal on float data (unit-norm mixture, D=96): BF16 and
FP8-E4M3 with per-row scales, exact FP32 rerank; recall and distance errors."""
import numpy as np
import pytest

from vann import workload

pytestmark = pytest.mark.gpu


def test_reduced_precision_float_data(oracle, vann_mod):
    import torch

    n, D = 30000, 96
    base = workload.mixture(n, D, 60, seed=71, sigma=0.05, integer=False, unit_norm=True)
    q = workload.mixture(300, D, 60, seed=72, sigma=0.05, integer=False, unit_norm=True)
    idx = vann_mod.Index(D, 32, 64, 1.2, capacity=n, stores=("f32", "bf16", "fp8"))
    idx.build(torch.from_numpy(base).cuda(), batch=10000, seed=4)
    qd = torch.from_numpy(q).cuda()
    truth, _ = oracle.bruteforce_knn(base, q, 10)
    ids32, _ = idx.search(qd, k=10, L=64)
    r32 = oracle.recall_at_k(ids32.cpu().numpy(), truth, 10)
    assert r32 >= 0.95
    # traversal distance error bounds: the 5M x 96 run measures at most 0.33% (BF16) and
    # 5.1% (FP8, per-row scale); the bounds add a margin over those
    for store, tol in (("bf16", 5e-3), ("fp8", 0.06)):
        ids, d = idx.search(qd, k=10, L=64, store=store, rerank=True)
        gi = ids.cpu().numpy()
        assert oracle.recall_at_k(gi, truth, 10) >= r32 - 0.01
        # reranked distances: exact FP32, within 1e-5 relative of FP64
        ex = ((base[gi].astype(np.float64) - q[:, None, :].astype(np.float64)) ** 2).sum(-1)
        assert np.allclose(d.cpu().numpy(), ex, rtol=1e-5, atol=1e-7)
        # traversal distances: bounded relative error against FP64
        ids2, d2 = idx.search(qd, k=10, L=64, store=store, rerank=False)
        g2 = ids2.cpu().numpy()
        ex2 = ((base[g2].astype(np.float64) - q[:, None, :].astype(np.float64)) ** 2).sum(-1)
        rel = np.abs(d2.cpu().numpy() - ex2) / np.maximum(ex2, 1e-30)
        assert rel.max() < tol, (store, rel.max())
