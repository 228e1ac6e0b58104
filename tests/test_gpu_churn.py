"""FreshVamana churn at small scale: rounds of lazy deletes, consolidation and uneven
insert batches; recall over the live points and the graph invariants after each round."""
import numpy as np
import pytest

from vann import workload

pytestmark = pytest.mark.gpu


def test_churn_rounds(oracle, vann_mod):
    import torch

    n, R, L, rounds = 20000, 32, 64, 3
    base = workload.mixture(n, 128, 40, seed=51)
    q = workload.mixture(200, 128, 40, seed=52)
    cap = int(n * 1.1)
    vec = np.zeros((cap, 128), np.float32)
    vec[:n] = base
    idx = vann_mod.Index(128, R, L, 1.2, capacity=cap, stores=("f32", "u8"))
    idx.build(torch.from_numpy(base).cuda(), batch=5000, seed=9)
    rng = np.random.default_rng(3)
    live = np.arange(n)
    qd = torch.from_numpy(q).cuda()
    truth0, _ = oracle.bruteforce_knn(base, q, 10)
    ids0, _ = idx.search(qd, k=10, L=L)
    recall0 = oracle.recall_at_k(ids0.cpu().numpy(), truth0, 10)
    print(f"recall before churn {recall0:.4f}")
    for r in range(rounds):
        ndel = int(0.05 * len(live))
        dels = rng.choice(live, ndel, replace=False)
        idx.delete(torch.from_numpy(dels.astype(np.int32)).cuda())
        # lazily deleted ids never come back from a search (the entry point aside)
        ids, _ = idx.search(qd, k=10, L=L)
        entry = idx.info()["entry"]
        assert not (set(ids.cpu().numpy().ravel().tolist()) & (set(dels.tolist()) - {entry}))
        idx.consolidate()
        live = np.setdiff1d(live, dels, assume_unique=True)
        newv = workload.mixture(ndel, 128, 40, seed=600 + r)
        off, new_ids = 0, []
        for s in (300, 50, ndel - 350):
            new_ids.append(idx.insert(torch.from_numpy(newv[off:off + s]).cuda()).cpu().numpy())
            off += s
        new_ids = np.concatenate(new_ids)
        assert set(new_ids.tolist()) <= set(dels.tolist())  # consolidated ids are reused
        vec[new_ids] = newv
        live = np.concatenate([live, new_ids])
        info = idx.info()
        assert info["size"] == n and info["free_ids"] == 0
        _, deg, adj = idx.get_graph()
        live_set = set(live.tolist())
        for i in rng.choice(live, 500, replace=False):
            assert set(adj[i, :deg[i]].tolist()) <= live_set
        truth, _ = oracle.bruteforce_knn(vec[live], q, 10)
        rec = {}
        for store in ("f32", "u8"):  # the u8 copy of reused rows was rewritten too
            ids, _ = idx.search(qd, k=10, L=L, store=store)
            rec[store] = oracle.recall_at_k(ids.cpu().numpy(), live[truth], 10)
        print(f"round {r + 1}: recall {rec}")
        # integer data: the exact uint8 copy must give the same results as FP32
        assert rec["u8"] == rec["f32"]
        # quality holds across churn: within 3 points of the index before any delete
        assert rec["f32"] >= recall0 - 0.03, (rec, recall0)
