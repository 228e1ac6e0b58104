"""The continuous-batching server: every result of a mixed burst of requests (uneven k
and L, inserts, deletes, consolidation) equals the same request run alone, one call at a
time, on an identically built index.  Search ids and distances are compared bit for bit."""
import numpy as np
import pytest

from vann import workload

pytestmark = pytest.mark.gpu


def _index(vann_mod, base):
    import torch

    idx = vann_mod.Index(128, 32, 64, 1.2, capacity=len(base) + 2000)
    idx.build(torch.from_numpy(base).cuda(), batch=0, seed=13)
    return idx


def test_server_mixed_results_equal_alone(vann_mod):
    import torch

    base = workload.mixture(8000, 128, 30, seed=81)
    served, alone = _index(vann_mod, base), _index(vann_mod, base)
    srv = vann_mod.Server(served, max_batch=256, slots=4, max_k=100)
    rng = np.random.default_rng(5)
    ops, live_initial = [], list(range(len(base)))
    for i in range(400):
        u = rng.random()
        if u < 0.9:
            nqr = int(rng.integers(1, 5))
            k = int(rng.choice([1, 10, 100]))
            L = max(k, int(rng.integers(16, 257)))
            ops.append(("search", workload.mixture(nqr, 128, 30, seed=10_000 + i), k, L))
        elif u < 0.95:
            ops.append(("insert", workload.mixture(int(rng.integers(1, 40)), 128, 30, seed=20_000 + i)))
        elif u < 0.99:
            pick = rng.choice(len(live_initial), int(rng.integers(1, 20)), replace=False)
            ids = np.array([live_initial[j] for j in pick], np.uint32)
            live_initial = [x for j, x in enumerate(live_initial) if j not in set(pick.tolist())]
            ops.append(("delete", ids))
        else:
            ops.append(("consolidate",))
    # the whole burst is queued at once, so searches share batches
    tickets = []
    for op in ops:
        if op[0] == "search":
            tickets.append(srv.submit_search(op[1], op[2], op[3]))
        elif op[0] == "insert":
            tickets.append(srv.submit_insert(op[1]))
        elif op[0] == "delete":
            tickets.append(srv.submit_delete(op[1]))
        else:
            tickets.append(srv.submit_consolidate())
    results = [srv.wait(t) for t in tickets]
    st = srv.stats()
    n_search = sum(op[0] == "search" for op in ops)
    print(st, n_search)
    assert st["batches"] < n_search  # requests were batched together
    srv.close()

    for op, (ids, d, lat) in zip(ops, results):
        assert lat > 0
        if op[0] == "search":
            gi, gd = alone.search(torch.from_numpy(op[1]).cuda(), k=op[2], L=op[3])
            assert np.array_equal(ids, gi.cpu().numpy().view(np.uint32))
            assert np.array_equal(d, gd.cpu().numpy())
        elif op[0] == "insert":
            new = alone.insert(torch.from_numpy(op[1]).cuda()).cpu().numpy().view(np.uint32)
            assert np.array_equal(ids, new)
        elif op[0] == "delete":
            alone.delete(torch.from_numpy(op[1].astype(np.int32)).cuda())
        else:
            alone.consolidate()


def test_server_budget_caps_slots(vann_mod):
    base = workload.mixture(2000, 128, 10, seed=82)
    idx = _index(vann_mod, base)
    slot = 64 * (128 * 4 + 10 * 8 + 8)
    srv = vann_mod.Server(idx, max_batch=64, slots=8, max_k=10, hbm_budget=3 * slot)
    assert srv.stats()["slots"] == 3
    srv.close()
    with pytest.raises(vann_mod.VannError):
        vann_mod.Server(idx, max_batch=64, slots=8, max_k=10, hbm_budget=slot - 1)


def test_group_commit_replays_by_epoch(vann_mod):
    """Group commit: searches flow past queued writes and report the epoch (number of
    writes applied) they were served at; writes are applied in submission order.
    Replaying the writes in order on an identical index and running each search after
    its epoch's writes gives bit-identical results."""
    import torch

    base = workload.mixture(8000, 128, 30, seed=83)
    served, alone = _index(vann_mod, base), _index(vann_mod, base)
    srv = vann_mod.Server(served, max_batch=256, slots=4, max_k=100, commit_interval_us=3000)
    rng = np.random.default_rng(6)
    ops, live = [], list(range(len(base)))
    for i in range(400):
        u = rng.random()
        if u < 0.88:
            k = int(rng.choice([1, 10, 100]))
            ops.append(("search", workload.mixture(int(rng.integers(1, 5)), 128, 30, seed=30_000 + i),
                        k, max(k, int(rng.integers(16, 257)))))
        elif u < 0.94:
            ops.append(("insert", workload.mixture(int(rng.integers(1, 40)), 128, 30, seed=40_000 + i)))
        elif u < 0.99:
            pick = set(rng.choice(len(live), int(rng.integers(1, 20)), replace=False).tolist())
            ops.append(("delete", np.array([live[j] for j in sorted(pick)], np.uint32)))
            live = [x for j, x in enumerate(live) if j not in pick]
        else:
            ops.append(("consolidate",))
    tickets = []
    for op in ops:
        if op[0] == "search":
            tickets.append(srv.submit_search(op[1], op[2], op[3]))
        elif op[0] == "insert":
            tickets.append(srv.submit_insert(op[1]))
        elif op[0] == "delete":
            tickets.append(srv.submit_delete(op[1]))
        else:
            tickets.append(srv.submit_consolidate())
    results = [srv.wait(t, with_epoch=True) for t in tickets]
    st = srv.stats()
    srv.close()
    writes = [i for i, op in enumerate(ops) if op[0] != "search"]
    assert st["writes"] == len(writes) and st["epoch"] == len(writes)
    # writes were applied in submission order: the j-th write has epoch j + 1
    assert [results[i][3] for i in writes] == list(range(1, len(writes) + 1))
    searches = [i for i, op in enumerate(ops) if op[0] == "search"]
    assert all(0 <= results[i][3] <= len(writes) for i in searches)
    assert st["batches"] < len(searches)

    by_epoch = {}
    for i in searches:
        by_epoch.setdefault(results[i][3], []).append(i)
    for e in range(len(writes) + 1):
        for i in by_epoch.get(e, []):
            op, (ids, d, _, _) = ops[i], results[i]
            gi, gd = alone.search(torch.from_numpy(op[1]).cuda(), k=op[2], L=op[3])
            assert np.array_equal(ids, gi.cpu().numpy().view(np.uint32))
            assert np.array_equal(d, gd.cpu().numpy())
        if e == len(writes):
            break
        op, res = ops[writes[e]], results[writes[e]]
        if op[0] == "insert":
            new = alone.insert(torch.from_numpy(op[1]).cuda()).cpu().numpy().view(np.uint32)
            assert np.array_equal(res[0], new)
        elif op[0] == "delete":
            alone.delete(torch.from_numpy(op[1].astype(np.int32)).cuda())
        else:
            alone.consolidate()


def test_large_batches_in_flight_together(vann_mod):
    """Batches larger than 16 queries per SM are ordered on the device before their
    search; several such batches on the server's slot streams at once each keep their
    own order workspace, so every result still equals the request run alone."""
    import torch

    base = workload.mixture(8000, 128, 30, seed=82)
    idx = _index(vann_mod, base)
    reqs = [workload.mixture(3000, 128, 30, seed=30_000 + i) for i in range(8)]
    want = [idx.search(torch.from_numpy(r).cuda(), k=10, L=48) for r in reqs]
    torch.cuda.synchronize()
    srv = vann_mod.Server(idx, max_batch=6000, slots=4, max_k=10)
    tickets = [srv.submit_search(r, 10, 48) for r in reqs]
    for t, (wi, wd) in zip(tickets, want):
        ids, d, _ = srv.wait(t)
        assert np.array_equal(ids, wi.cpu().numpy().view(np.uint32))
        assert np.array_equal(d, wd.cpu().numpy())
    st = srv.stats()
    assert st["max_inflight"] >= 2, st  # batches overlapped on the device
    srv.close()


def test_server_float_rows_on_the_uint8_grid(vann_mod):
    """Searches served from the uint8 copy of float rows (scalar quantization on the fitted
    grid, exact FP32 rerank), batched together with uneven k and L, equal the same
    searches run alone."""
    import torch

    D = 96
    base = workload.mixture(6000, D, 30, seed=91, sigma=0.05, integer=False, unit_norm=True)
    idx = vann_mod.Index(D, 32, 64, 1.2, capacity=len(base), stores=("f32", "u8"))
    idx.build(torch.from_numpy(base).cuda(), batch=0, seed=14)
    srv = vann_mod.Server(idx, max_batch=128, slots=3, max_k=32, store="u8", rerank=True)
    rng = np.random.default_rng(9)
    ops = []
    for i in range(120):
        k = int(rng.choice([1, 10, 32]))
        L = max(k, int(rng.integers(16, 129)))
        ops.append((workload.mixture(int(rng.integers(1, 6)), D, 30, seed=30_000 + i, sigma=0.05, integer=False,
                                     unit_norm=True), k, L))
    tickets = [srv.submit_search(q, k, L) for q, k, L in ops]
    results = [srv.wait(t) for t in tickets]
    assert srv.stats()["batches"] < len(ops)
    srv.close()
    for (q, k, L), (ids, d, _) in zip(ops, results):
        gi, gd = idx.search(torch.from_numpy(q).cuda(), k=k, L=L, store="u8", rerank=True)
        assert np.array_equal(ids, gi.cpu().numpy().view(np.uint32))
        assert np.array_equal(d, gd.cpu().numpy())
