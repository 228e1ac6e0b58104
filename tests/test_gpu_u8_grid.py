"""The uint8 traversal copy on float rows: scalar quantization onto a fitted grid.

Rows that are not all integers in [0, 255] get a grid with one offset per dimension
(the column minimum) and one scale s = max over dimensions of (max - min) / 255.
Codes are round((x - lo) / s), clamped to [0, 255]; a query is mapped onto the same
grid and rounded, and the search runs the exact dp4a path on the codes.  Returned
traversal distances are the code distances times s^2, so they are restated here bit
for bit from the oracle's restatement of the grid (vo_u8_grid, vo_u8_codes: FP32
arithmetic, as the kernels do it).  With rerank the returned
distances are exact FP32 and recall matches the FP32 form's.
"""
import numpy as np
import pytest

from vann import workload

pytestmark = pytest.mark.gpu


def _grid(oracle, rows):
    """The grid the library fits to `rows` (the oracle's vo_u8_grid): offsets, scale,
    1 / scale, all FP32; these rows are float, so the grid is a fitted one."""
    fitted, lo, s, inv = oracle.u8_grid(rows)
    assert fitted
    return lo, s, inv


def _codes(oracle, x, lo, inv):
    return oracle.u8_codes(x, lo, inv).astype(np.int64)


def _code_dists(oracle, q, base, ids, lo, s, inv):
    """s^2 * squared code distance of every returned id, as the kernel forms it."""
    qc = _codes(oracle, q, lo, inv)
    bc = _codes(oracle, base, lo, inv)
    out = np.empty(ids.shape, np.float32)
    s2 = np.float32(s) * np.float32(s)
    for i in range(ids.shape[0]):
        dd = ((bc[ids[i]] - qc[i][None, :]) ** 2).sum(-1)
        out[i] = dd.astype(np.float32) * s2
    return out


def _fixture(n=6000, D=96, seed=81):
    base = workload.mixture(n, D, 30, seed=seed, sigma=0.05, integer=False, unit_norm=True)
    q = workload.mixture(200, D, 30, seed=seed + 1, sigma=0.05, integer=False, unit_norm=True)
    return base, q


@pytest.mark.parametrize("D", [48, 96, 256])
def test_fitted_grid_traversal_distances_bit_exact(oracle, vann_mod, D):
    import torch

    base, q = _fixture(D=D)
    n = base.shape[0]
    idx = vann_mod.Index(D, 32, 48, 1.2, capacity=n, stores=("f32", "u8"))
    idx.build(torch.from_numpy(base).cuda(), batch=2000, seed=5)
    assert idx.info()["entry"] < n
    lo, s, inv = _grid(oracle, base)
    qd = torch.from_numpy(q).cuda()
    for L in (32, 48):
        ids, d = idx.search(qd, k=10, L=L, store="u8", rerank=False)
        gi = ids.cpu().numpy().view(np.uint32)
        gd = d.cpu().numpy()
        assert (gi < n).all()
        assert np.array_equal(gd, _code_dists(oracle, q, base, gi.astype(np.int64), lo, s, inv))
        assert (np.diff(gd, axis=1) >= 0).all()


def test_fitted_grid_rerank_recall_and_exact_distances(oracle, vann_mod):
    import torch

    base, q = _fixture(n=20000, seed=83)
    n, D = base.shape
    idx = vann_mod.Index(D, 32, 64, 1.2, capacity=n, stores=("f32", "u8"))
    idx.build(torch.from_numpy(base).cuda(), batch=5000, seed=6)
    qd = torch.from_numpy(q).cuda()
    truth, _ = oracle.bruteforce_knn(base, q, 10)
    ids32, _ = idx.search(qd, k=10, L=64)
    r32 = oracle.recall_at_k(ids32.cpu().numpy(), truth, 10)
    assert r32 >= 0.95
    ids, d = idx.search(qd, k=10, L=64, store="u8", rerank=True)
    gi = ids.cpu().numpy()
    assert oracle.recall_at_k(gi, truth, 10) >= r32 - 0.01
    ex = ((base[gi].astype(np.float64) - q[:, None, :].astype(np.float64)) ** 2).sum(-1)
    assert np.allclose(d.cpu().numpy(), ex, rtol=1e-5, atol=1e-7)
    # traversal distances against FP64: on this recipe at 1M and 5M rows the error is
    # at most 3.1% of the distance, 0.5% on average; the bounds add a margin
    ids2, d2 = idx.search(qd, k=10, L=64, store="u8", rerank=False)
    g2 = ids2.cpu().numpy()
    ex2 = ((base[g2].astype(np.float64) - q[:, None, :].astype(np.float64)) ** 2).sum(-1)
    rel = np.abs(d2.cpu().numpy() - ex2) / np.maximum(ex2, 1e-30)
    assert rel.mean() < 8e-3 and rel.max() < 0.05, (rel.mean(), rel.max())


def test_grid_fixed_for_later_inserts(oracle, vann_mod):
    """Rows inserted after the build are coded on the build's grid (no refit), values
    beyond its range clamped to the end codes."""
    import torch

    base, q = _fixture(n=5000, seed=85)
    n, D = base.shape
    first = 4000
    extra = base[first:].copy()
    extra[:50] *= 1.5  # some rows beyond the fitted range
    rows = np.concatenate([base[:first], extra])
    idx = vann_mod.Index(D, 32, 48, 1.2, capacity=n, stores=("f32", "u8"))
    idx.build(torch.from_numpy(rows[:first]).cuda(), batch=0, seed=7)
    idx.insert(torch.from_numpy(rows[first:]).cuda())
    idx.sync()
    lo, s, inv = _grid(oracle, rows[:first])
    ids, d = idx.search(torch.from_numpy(q).cuda(), k=10, L=48, store="u8", rerank=False)
    gi = ids.cpu().numpy().view(np.uint32).astype(np.int64)
    assert np.array_equal(d.cpu().numpy(), _code_dists(oracle, q, rows, gi, lo, s, inv))
    assert (gi >= first).any()  # inserted rows are found


def test_integer_rows_keep_the_identity_grid(oracle, vann_mod):
    """Integer rows in [0, 255]: the copy stays exact and distances are the oracle's."""
    import torch

    base = workload.mixture(3000, 128, 20, seed=87)
    q = workload.mixture(64, 128, 20, seed=88)
    g, entry = oracle.build_index(base, R=32, L=48, alpha=1.2, seed=1)
    idx = vann_mod.Index(128, 32, 48, 1.2, capacity=3000, stores=("f32", "u8"))
    idx.set_graph(base, g.deg, g.adj, entry, consistent=True)
    ids, d = idx.search(torch.from_numpy(q).cuda(), k=10, L=48, store="u8")
    st, oids, od, _, _ = g.search(q, 48, 10, entry)
    assert st == 0
    assert np.array_equal(ids.cpu().numpy().view(np.uint32), oids)
    assert np.array_equal(d.cpu().numpy(), od)


@pytest.mark.parametrize("D", [96, 384])
def test_fitted_grid_rerank_takes_the_best_of_each_list(vann_mod, D):
    """With rerank, each query's k results are the k closest (exact distances) of the
    list the traversal ends with, in order; uneven per-query L and k give what separate
    searches give."""
    import torch

    base, q = _fixture(n=8000, D=D, seed=89)
    n = base.shape[0]
    idx = vann_mod.Index(D, 32, 48, 1.2, capacity=n, stores=("f32", "u8"))
    idx.build(torch.from_numpy(base).cuda(), batch=4000, seed=8)
    qd = torch.from_numpy(q).cuda()
    L, k = 40, 10
    lists, _ = idx.search(qd, k=L, L=L, store="u8", rerank=False)
    ids, d = idx.search(qd, k=k, L=L, store="u8", rerank=True)
    lists = lists.cpu().numpy().view(np.uint32).astype(np.int64)
    ids = ids.cpu().numpy().view(np.uint32).astype(np.int64)
    d = d.cpu().numpy()
    for i in range(q.shape[0]):
        c = lists[i][lists[i] != 0xFFFFFFFF]
        ex = ((base[c].astype(np.float64) - q[i].astype(np.float64)) ** 2).sum(-1)
        order = np.argsort(ex, kind="stable")[:k]
        assert set(ids[i].tolist()) <= set(c.tolist())
        # the same k rows, in exact-distance order (FP32 sums may swap near-ties only)
        assert np.allclose(np.sort(ex[order]), np.sort(((base[ids[i]].astype(np.float64) -
                                                         q[i].astype(np.float64)) ** 2).sum(-1)), rtol=1e-6)
        assert (np.diff(d[i]) >= 0).all()
    # uneven: two groups of (L, k) in one launch equal the two separate searches
    Lq = torch.tensor([32 if i % 2 else 48 for i in range(q.shape[0])], dtype=torch.int32, device="cuda")
    kq = torch.tensor([5 if i % 2 else 10 for i in range(q.shape[0])], dtype=torch.int32, device="cuda")
    ui, ud = idx.search_uneven(qd, Lq, kq, store="u8", rerank=True)
    ui, ud = ui.cpu().numpy(), ud.cpu().numpy()
    for Lg, kg, sel in ((48, 10, slice(0, None, 2)), (32, 5, slice(1, None, 2))):
        si, sd = idx.search(qd[sel].contiguous(), k=kg, L=Lg, store="u8", rerank=True)
        assert np.array_equal(ui[sel][:, :kg], si.cpu().numpy())
        assert np.array_equal(ud[sel][:, :kg], sd.cpu().numpy())
        assert (ui[sel][:, kg:] == -1).all()


@pytest.mark.parametrize("L", [32, 64, 100])
def test_fitted_grid_search_is_the_oracle_search_on_the_codes(oracle, vann_mod, L):
    """On its fitted grid the uint8 search is the reference's GreedySearch over the code
    rows with the rounded queries: the oracle, given the codes as its rows, returns the
    same ids, hops and distance evaluations, and its (exact integer) distances times s^2
    are the returned distances, bit for bit; L = 100 takes the shared-memory worklist."""
    import torch

    base, q = _fixture(n=6000, seed=93)
    n, D = base.shape
    idx = vann_mod.Index(D, 32, 64, 1.2, capacity=n, stores=("f32", "u8"))
    idx.build(torch.from_numpy(base).cuda(), batch=2000, seed=9)
    _, deg, adj = idx.get_graph()
    entry = idx.info()["entry"]
    lo, s, inv = _grid(oracle, base)
    codes = _codes(oracle, base, lo, inv).astype(np.float32)
    qcodes = _codes(oracle, q, lo, inv).astype(np.float32)
    g = oracle.Graph(codes, deg, adj)
    st, oids, od, ohops, oevals = g.search(qcodes, L, 10, entry, bloom_mode=oracle.BLOOM_SNAPSHOT)
    assert st == 0
    ids, d, stats = idx.search_stats(torch.from_numpy(q).cuda(), k=10, L=L, store="u8", rerank=False)
    assert np.array_equal(ids.cpu().numpy().view(np.uint32), oids)
    s2 = np.float32(s) * np.float32(s)
    assert np.array_equal(d.cpu().numpy(), od.astype(np.float32) * s2)
    stats = stats.cpu().numpy()
    assert np.array_equal(stats[0], ohops) and np.array_equal(stats[1].astype(np.int64), oevals)
