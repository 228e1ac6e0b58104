"""Index files on the GPU path: the versioned full-state file resumes a FreshVamana
index exactly; the BANG export of a live index equals converting its 772-byte file."""
import numpy as np
import pytest

from vann import workload

pytestmark = pytest.mark.gpu


def test_index_file_resumes_exactly(vann_mod, tmp_path):
    import torch

    base = workload.mixture(4000, 128, 30, seed=91)
    a = vann_mod.Index(128, 32, 64, 1.2, capacity=5000, stores=("f32", "u8"))
    a.build(torch.from_numpy(base).cuda(), batch=1000, seed=3)
    rng = np.random.default_rng(4)
    a.delete(torch.from_numpy(rng.choice(4000, 300, replace=False).astype(np.int32)).cuda())
    a.consolidate()                                                   # 300 ids freed
    late = rng.choice(4000, 50, replace=False).astype(np.int32)
    a.delete(torch.from_numpy(late).cuda())                           # tombstoned, not freed
    p = str(tmp_path / "idx.vann")
    a.save_index(p)
    b = vann_mod.Index(128, 32, 64, 1.2, capacity=5000, stores=("f32", "u8"))
    b.load_index(p)
    ia, ib = a.info(), b.info()
    for k in ("size", "live", "free_ids", "entry", "consistent"):
        assert ia[k] == ib[k], k
    va, da, aa = a.get_graph()
    vb, db, ab = b.get_graph()
    assert np.array_equal(va, vb) and np.array_equal(da, db)
    assert all(np.array_equal(aa[i, :da[i]], ab[i, :db[i]]) for i in range(len(da)))
    q = torch.from_numpy(workload.mixture(200, 128, 30, seed=92)).cuda()
    for idx in (a, b):
        idx.consolidate()
    ra, rb = a.search(q, k=10, L=64), b.search(q, k=10, L=64)
    assert torch.equal(ra[0], rb[0]) and torch.equal(ra[1], rb[1])
    extra = torch.from_numpy(workload.mixture(100, 128, 30, seed=93)).cuda()
    assert torch.equal(a.insert(extra), b.insert(extra))              # the same ids reused
    _, da, aa = a.get_graph()
    _, db, ab = b.get_graph()
    assert all(np.array_equal(aa[i, :da[i]], ab[i, :db[i]]) for i in range(len(da)))


def test_bang_export_equals_converting_the_record_file(vann_mod, tmp_path):
    import torch

    base = workload.mixture(2000, 128, 20, seed=94)
    idx = vann_mod.Index(128, 32, 64, 1.2, capacity=2000)
    idx.build(torch.from_numpy(base).cuda(), batch=0, seed=5)
    rec = str(tmp_path / "g.bin")
    idx.save_graph(rec)
    idx.save_graph_bang(str(tmp_path / "live"))
    vann_mod.convert_graph_file(rec, 2000, 128, 32, idx.info()["entry"], str(tmp_path / "conv"))
    for suffix in ("_disk.bin", "_disk_metadata.bin"):
        assert open(str(tmp_path / "live") + suffix, "rb").read() == open(str(tmp_path / "conv") + suffix, "rb").read()
    meta = np.fromfile(str(tmp_path / "live") + "_disk_metadata.bin", dtype=np.uint8)
    assert int(meta[:8].view(np.uint64)[0]) == idx.info()["entry"]
