"""vann_search is stream-ordered with no host synchronisation or allocation, so a
batched search can be captured into a CUDA graph and replayed: each replay re-reads
the captured query buffer and gives exactly the direct call's results."""
import numpy as np
import pytest

from vann import workload

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("store,L,rerank,beam", [("u8", 32, False, 1), ("f32", 100, False, 1),
                                                 ("u8", 48, True, 1), ("u8", 40, False, 2)])
def test_captured_search_replays_exactly(vann_mod, store, L, rerank, beam):
    import torch

    base = workload.mixture(5000, 128, 30, seed=131)
    idx = vann_mod.Index(128, 32, 64, 1.2, capacity=5000, stores=("f32", "u8"))
    idx.build(torch.from_numpy(base).cuda(), batch=0, seed=2)
    batches = [torch.from_numpy(workload.mixture(700, 128, 30, seed=132 + i)).cuda() for i in range(3)]
    want = [idx.search(b, k=10, L=L, store=store, rerank=rerank, beam=beam) for b in batches]
    torch.cuda.synchronize()

    q = batches[0].clone()
    out = (torch.empty((700, 10), dtype=torch.int32, device="cuda"),
           torch.empty((700, 10), dtype=torch.float32, device="cuda"))
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s):  # warm the launch configuration outside the capture
        idx.search(q, k=10, L=L, store=store, rerank=rerank, beam=beam, out=out)
    torch.cuda.current_stream().wait_stream(s)
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        idx.search(q, k=10, L=L, store=store, rerank=rerank, beam=beam, out=out)
    for i, b in enumerate(batches):
        q.copy_(b)
        g.replay()
        torch.cuda.synchronize()
        assert torch.equal(out[0], want[i][0]) and torch.equal(out[1], want[i][1]), i
    del g


def test_captured_large_batches(vann_mod):
    """Batches above 16 queries per SM use the order workspace.  Captured without an
    uncaptured call on the capture stream first, the search allocates nothing and runs
    in input order; after a warm-up on that stream it captures the ordered search.  A
    later, larger uncaptured search on the same stream grows the workspace without
    freeing the one the graph holds.  Every replay equals the direct call."""
    import torch

    nsm = torch.cuda.get_device_properties(0).multi_processor_count
    nq = 16 * nsm + 700
    base = workload.mixture(5000, 128, 30, seed=141)
    idx = vann_mod.Index(128, 32, 64, 1.2, capacity=5000, stores=("f32", "u8"))
    idx.build(torch.from_numpy(base).cuda(), batch=0, seed=2)
    batches = [torch.from_numpy(workload.mixture(nq, 128, 30, seed=142 + i)).cuda() for i in range(2)]
    want = [idx.search(b, k=10, L=32, store="u8") for b in batches]
    torch.cuda.synchronize()
    q = batches[0].clone()
    out = (torch.empty((nq, 10), dtype=torch.int32, device="cuda"),
           torch.empty((nq, 10), dtype=torch.float32, device="cuda"))
    big = torch.from_numpy(workload.mixture(4 * nq, 128, 30, seed=149)).cuda()
    graphs = []
    for warm in (False, True):
        s = torch.cuda.Stream()
        s.wait_stream(torch.cuda.current_stream())
        if warm:
            with torch.cuda.stream(s):
                idx.search(q, k=10, L=32, store="u8", out=out)
        torch.cuda.current_stream().wait_stream(s)
        torch.cuda.synchronize()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=s):
            idx.search(q, k=10, L=32, store="u8", out=out)
        with torch.cuda.stream(s):
            idx.search(big, k=10, L=32, store="u8")  # grows this stream's workspace
        torch.cuda.synchronize()
        graphs.append(g)
    for g in graphs:
        for i, b in enumerate(batches):
            q.copy_(b)
            g.replay()
            torch.cuda.synchronize()
            assert torch.equal(out[0], want[i][0]) and torch.equal(out[1], want[i][1]), i
    del graphs


@pytest.mark.parametrize("rerank", [True, False])
def test_captured_search_on_the_uint8_grid(vann_mod, rerank):
    """Float rows searched from their uint8 copy (fitted grid): the query mapping, the
    search and the rerank (or distance scaling) are captured together after one call on
    the capture stream; every replay equals the direct call.  Captured on a stream that
    has not searched yet, the call fails with VANN_ERR_STATE instead of allocating."""
    import torch

    D = 96
    base = workload.mixture(5000, D, 30, seed=151, sigma=0.05, integer=False, unit_norm=True)
    idx = vann_mod.Index(D, 32, 64, 1.2, capacity=5000, stores=("f32", "u8"))
    idx.build(torch.from_numpy(base).cuda(), batch=0, seed=2)
    batches = [torch.from_numpy(workload.mixture(700, D, 30, seed=152 + i, sigma=0.05, integer=False,
                                                 unit_norm=True)).cuda() for i in range(3)]
    want = [idx.search(b, k=10, L=48, store="u8", rerank=rerank) for b in batches]
    torch.cuda.synchronize()
    q = batches[0].clone()
    out = (torch.empty((700, 10), dtype=torch.int32, device="cuda"),
           torch.empty((700, 10), dtype=torch.float32, device="cuda"))
    cold = torch.cuda.Stream()
    cold.wait_stream(torch.cuda.current_stream())
    g0 = torch.cuda.CUDAGraph()
    with pytest.raises(vann_mod.VannError) as e:
        with torch.cuda.graph(g0, stream=cold):
            idx.search(q, k=10, L=48, store="u8", rerank=rerank, out=out)
    assert e.value.status == vann_mod.ERR_STATE
    del g0
    torch.cuda.synchronize()
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s):
        idx.search(q, k=10, L=48, store="u8", rerank=rerank, out=out)
    torch.cuda.current_stream().wait_stream(s)
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=s):
        idx.search(q, k=10, L=48, store="u8", rerank=rerank, out=out)
    for i, b in enumerate(batches):
        q.copy_(b)
        g.replay()
        torch.cuda.synchronize()
        assert torch.equal(out[0], want[i][0]) and torch.equal(out[1], want[i][1]), i
    del g
