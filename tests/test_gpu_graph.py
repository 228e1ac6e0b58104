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
