"""The allocation-free entry point, vann_medoid_noalloc, called through the C ABI.

It serves callers that cannot call cudaMalloc -- code running while a stream
is captured into a CUDA graph, processes whose device memory belongs to another
allocator, and latency-bound threads that must not wait on the allocator -- by
keeping its scratch in a fixed device array inside libvann.so.  The test checks
two calls in a row against the medoid that vann_build chose for the same
vectors (the existing path, which allocates its scratch), and against the CPU
oracle.  This file is collected last on purpose.
"""
import ctypes

import numpy as np
import pytest

from vann import workload

pytestmark = pytest.mark.gpu


def test_medoid_noalloc_matches_build_twice(oracle, vann_mod):
    import torch

    L = vann_mod.lib()
    base = workload.mixture(5000, 128, 25, seed=77)
    d_base = torch.from_numpy(base).cuda()
    idx = vann_mod.Index(128, 32, 32, 1.2, capacity=5000)
    idx.build(d_base, batch=0, seed=3)  # entry = medoid of all 5000 rows
    expected = idx.info()["entry"]
    assert expected == oracle.medoid(base)
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    for _ in range(2):  # the shared scratch keeps the previous call's contents
        out = torch.full((1,), -1, dtype=torch.int32, device="cuda")
        st = L.vann_medoid_noalloc(ctypes.c_void_p(d_base.data_ptr()), 5000, 128,
                                   ctypes.c_void_p(out.data_ptr()), stream)
        assert st == vann_mod.OK, L.vann_last_error()
        torch.cuda.synchronize()
        assert int(out.item()) == expected
    # a different input right after gives its own medoid
    other = workload.mixture(3000, 64, 10, seed=78)
    d_other = torch.from_numpy(other).cuda()
    out = torch.full((1,), -1, dtype=torch.int32, device="cuda")
    assert L.vann_medoid_noalloc(ctypes.c_void_p(d_other.data_ptr()), 3000, 64,
                                 ctypes.c_void_p(out.data_ptr()), stream) == vann_mod.OK
    torch.cuda.synchronize()
    assert int(out.item()) == oracle.medoid(other)
    # beyond the fixed scratch the call is rejected, with a message
    assert L.vann_medoid_noalloc(ctypes.c_void_p(d_base.data_ptr()), 1, 4100,
                                 ctypes.c_void_p(out.data_ptr()), stream) == vann_mod.ERR_UNSUPPORTED
    assert b"4096" in L.vann_last_error()
