"""The allocation-free entry point, vann_medoid_noalloc, called through the C ABI.

It serves callers that cannot call cudaMalloc: a process whose device memory is
owned by another allocator under a fixed budget (a host application that reserved
the GPU's memory up front), a thread on a latency-critical path where cudaMalloc
and cudaFree would synchronise the device, and code that must not meet an
allocation failure at call time.  Its scratch is a fixed array inside libvann.so.
The test checks two calls in a row against the medoid that vann_build chose for
the same vectors (the existing path, which allocates its scratch), against the
CPU oracle, on integer and on float rows, and that the calls leave the device's
free memory unchanged.  This file is collected last on purpose.
"""
import ctypes

import numpy as np
import pytest

from vann import workload

pytestmark = pytest.mark.gpu


def _call(lib, d_vecs, n, dim, out, stream):
    return lib.vann_medoid_noalloc(ctypes.c_void_p(d_vecs.data_ptr()), n, dim, ctypes.c_void_p(out.data_ptr()),
                                   stream)


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
    out = torch.full((1,), -1, dtype=torch.int32, device="cuda")
    for _ in range(2):  # the shared scratch keeps the previous call's contents
        out.fill_(-1)
        st = _call(L, d_base, 5000, 128, out, stream)
        assert st == vann_mod.OK, L.vann_last_error()
        torch.cuda.synchronize()
        assert int(out.item()) == expected
    # a different input right after gives its own medoid
    other = workload.mixture(3000, 64, 10, seed=78)
    d_other = torch.from_numpy(other).cuda()
    assert _call(L, d_other, 3000, 64, out, stream) == vann_mod.OK
    torch.cuda.synchronize()
    assert int(out.item()) == oracle.medoid(other)
    # beyond the fixed scratch the call is rejected, with a message
    assert _call(L, d_base, 1, 4100, out, stream) == vann_mod.ERR_UNSUPPORTED
    assert b"4096" in L.vann_last_error()


def test_medoid_noalloc_float_rows_and_no_allocation(vann_mod):
    """Float rows: the column sums are exact fixed-point integer sums, so the medoid is
    the same on every call and equals vann_build's; it is the FP64 argmin to within
    rounding.  Repeated calls change neither the device's free memory nor torch's."""
    import torch

    L = vann_mod.lib()
    n, dim = 20000, 96
    base = workload.mixture(n, dim, 40, seed=79, sigma=0.05, integer=False, unit_norm=True)
    d_base = torch.from_numpy(base).cuda()
    idx = vann_mod.Index(dim, 32, 32, 1.2, capacity=n)
    idx.build(d_base, batch=0, seed=3)
    expected = idx.info()["entry"]
    del idx
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    out = torch.full((1,), -1, dtype=torch.int32, device="cuda")
    assert _call(L, d_base, n, dim, out, stream) == vann_mod.OK  # first call: module and set-up
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    reserved0 = torch.cuda.memory_reserved()
    got = []
    for _ in range(3):
        out.fill_(-1)
        assert _call(L, d_base, n, dim, out, stream) == vann_mod.OK, L.vann_last_error()
        torch.cuda.synchronize()
        got.append(int(out.item()))
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0 and torch.cuda.memory_reserved() == reserved0
    assert got == [expected] * 3
    x = base.astype(np.float64)
    d = ((x - x.mean(0)) ** 2).sum(1)
    assert d[expected] <= d.min() * (1 + 1e-12)
