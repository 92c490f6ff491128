"""wn_forward_fp64_device_noalloc: the FP64 forward without any GPU allocation.

For callers that own all device memory (an application's own pool or fixed
budget) and may not let a library call cudaMalloc: the entry point keeps its
face-split scratch in a fixed array inside the library. These tests call it
through the C ABI, twice in a row on the same inputs, and compare each result
with the allocating entry point wn_forward_fp64_device at the FP64 parity
tolerance (1e-12); they also check that query counts beyond its limit
(2^19) are refused, that a call succeeds while the library's next device
allocation is set to fail (it makes none), and that a stream under capture is
refused without ending the caller's capture (the call waits for its stream).
This file sorts last so a stop-at-first-failure run has already run every
other test.
"""

import ctypes

import numpy as np
import pytest

import igl
from igl import _lib

pytestmark = pytest.mark.gpu
TOL = 1e-12
MAX_QUERIES = 1 << 19


def _noalloc(handle):
    fn = handle.wn_forward_fp64_device_noalloc
    fn.argtypes = [ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p, ctypes.c_void_p,
                   ctypes.c_int64, ctypes.c_int64, ctypes.c_int, ctypes.c_void_p]
    fn.restype = ctypes.c_int
    return fn


def _device_soup(torch, V, F):
    tri = igl._triangle_soa(V, F)
    nf = tri.shape[1]
    ld = nf + (nf & 1)
    tri_d = torch.zeros((9, ld), dtype=torch.float64, device="cuda")
    tri_d[:, :nf] = torch.from_numpy(tri)
    return tri_d, ld, nf


@pytest.mark.parametrize("nq", [1, 1000, 40000])
@pytest.mark.parametrize("mode", [0, 1])
def test_noalloc_matches_allocating_entry_twice(gpu_required, nq, mode):
    import torch

    handle = _lib.lib()
    noalloc = _noalloc(handle)
    V, F, O, _ = igl.synthetic.workload("c2_open", n_queries=nq)
    tri_d, ld, nf = _device_soup(torch, V, F)
    q_d = torch.from_numpy(O).cuda()
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    expected = torch.empty(nq, dtype=torch.float64, device="cuda")
    rc = handle.wn_forward_fp64_device(tri_d.data_ptr(), ld, q_d.data_ptr(),
                                       expected.data_ptr(), nf, nq, mode, stream)
    assert rc == 0, _lib.last_error()
    assert handle.wn_stream_check(stream) == 0
    for _ in range(2):  # the shared array keeps the previous call's contents
        got = torch.full((nq,), float("nan"), dtype=torch.float64, device="cuda")
        rc = noalloc(tri_d.data_ptr(), ld, q_d.data_ptr(), got.data_ptr(), nf, nq, mode, stream)
        assert rc == 0, _lib.last_error()
        assert torch.isfinite(got).all()
        assert float((got - expected).abs().max()) <= TOL


def test_noalloc_refuses_more_than_its_limit(gpu_required):
    import torch

    handle = _lib.lib()
    noalloc = _noalloc(handle)
    V, F = igl.synthetic.bumpy_icosphere(1, seed=1)
    tri_d, ld, nf = _device_soup(torch, V, F)
    nq = MAX_QUERIES + 1
    q_d = torch.zeros((nq, 3), dtype=torch.float64, device="cuda")
    w_d = torch.empty(nq, dtype=torch.float64, device="cuda")
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    rc = noalloc(tri_d.data_ptr(), ld, q_d.data_ptr(), w_d.data_ptr(), nf, nq, 0, stream)
    assert rc != 0
    assert "524288" in _lib.last_error()


def test_noalloc_makes_no_device_allocation(gpu_required):
    """With the library's next device allocation armed to fail, the call still
    succeeds and leaves the fault armed: it allocated nothing."""
    import torch

    handle = _lib.lib()
    noalloc = _noalloc(handle)
    V, F, O, _ = igl.synthetic.workload("c2_open", n_queries=3000)
    tri_d, ld, nf = _device_soup(torch, V, F)
    q_d = torch.from_numpy(O).cuda()
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    expected = torch.empty(len(O), dtype=torch.float64, device="cuda")
    assert handle.wn_forward_fp64_device(tri_d.data_ptr(), ld, q_d.data_ptr(),
                                         expected.data_ptr(), nf, len(O), 0, stream) == 0
    got = torch.empty_like(expected)
    assert handle.wn_inject_fault(1, 0) == 0  # WN_FAULT_ALLOC: the next allocation fails
    try:
        rc = noalloc(tri_d.data_ptr(), ld, q_d.data_ptr(), got.data_ptr(), nf, len(O), 0, stream)
        assert rc == 0, _lib.last_error()
        assert handle.wn_fault_armed() == 1
    finally:
        handle.wn_inject_fault(0, 0)
    assert float((got - expected).abs().max()) <= TOL


def test_noalloc_refuses_a_capturing_stream(gpu_required):
    """The call waits for its stream before returning, so on a stream under
    capture it returns an error before touching the stream; the caller's capture
    stays valid."""
    import torch

    handle = _lib.lib()
    noalloc = _noalloc(handle)
    V, F = igl.synthetic.bumpy_icosphere(1, seed=1)
    tri_d, ld, nf = _device_soup(torch, V, F)
    q_d = torch.zeros((16, 3), dtype=torch.float64, device="cuda")
    w_d = torch.empty(16, dtype=torch.float64, device="cuda")
    x = torch.zeros(8, device="cuda")
    side = torch.cuda.Stream()
    graph = torch.cuda.CUDAGraph()
    torch.cuda.synchronize()
    with torch.cuda.stream(side):
        graph.capture_begin()
        x.add_(1.0)
        rc = noalloc(tri_d.data_ptr(), ld, q_d.data_ptr(), w_d.data_ptr(), nf, 16, 0,
                     ctypes.c_void_p(side.cuda_stream))
        graph.capture_end()
    assert rc != 0
    assert "captured" in _lib.last_error()
    graph.replay()
    torch.cuda.synchronize()
    assert float(x.sum()) == 8.0
