"""Fast (hierarchical) winding numbers on the B200 vs the host evaluator.

Both sides run the same tree, the same moments and the same traversal order;
they differ only in CUDA's vs the C library's atan2 and in the rounding of
fused multiply-adds, so the bar is 1e-12. Accuracy against the exact winding
number is checked on the c3 mesh (327,680 faces) against the plain FP64 kernel
(itself parity-pinned to the reference arithmetic): max 1e-2 at beta = 2.
"""

import ctypes

import numpy as np
import pytest

import igl

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n", [1000, 65536])  # input order, Morton order
def test_gpu_matches_host_evaluator(gpu_required, n):
    V, F, O, _ = igl.synthetic.workload("c2_open", n_queries=n)
    fwn = igl.FastWindingNumber(V, F)
    for beta in (1.0, 2.0, 4.0):
        host = fwn.evaluate(O, beta=beta)
        gpu = fwn.evaluate(O, device="gpu", beta=beta)
        assert np.abs(gpu - host).max() <= 1e-12
    fwn.close()


def test_device_entry_point_and_repeatability(gpu_required):
    import torch

    V, F, O, _ = igl.synthetic.workload("c2_open", n_queries=50_000)
    fwn = igl.FastWindingNumber(V, F)
    Ot = torch.from_numpy(O).cuda()
    a = fwn.evaluate_torch(Ot)
    b = fwn.evaluate_torch(Ot)
    torch.cuda.synchronize()
    assert torch.equal(a, b)
    assert np.array_equal(a.cpu().numpy(), fwn.evaluate(O, device="gpu"))
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    assert igl.lib().wn_stream_check(stream) == 0
    fwn.close()


def test_accuracy_against_exact_fp64_at_327k_faces(gpu_required):
    import torch

    from igl import autograd as wa

    V, F, O, _ = igl.synthetic.workload("c3_mixed", n_queries=65536)
    fwn = igl.FastWindingNumber(V, F)
    Ot = torch.from_numpy(O).cuda()
    tri, ld, nf = wa.triangle_soa(torch.from_numpy(V).cuda(), torch.from_numpy(F).cuda())
    exact = wa.forward_fp64(tri, ld, nf, Ot)
    for beta, bound in ((2.0, 1e-2), (4.0, 1e-3)):
        err = (fwn.evaluate_torch(Ot, beta=beta) - exact).abs().max().item()
        assert err <= bound, (beta, err)
    fwn.close()


def test_empty_inputs(gpu_required):
    V, F, O, _ = igl.synthetic.workload("c1_cpu", n_queries=10)
    assert igl.fast_winding_number(V, F, np.zeros((0, 3)), device="gpu").shape == (0,)
    w = igl.fast_winding_number(V, np.zeros((0, 3), np.int64), O, device="gpu")
    assert np.array_equal(w, np.zeros(10))


def test_gpu_matches_host_on_a_degenerate_soup(gpu_required):
    from test_fwn import _degenerate_soup

    V, F, O = _degenerate_soup()
    fwn = igl.FastWindingNumber(V, F)
    for beta in (1.0, 2.0, 1e9):  # the same tree on both sides: beta = 1 included
        assert np.abs(fwn.evaluate(O, device="gpu", beta=beta)
                      - fwn.evaluate(O, beta=beta)).max() <= 1e-12
    fwn.close()
