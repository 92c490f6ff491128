"""Failure detection on the GPU without a fault (B200).

Every wait in the kernels is bounded; when one runs out the kernel sets a bit
in a device error word and returns, and the host call reports WN_EDEVICE. The
self-test makes a wait run out on purpose (a phase nothing completes, a short
poll limit) and checks that the status comes back and the context still works.
"""

import numpy as np
import pytest

import igl
from igl import _lib

pytestmark = pytest.mark.gpu
WN_EDEVICE = 4


def test_bounded_wait_reports_timeout_and_context_survives(gpu_required, oracle_mod):
    h = _lib.lib()
    assert h.wn_selftest_bounded_wait(1000) == WN_EDEVICE
    assert "bounded wait" in _lib.last_error()
    # The error word was cleared and the context is usable.
    V, F, O, _ = igl.synthetic.workload("c1_cpu", n_queries=256)
    W = igl.winding_number(V, F, O, device="gpu")
    assert np.abs(W - oracle_mod.winding_number(V, F, O)).max() <= 1e-12
    assert h.wn_selftest_bounded_wait(0) != 0  # argument check, nothing launched


def test_kernel_failure_surfaces_as_runtime_error(gpu_required, monkeypatch):
    """The drop-in raises on a failed GPU call; it never retries on the CPU."""
    V, F = igl.synthetic.bumpy_icosphere(1, seed=1)
    handle = _lib.lib()

    class Failing:
        def __getattr__(self, name):
            return getattr(handle, name)

        @staticmethod
        def mli_winding_gpu(*args):
            return 0

    monkeypatch.setattr(igl, "lib", lambda: Failing())
    with pytest.raises(RuntimeError, match="GPU"):
        igl.winding_number(V, F, [[0.0, 0.0, 0.0]], device="gpu")


def test_sizes_beyond_the_limits_are_refused_before_any_work(gpu_required, oracle_mod):
    """Counts past the 32-bit limits of the grids and index types come back as
    errors (small real buffers stand behind every pointer; none is read past
    its end, and nothing is launched), and the device keeps working."""
    import ctypes

    import torch

    from igl import autograd as wa
    from igl import distance

    h = _lib.lib()
    big = 1 << 31
    V, F, O, _ = igl.synthetic.workload("c1_cpu", n_queries=64)
    Vt, Ft, Ot = (torch.from_numpy(x).cuda() for x in (V, F, O))
    tri, ld, nf = wa.triangle_soa(Vt, Ft)
    w = torch.empty(64, dtype=torch.float64, device="cuda")
    sp = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    mesh = wa.PreparedMesh(tri, ld, nf)
    tree = distance.DeviceAABB(V, F)
    fwn = igl.FastWindingNumber(V, F)
    try:
        perm = torch.empty(64, dtype=torch.int32, device="cuda")
        idx = torch.empty(64, dtype=torch.int64, device="cuda")
        pts = torch.empty((64, 3), dtype=torch.float64, device="cuda")
        assert h.wn_forward_mixed_device(mesh.mesh, Ot.data_ptr(), big, w.data_ptr(), sp) != 0
        assert h.wn_mixed_sort_queries(Ot.data_ptr(), big, perm.data_ptr(), sp) != 0
        assert h.wn_forward_fp64_device(tri.data_ptr(), ld, Ot.data_ptr(), w.data_ptr(), nf,
                                        1 << 40, 0, sp) != 0
        assert h.wn_aabb_squared_distance_device(tree.tree, Ot.data_ptr(), big, w.data_ptr(),
                                                 idx.data_ptr(), pts.data_ptr(), sp) != 0
        assert h.wn_fast_eval_device(fwn._handle, Ot.data_ptr(), big, 2.0, w.data_ptr(), sp) != 0
        out = ctypes.c_void_p()
        assert h.wn_mixed_mesh_create(tri.data_ptr(), big, big, 4.0, sp, ctypes.byref(out)) != 0
        assert not out
        Fh = np.ascontiguousarray(F)
        assert h.wn_normals_create(Fh.ctypes.data, big, len(V), sp, ctypes.byref(out)) != 0
        assert not out
        torch.cuda.synchronize()
        assert h.wn_stream_check(sp) == 0
        W = igl.winding_number(V, F, O, device="gpu")
        assert np.abs(W - oracle_mod.winding_number(V, F, O)).max() <= 1e-12
    finally:
        fwn.close()
        tree.close()
        mesh.close()
