"""Full-size checks through size-independent properties (B200).

At the configurations' full sizes the oracle is too slow, so the plain FP64
kernel (pinned to the oracle at <= 1e-12 elsewhere) is the reference, and
properties that hold at any size are checked: mixed vs FP64 <= 1e-6 on every
query, closed-mesh integrality for queries away from the surface, and
agreement of the two FP64 kernels.
"""

import numpy as np
import pytest

import igl
from igl import autograd as wa

pytestmark = pytest.mark.gpu


def _run(name, n_queries=None):
    import torch

    V, F, O, _ = igl.synthetic.workload(name, n_queries=n_queries)
    Vt, Ft, Ot = (torch.from_numpy(x).cuda() for x in (V, F, O))
    tri, ld, nf = wa.triangle_soa(Vt, Ft)
    mesh = wa.PreparedMesh(tri, ld, nf)
    try:
        w_mixed = mesh.forward(Ot).cpu().numpy()
        w_stream = wa.forward_fp64(tri, ld, nf, Ot).cpu().numpy()
        import ctypes

        from igl import _lib

        w_tiled = torch.empty(len(O), dtype=torch.float64, device="cuda")
        rc = _lib.lib().wn_forward_fp64_mesh_device(
            mesh.mesh, Ot.data_ptr(), len(O), w_tiled.data_ptr(),
            ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
        assert rc == 0, _lib.last_error()
        return V, F, O, w_mixed, w_stream, w_tiled.cpu().numpy()
    finally:
        mesh.close()


def test_c2_open_full_size(gpu_required):
    V, F, O, wm, ws, wt = _run("c2_open")  # 18,842 F x 2^20 Q
    assert np.abs(ws - wt).max() <= 1e-12
    assert np.abs(wm - ws).max() <= 1e-6
    assert np.isfinite(wm).all()


def test_c3_closed_full_size_properties(gpu_required):
    V, F, O, wm, ws, wt = _run("c3_mixed", n_queries=1 << 18)  # 327,680 F x 262,144 Q
    assert np.abs(ws - wt).max() <= 1e-12
    assert np.abs(wm - ws).max() <= 1e-6
    # Closed mesh: W is 0 or 1 off the surface (box half of the queries).
    box = wm[: len(O) // 2]
    assert np.abs(box - np.round(box)).max() <= 1e-6
    assert set(np.unique(np.round(box))) <= {0.0, 1.0}
