"""Per-vertex normals on the B200 vs the reference-generated fixtures and the
host path: bit-identical for uniform and area weights (the same separately
rounded arithmetic, summed per vertex in the reference's face order), within
1e-14 for angle weights (CUDA's acos vs the C library's)."""

import glob
import os

import numpy as np
import pytest

import igl
from conftest import GOLDEN

pytestmark = pytest.mark.gpu

CASES = sorted(os.path.basename(p)[8:-4] for p in glob.glob(os.path.join(GOLDEN, "normals_*.npz")))


def _same(actual, expected, weighting):
    if weighting == 2:
        return np.abs(actual - expected).max() <= 1e-14
    return actual.tobytes() == expected.tobytes()


@pytest.mark.parametrize("name", CASES)
@pytest.mark.parametrize("weighting", [0, 1, 2, 3])
def test_golden(gpu_required, name, weighting):
    g = np.load(os.path.join(GOLDEN, f"normals_{name}.npz"))
    actual = igl.per_vertex_normals(g["V"], g["F"], weighting, device="gpu")
    assert _same(actual, g[f"N{weighting}"], weighting)


def test_large_soup_matches_host(gpu_required):
    V, F = igl.synthetic.bumpy_icosphere(7, seed=31)
    degenerate = [[5, 5, 9], [7, 7, 7]]
    # Flipped copies cancel their originals exactly; bit-identical sums still agree.
    soup = np.concatenate([F, F[:1000, [0, 2, 1]], degenerate])
    for weighting in (0, 1):
        host = igl.per_vertex_normals(V, soup, weighting)
        assert _same(igl.per_vertex_normals(V, soup, weighting, device="gpu"), host, weighting)
    # Angle weights differ in the last bit of acos, so they are compared where the
    # sums do not cancel: normalising a cancelled sum's rounding residue would turn
    # that last bit into an arbitrary direction.
    closed = np.concatenate([F, degenerate])
    host = igl.per_vertex_normals(V, closed, 2)
    assert _same(igl.per_vertex_normals(V, closed, 2, device="gpu"), host, 2)


def test_device_topology_reused_for_new_positions(gpu_required):
    import torch

    from igl import normals

    V, F = igl.synthetic.bumpy_icosphere(5, seed=3)
    dn = normals.DeviceNormals(F, len(V))
    for step in range(3):
        Vs = V * (1.0 + 0.1 * step) + 0.01 * step
        got = dn.evaluate(torch.from_numpy(Vs).cuda(), 1)
        torch.cuda.synchronize()
        assert got.cpu().numpy().tobytes() == igl.per_vertex_normals(Vs, F, 1).tobytes()
    dn.close()


def test_unreferenced_vertices_and_empty_faces(gpu_required):
    V, F = igl.synthetic.bumpy_icosphere(2, seed=4)
    V = np.concatenate([V, [[9.0, 9.0, 9.0], [8.0, 8.0, 8.0]]])
    N = igl.per_vertex_normals(V, F, device="gpu")
    assert np.array_equal(N[-2:], np.zeros((2, 3)))
    assert N.tobytes() == igl.per_vertex_normals(V, F).tobytes()
    assert np.array_equal(igl.per_vertex_normals(V, np.zeros((0, 3), np.int64), device="gpu"),
                          np.zeros_like(V))


def test_out_of_range_faces_rejected_on_the_device(gpu_required):
    """The C entry checks F on the device: out-of-range indices give WN_EINVAL, no access."""
    import ctypes

    V, F = igl.synthetic.bumpy_icosphere(2, seed=4)
    bad = F.copy()
    bad[7, 1] = len(V)
    bad[9, 2] = -3
    N = np.zeros_like(V)
    lib = igl.lib()
    assert lib.wn_vertex_normals_host(V.ctypes.data, len(V), bad.ctypes.data, len(bad), 1,
                                      N.ctypes.data) == 1
    assert "2 face indices outside V" in igl._lib.last_error()
    handle = ctypes.c_void_p()
    assert lib.wn_normals_create(bad.ctypes.data, len(bad), len(V), None, ctypes.byref(handle)) == 1
    # The library keeps working afterwards.
    assert igl.per_vertex_normals(V, F, device="gpu").tobytes() == igl.per_vertex_normals(V, F).tobytes()


def test_unaligned_positions_and_long_incidence_lists(gpu_required):
    """Positions that start 8 bytes past a 16-byte boundary (a tensor view), and a
    vertex on 300 faces (its list spans several of the gather's chunks, and the
    lists of the vertices around it start and end inside them)."""
    import torch

    from igl import normals

    V, F = igl.synthetic.bumpy_icosphere(4, seed=8)
    nv0 = len(V)
    ring = 300
    t = np.linspace(0.0, 2.0 * np.pi, ring, endpoint=False)
    fan_v = np.concatenate([[[0.0, 0.0, 3.0]],
                            np.stack([np.cos(t), np.sin(t), 3.0 + 0.1 * np.sin(3 * t)], 1)])
    fan_f = np.stack([np.zeros(ring, np.int64), 1 + np.arange(ring),
                      1 + (np.arange(ring) + 1) % ring], 1) + nv0
    V = np.concatenate([V, fan_v])
    F = np.concatenate([F[: len(F) // 2], fan_f, F[len(F) // 2:]])
    nv = len(V)
    buf = torch.zeros(3 * nv + 1, dtype=torch.float64, device="cuda")
    view = buf[1:].view(nv, 3)
    view.copy_(torch.from_numpy(V))
    assert view.data_ptr() % 16 == 8
    dn = normals.DeviceNormals(F, nv)
    for weighting in (0, 1, 2):
        got = dn.evaluate(view, weighting)
        torch.cuda.synchronize()
        assert _same(got.cpu().numpy(), igl.per_vertex_normals(V, F, weighting), weighting)
    dn.close()
