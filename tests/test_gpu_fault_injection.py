"""Out-of-memory paths on a real device, by host-side fault injection (B200).

``wn_inject_fault(WN_FAULT_ALLOC, k)`` makes the (k+1)-th device allocation of
the library report failure without allocating. Each test runs one public call
with k = 0, 1, 2, ... until the call gets past its last allocation: every
faulted call must raise RuntimeError and leave the fault consumed, nothing
may fail afterwards on the stream, and the first call that completes must
return exactly what the call returned before the sweep. Every entry point
returns before launching work that needs a failed allocation, so nothing on
the device runs differently; no test faults, traps or hangs a GPU.
"""

import numpy as np
import pytest
import torch

import igl
from igl import _lib
from igl import autograd as wa

pytestmark = pytest.mark.gpu
WN_FAULT_NONE, WN_FAULT_ALLOC = 0, 1


@pytest.fixture
def lib(gpu_required):
    handle = _lib.lib()
    yield handle
    handle.wn_inject_fault(WN_FAULT_NONE, 0)


def _same(a, b):
    if isinstance(a, (tuple, list)):
        assert len(a) == len(b)
        for x, y in zip(a, b):
            _same(x, y)
    elif isinstance(a, torch.Tensor):
        assert torch.equal(a, b)
    else:
        assert np.array_equal(np.asarray(a), np.asarray(b))


def _sweep(lib, call, message="out of memory", limit=128):
    """Faults each allocation of call() in turn; returns how many it made."""
    expected = call()
    torch.cuda.synchronize()
    for k in range(limit):
        assert lib.wn_inject_fault(WN_FAULT_ALLOC, k) == 0
        try:
            got = call()
        except RuntimeError as err:
            assert lib.wn_fault_armed() == 0, f"failed with the fault still armed: {err}"
            assert message in str(err)
            torch.cuda.synchronize()
            continue
        torch.cuda.synchronize()
        armed = lib.wn_fault_armed()
        lib.wn_inject_fault(WN_FAULT_NONE, 0)
        assert armed == 1, f"allocation {k} failed but the call reported success"
        _same(expected, got)
        return k
    raise AssertionError("more allocations than the sweep limit")


def _open_mesh(level=3, n=3000, seed=5):
    V, F = igl.synthetic.bumpy_icosphere(level, seed=seed)
    F = igl.synthetic.delete_faces(F, 0.08, seed=seed + 1)
    O = igl.synthetic.mixed_queries(V, F, n, seed=seed + 2, near_sigma=1e-3)
    return V, F, O


def test_injection_arms_and_disarms(lib):
    assert lib.wn_inject_fault(WN_FAULT_ALLOC, 3) == 0
    assert lib.wn_fault_armed() == 1
    assert lib.wn_inject_fault(WN_FAULT_NONE, 0) == 0
    assert lib.wn_fault_armed() == 0


def test_prepared_mesh_forward_and_backward(lib):
    V, F, O = _open_mesh()
    Vt, Ft, Ot = (torch.from_numpy(x).cuda() for x in (V, F, O))
    tri, ld, nf = wa.triangle_soa(Vt, Ft)
    g = torch.from_numpy(np.random.default_rng(3).normal(size=len(O))).cuda()

    def call():
        mesh = wa.PreparedMesh(tri, ld, nf)
        try:
            w = mesh.forward(Ot)
            dq, dtri = mesh.backward(Ot, g)
            return w, dq, dtri
        finally:
            mesh.close()

    assert _sweep(lib, call) >= 6  # 4 mesh arrays + preparation, forward and adjoint scratch


def test_fp64_forward_with_face_split(lib):
    V, F, O = _open_mesh(level=5, n=512)  # few queries: the face range is split (scratch)
    Vt, Ft, Ot = (torch.from_numpy(x).cuda() for x in (V, F, O))
    tri, ld, nf = wa.triangle_soa(Vt, Ft)
    assert _sweep(lib, lambda: wa.forward_fp64(tri, ld, nf, Ot)) >= 1


def test_boundary_edge_and_face_adjoints(lib):
    V, F, O = _open_mesh()
    Vt, Ft, Ot = (torch.from_numpy(x).cuda() for x in (V, F, O))
    g = torch.from_numpy(np.random.default_rng(4).normal(size=len(O))).cuda()
    assert _sweep(lib, lambda: wa.backward_edges(Vt, Ft, Ot, g)) >= 1
    tri, ld, nf = wa.triangle_soa(Vt, Ft)
    assert _sweep(lib, lambda: wa.backward_fp64(tri, ld, nf, Ot, g, Ft, len(V))) >= 1


def test_batch_create_forward_backward(lib):
    meshes, queries = [], []
    for i, level in enumerate((1, 2, 3)):
        V, F, O = _open_mesh(level=level, n=700 + 300 * i, seed=20 + i)
        meshes.append((V, F))
        queries.append(O)

    def call():
        batch = igl.batched.Batch(meshes, queries)
        try:
            w = batch.forward().clone()
            dv, dq = batch.backward(torch.ones_like(batch.W))
            return w, dv.clone(), dq.clone()
        finally:
            batch.close()

    assert _sweep(lib, call) >= 30


def test_closest_point_and_signed_distance(lib):
    V, F, O = _open_mesh()
    Ot = torch.from_numpy(O).cuda()

    def call():
        tree = igl.distance.DeviceAABB(V, F)
        try:
            out = list(tree.query(Ot))
            for precision in ("fp64", "mixed", "fast"):
                out += [x.clone() for x in tree.signed_distance(Ot, precision=precision)]
            return out
        finally:
            tree.close()

    assert _sweep(lib, call) >= 4


def test_fast_winding_number(lib):
    V, F, O = _open_mesh()
    Ot = torch.from_numpy(O).cuda()

    def call():
        fwn = igl.FastWindingNumber(V, F)
        try:
            return fwn.evaluate_torch(Ot), fwn.evaluate(O, device="gpu")
        finally:
            torch.cuda.synchronize()
            fwn.close()

    assert _sweep(lib, call, message="") >= 3  # the tree upload's three arrays


def test_vertex_normals(lib):
    V, F, _ = _open_mesh()
    Vt = torch.from_numpy(V).cuda()

    def call():
        normals = igl.normals.DeviceNormals(F, len(V))
        try:
            return [normals.evaluate(Vt, weighting=w) for w in (0, 1, 2)]
        finally:
            normals.close()

    assert _sweep(lib, call) >= 4  # topology arrays, build scratch, contributions


def test_drop_in_winding_number_raises_and_recovers(lib, oracle_mod):
    """A failed allocation in the drop-in's GPU call raises the reference's
    RuntimeError mentioning the GPU; the next call works."""
    V, F = igl.synthetic.bumpy_icosphere(1, seed=2)
    O = np.random.default_rng(9).uniform(-1.5, 1.5, size=(1 << 22, 3))  # grows the host buffers
    assert lib.wn_inject_fault(WN_FAULT_ALLOC, 0) == 0
    with pytest.raises(RuntimeError, match="GPU"):
        igl.winding_number(V, F, O, device="gpu")
    assert lib.wn_fault_armed() == 0
    W = igl.winding_number(V, F, O[:4096], device="gpu")
    assert np.abs(W - oracle_mod.winding_number(V, F, O[:4096])).max() <= 1e-12
