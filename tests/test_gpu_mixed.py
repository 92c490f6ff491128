"""Mixed-precision GPU kernel: FP32 pairs + FP64 refinement (needs a B200).

Bar: max |W_mixed - W_oracle| <= 1e-6 per query (the target error of the
mixed form), on the reference's cases, seeded open and closed meshes, edge
cases (queries on vertices, edges and inside faces; collapsed faces; tiny and
huge coordinate scales; queries very far away), and the FP64 refinement must
actually run for near-surface queries.
"""

import ctypes

import numpy as np
import pytest

import igl
from igl import _lib
from conftest import GOLDEN_CASES, load_golden, tetrahedron

pytestmark = pytest.mark.gpu
TOL = 1e-6


def mixed_host(tri, O, kappa=4.0):
    tri = np.ascontiguousarray(tri, dtype=np.float64)
    O = np.ascontiguousarray(O, dtype=np.float64).reshape(-1, 3)
    out = np.full(len(O), np.nan)
    rc = _lib.lib().wn_forward_mixed_host(tri.ctypes.data, O.ctypes.data, out.ctypes.data,
                                          tri.shape[1], len(O), kappa)
    assert rc == 0, _lib.last_error()
    return out


def stats(reset=True):
    r, c = ctypes.c_int64(0), ctypes.c_int64(0)
    assert _lib.lib().wn_mixed_stats(ctypes.byref(r), ctypes.byref(c), int(reset)) == 0
    return r.value, c.value


@pytest.mark.parametrize("name", GOLDEN_CASES)
def test_golden_cases(gpu_required, name):
    g = load_golden(name)
    W = mixed_host(igl._triangle_soa(g["V"], g["F"]), g["O"])
    assert np.abs(W - g["W"]).max() <= TOL


def test_public_api_mixed(gpu_required):
    V, F = tetrahedron()
    Q = np.array([[0.1, 0.1, 0.1], [2.0, 2.0, 2.0]])
    W = igl.winding_number(V, F, Q, device="gpu", precision="mixed")
    assert abs(W[0] - 1.0) <= TOL and abs(W[1]) <= TOL


@pytest.mark.parametrize("kappa", [3.0, 4.0, 8.0])
def test_open_mesh_c2_subset(gpu_required, oracle_mod, kappa):
    V, F, O, _ = igl.synthetic.workload("c2_open", n_queries=4096)
    tri = igl._triangle_soa(V, F)
    ref = oracle_mod.winding_soa(tri, O, workers=8)
    stats()
    W = mixed_host(tri, O, kappa)
    refined, careful = stats()
    err = np.abs(W - ref)
    assert err.max() <= TOL, (kappa, err.max())
    assert refined > 0 and careful > 0


def test_closed_mesh_c1(gpu_required, oracle_mod):
    V, F, O, _ = igl.synthetic.workload("c1_cpu")
    tri = igl._triangle_soa(V, F)
    W = mixed_host(tri, O)
    assert np.abs(W - oracle_mod.winding_soa(tri, O, workers=8)).max() <= TOL
    assert np.abs(W - np.round(W)).max() <= TOL


def test_near_surface_c3_mesh_sample(gpu_required, oracle_mod):
    V, F = igl.synthetic.bumpy_icosphere(7, seed=31)
    O = igl.synthetic.mixed_queries(V, F, 256, seed=99, near_sigma=1e-4)
    tri = igl._triangle_soa(V, F)
    W = mixed_host(tri, O)
    assert np.abs(W - oracle_mod.winding_soa(tri, O, workers=8)).max() <= TOL


def test_degenerate_queries(gpu_required, oracle_mod):
    V, F = igl.synthetic.bumpy_icosphere(3, seed=9)
    tri = igl._triangle_soa(V, F)
    t = V[F]
    Q = np.concatenate([V[:50], 0.5 * (t[:50, 0] + t[:50, 1]),
                        (t[:50, 0] + t[:50, 1] + t[:50, 2]) / 3,
                        [[0.0, 0.0, 0.0], [1e3, 1e3, 1e3], [1e25, -1e25, 3e24]]])
    W = mixed_host(tri, Q)
    assert np.abs(W - oracle_mod.winding_soa(tri, Q)).max() <= TOL


def test_collapsed_and_sliver_faces(gpu_required, oracle_mod):
    rng = np.random.default_rng(5)
    tri = rng.normal(size=(9, 300))
    tri[:, :50] = 0.0
    tri[3:6, 50:100] = tri[0:3, 50:100]
    tri[6:9, 100:150] = 2 * tri[3:6, 100:150] - tri[0:3, 100:150]
    O = rng.normal(size=(300, 3))
    O[0] = 0.0
    O[1] = tri[0:3, 60]
    W = mixed_host(tri, O)
    assert np.abs(W - oracle_mod.winding_soa(tri, O)).max() <= TOL


@pytest.mark.parametrize("scale", [1e-12, 1e-3, 1e3, 1e12])
def test_scale_invariance(gpu_required, oracle_mod, scale):
    V, F = igl.synthetic.bumpy_icosphere(3, seed=4)
    O = igl.synthetic.mixed_queries(V, F, 512, seed=5, near_sigma=1e-3)
    tri = igl._triangle_soa(V * scale, F)
    W = mixed_host(tri, O * scale)
    assert np.abs(W - oracle_mod.winding_soa(tri, O * scale)).max() <= TOL


@pytest.mark.parametrize("nf,nq", [(1, 1), (63, 5), (64, 64), (65, 257), (1000, 1)])
def test_odd_sizes(gpu_required, oracle_mod, nf, nq):
    rng = np.random.default_rng(nf + 31 * nq)
    tri = rng.normal(size=(9, nf))
    O = rng.normal(size=(nq, 3))
    W = mixed_host(tri, O)
    assert np.abs(W - oracle_mod.winding_soa(tri, O)).max() <= TOL


def test_empty_faces_and_queries(gpu_required):
    assert np.array_equal(mixed_host(np.zeros((9, 0)), np.ones((4, 3))), np.zeros(4))
    assert mixed_host(np.zeros((9, 3)), np.zeros((0, 3))).shape == (0,)


def test_kappa_below_bound_is_rejected(gpu_required):
    tri = np.zeros((9, 3))
    O = np.zeros((1, 3))
    out = np.zeros(1)
    rc = _lib.lib().wn_forward_mixed_host(tri.ctypes.data, O.ctypes.data, out.ctypes.data, 3, 1,
                                          2.0)
    assert rc != 0 and "kappa" in _lib.last_error()


def test_device_path_with_prepared_mesh(gpu_required, oracle_mod):
    import torch

    V, F, O, _ = igl.synthetic.workload("c2_open", n_queries=3000)
    tri = igl._triangle_soa(V, F)
    nf = tri.shape[1]
    ld = nf + (nf & 1)
    tri_d = torch.zeros((9, ld), dtype=torch.float64, device="cuda")
    tri_d[:, :nf] = torch.from_numpy(tri)
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    h = _lib.lib()
    mesh = ctypes.c_void_p()
    assert h.wn_mixed_mesh_create(tri_d.data_ptr(), ld, nf, 4.0, stream, ctypes.byref(mesh)) == 0
    try:
        ref = oracle_mod.winding_soa(tri, O, workers=8)
        for chunk in (O[:1000], O):
            q_d = torch.from_numpy(np.ascontiguousarray(chunk)).cuda()
            w_d = torch.empty(len(chunk), dtype=torch.float64, device="cuda")
            assert h.wn_forward_mixed_device(mesh, q_d.data_ptr(), len(chunk), w_d.data_ptr(),
                                             stream) == 0, _lib.last_error()
            assert h.wn_stream_check(stream) == 0
            assert np.abs(w_d.cpu().numpy() - ref[: len(chunk)]).max() <= TOL
    finally:
        h.wn_mixed_mesh_destroy(mesh)


def test_deterministic_repeat(gpu_required):
    V, F, O, _ = igl.synthetic.workload("c2_open", n_queries=2048)
    tri = igl._triangle_soa(V, F)
    a = mixed_host(tri, O)
    assert np.array_equal(mixed_host(tri, O), a)


@pytest.mark.parametrize("offset", [1e2, 1e4, 1e6])
def test_translated_far_from_origin(gpu_required, oracle_mod, offset):
    """A unit-size mesh far from the origin: the FP32 frames are tile-local, so the
    error must not grow with the offset (FP64 tile centres absorb it)."""
    V, F = igl.synthetic.bumpy_icosphere(4, seed=6)
    O = igl.synthetic.mixed_queries(V, F, 1024, seed=7, near_sigma=1e-4)
    t = np.array([offset, -0.7 * offset, 0.3 * offset])
    tri = igl._triangle_soa(V + t, F)
    W = mixed_host(tri, O + t)
    assert np.abs(W - oracle_mod.winding_soa(tri, O + t)).max() <= TOL


def test_random_soup_multiscale(gpu_required, oracle_mod):
    """Self-intersecting soup, triangle sizes log-uniform over four decades, queries
    uniform in the cube and within 1e-5..1e-2 of random faces."""
    rng = np.random.default_rng(8)
    nf = 6000
    centre = rng.uniform(-1, 1, size=(nf, 1, 3))
    size = 10.0 ** rng.uniform(-4, 0, size=(nf, 1, 1))
    corners = centre + size * rng.normal(size=(nf, 3, 3))
    tri = np.ascontiguousarray(corners.transpose(1, 2, 0).reshape(9, nf))
    box = rng.uniform(-1.2, 1.2, size=(1024, 3))
    pick = rng.integers(0, nf, size=1024)
    u = rng.dirichlet([1, 1, 1], size=1024)
    on = (u[:, :, None] * corners[pick]).sum(1)
    n = np.cross(corners[pick, 1] - corners[pick, 0], corners[pick, 2] - corners[pick, 0])
    n /= np.linalg.norm(n, axis=1, keepdims=True)
    near = on + n * (10.0 ** rng.uniform(-5, -2, size=(1024, 1))) * rng.choice([-1, 1], (1024, 1))
    O = np.concatenate([box, near])
    W = mixed_host(tri, O)
    assert np.abs(W - oracle_mod.winding_soa(tri, O)).max() <= TOL


def test_queries_clustered_at_vertex_fans(gpu_required, oracle_mod):
    """Queries 1e-9..1e-3 from vertices where five or six faces meet."""
    V, F = igl.synthetic.bumpy_icosphere(3, seed=9)
    rng = np.random.default_rng(10)
    vid = rng.integers(0, len(V), size=600)
    d = rng.normal(size=(600, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    O = V[vid] + d * 10.0 ** rng.uniform(-9, -3, size=(600, 1))
    tri = igl._triangle_soa(V, F)
    W = mixed_host(tri, O)
    assert np.abs(W - oracle_mod.winding_soa(tri, O)).max() <= TOL


@pytest.mark.parametrize("workload", ["c2_open", "c3_mixed", "soup"])
def test_half_tiles_keep_the_bound(gpu_required, oracle_mod, workload):
    """32 faces per far test and angle product (each half of a 64-face tile on its
    own): the same 1e-6 bound as 64-face tiles, on an open mesh, on near-surface
    queries of the c3 mesh, and on a multiscale soup whose halves' balls differ."""
    import torch

    if workload == "soup":
        rng = np.random.default_rng(18)
        nf = 3000
        corners = rng.uniform(-1, 1, (nf, 1, 3)) + 10.0 ** rng.uniform(-3, 0, (nf, 1, 1)) * \
            rng.normal(size=(nf, 3, 3))
        tri = np.ascontiguousarray(corners.transpose(1, 2, 0).reshape(9, nf))
        pick = rng.integers(0, nf, 1000)
        O = np.concatenate([rng.uniform(-1.2, 1.2, (1000, 3)),
                            corners[pick].mean(1) + 1e-4 * rng.normal(size=(1000, 3))])
    else:
        V, F, O, _ = igl.synthetic.workload(workload, n_queries=4096)
        tri = igl._triangle_soa(V, F)
    nf = tri.shape[1]
    ld = nf + (nf & 1)
    tri_d = torch.zeros((9, ld), dtype=torch.float64, device="cuda")
    tri_d[:, :nf] = torch.from_numpy(tri)
    q_d = torch.from_numpy(np.ascontiguousarray(O)).cuda()
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    h = _lib.lib()
    mesh = ctypes.c_void_p()
    assert h.wn_mixed_mesh_create(tri_d.data_ptr(), ld, nf, 4.0, stream, ctypes.byref(mesh)) == 0
    try:
        out = {}
        for tf in (64, 32):
            assert h.wn_mixed_mesh_set_tile_faces(mesh, tf) == 0
            w_d = torch.empty(len(O), dtype=torch.float64, device="cuda")
            assert h.wn_forward_mixed_device(mesh, q_d.data_ptr(), len(O), w_d.data_ptr(),
                                             stream) == 0, _lib.last_error()
            assert h.wn_stream_check(stream) == 0
            out[tf] = w_d.cpu().numpy()
        assert h.wn_mixed_mesh_set_tile_faces(mesh, 48) != 0
    finally:
        h.wn_mixed_mesh_destroy(mesh)
    ref = oracle_mod.winding_soa(tri, O, workers=8)
    assert np.abs(out[64] - ref).max() <= TOL
    assert np.abs(out[32] - ref).max() <= TOL
