"""Plain FP64 GPU kernel vs the oracle (needs a B200).

Bar: |W_gpu - W_oracle| <= 1e-12 per query (the pair terms are bit-identical
to the reference's, only the summation differs), on the reference's own cases,
seeded meshes, odd sizes that exercise partial tiles and face splits, and
degenerate queries (on vertices, on edges, inside faces).
"""

import ctypes

import numpy as np
import pytest

import igl
from igl import _lib
from conftest import GOLDEN_CASES, load_golden, tetrahedron

pytestmark = pytest.mark.gpu
TOL = 1e-12
MODES = {"argprod": 0, "direct": 1, "tiled": 2}


def gpu_host(tri, O, mode="argprod"):
    tri = np.ascontiguousarray(tri, dtype=np.float64)
    O = np.ascontiguousarray(O, dtype=np.float64).reshape(-1, 3)
    out = np.full(len(O), np.nan)
    handle = _lib.lib()
    rc = handle.wn_forward_fp64_host(tri.ctypes.data, O.ctypes.data, out.ctypes.data,
                                     tri.shape[1], len(O), MODES[mode])
    assert rc == 0, _lib.last_error()
    return out


@pytest.mark.parametrize("name", GOLDEN_CASES)
@pytest.mark.parametrize("mode", list(MODES))
def test_golden_cases(gpu_required, name, mode):
    g = load_golden(name)
    tri = igl._triangle_soa(g["V"], g["F"])
    W = gpu_host(tri, g["O"], mode)
    assert np.abs(W - g["W"]).max() <= TOL


def test_reference_api_gpu_request(gpu_required, oracle_mod):
    """tests/test_parity.py:108-114: GPU equals CPU at 1e-14 on the tetrahedron."""
    V, F = tetrahedron()
    Q = np.array([[0.1, 0.1, 0.1], [2.0, 2.0, 2.0]])
    expected = oracle_mod.winding_number(V, F, Q)
    got = igl.winding_number(V, F, Q, device="gpu")
    assert np.abs(got - expected).max() <= 1e-14
    assert igl.winding_number(V, F, Q[0], device="GPU") == pytest.approx(1.0, abs=1e-14)


@pytest.mark.parametrize("nf,nq", [(1, 1), (2, 3), (3, 129), (127, 255), (128, 256), (129, 257),
                                   (255, 1), (1000, 17), (4097, 513)])
@pytest.mark.parametrize("mode", list(MODES))
def test_odd_sizes_random_soup(gpu_required, oracle_mod, nf, nq, mode):
    rng = np.random.default_rng(nf * 7919 + nq)
    tri = rng.normal(size=(9, nf))
    O = rng.normal(size=(nq, 3)) * 1.5
    W = gpu_host(tri, O, mode)
    ref = oracle_mod.winding_soa(tri, O)
    assert np.abs(W - ref).max() <= TOL


def test_bumpy_c1_full(gpu_required, oracle_mod):
    V, F, O, _ = igl.synthetic.workload("c1_cpu")
    tri = igl._triangle_soa(V, F)
    ref = oracle_mod.winding_soa(tri, O, workers=8)
    for mode in MODES:
        W = gpu_host(tri, O, mode)
        assert np.abs(W - ref).max() <= TOL
    assert np.abs(W - np.round(W)).max() < 1e-9  # closed mesh: W in {0, 1}


def test_open_mesh_c2_subset(gpu_required, oracle_mod):
    V, F, O, _ = igl.synthetic.workload("c2_open", n_queries=2048)
    tri = igl._triangle_soa(V, F)
    ref = oracle_mod.winding_soa(tri, O, workers=8)
    W = gpu_host(tri, O)
    assert np.abs(W - ref).max() <= TOL
    assert np.abs(W - np.round(W)).max() > 1e-3  # open mesh: fractional W exist


def test_degenerate_queries_match_oracle_exactly(gpu_required, oracle_mod):
    V, F = igl.synthetic.bumpy_icosphere(2, seed=9)
    tri = igl._triangle_soa(V, F)
    t = V[F]
    Q = np.concatenate([
        V[:40],                                   # on vertices: pairs with det=denom=0
        0.5 * (t[:40, 0] + t[:40, 1]),            # on edges
        (t[:40, 0] + t[:40, 1] + t[:40, 2]) / 3,  # inside faces: det ~ +-0, denom < 0
        [[0.0, 0.0, 0.0], [1e3, 1e3, 1e3], [1e-200, 0.0, 0.0]],
    ])
    ref = oracle_mod.winding_soa(tri, Q)
    for mode in MODES:
        W = gpu_host(tri, Q, mode)
        assert np.abs(W - ref).max() <= TOL, mode


def test_degenerate_faces(gpu_required, oracle_mod):
    rng = np.random.default_rng(5)
    tri = rng.normal(size=(9, 300))
    tri[:, :50] = 0.0                     # collapsed to the origin
    tri[3:6, 50:100] = tri[0:3, 50:100]   # two equal corners
    tri[6:9, 100:150] = 2 * tri[3:6, 100:150] - tri[0:3, 100:150]  # collinear
    O = rng.normal(size=(200, 3))
    O[0] = 0.0
    for mode in MODES:
        W = gpu_host(tri, O, mode)
        assert np.abs(W - oracle_mod.winding_soa(tri, O)).max() <= TOL


def test_empty_face_set_and_empty_queries(gpu_required):
    O = np.ones((5, 3))
    assert np.array_equal(gpu_host(np.zeros((9, 0)), O), np.zeros(5))
    assert gpu_host(np.zeros((9, 4)), np.zeros((0, 3))).shape == (0,)


def test_deterministic_repeat(gpu_required):
    V, F, O, _ = igl.synthetic.workload("c1_cpu")
    tri = igl._triangle_soa(V, F)
    a = gpu_host(tri, O)
    for _ in range(3):
        assert np.array_equal(gpu_host(tri, O), a)


def test_device_entry_point_with_torch_tensors(gpu_required, oracle_mod):
    import torch

    V, F, O, _ = igl.synthetic.workload("c1_cpu", n_queries=1000)
    tri = igl._triangle_soa(V, F)
    nf = tri.shape[1]
    ld = nf + (nf & 1)
    tri_d = torch.zeros((9, ld), dtype=torch.float64, device="cuda")
    tri_d[:, :nf] = torch.from_numpy(tri)
    q_d = torch.from_numpy(O).cuda()
    w_d = torch.empty(len(O), dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    handle = _lib.lib()
    rc = handle.wn_forward_fp64_device(tri_d.data_ptr(), ld, q_d.data_ptr(), w_d.data_ptr(), nf,
                                       len(O), 0, ctypes.c_void_p(stream))
    assert rc == 0, _lib.last_error()
    assert handle.wn_stream_check(ctypes.c_void_p(stream)) == 0
    assert np.abs(w_d.cpu().numpy() - oracle_mod.winding_soa(tri, O)).max() <= TOL


def test_device_entry_rejects_bad_layout(gpu_required):
    handle = _lib.lib()
    assert handle.wn_forward_fp64_device(None, 3, None, None, 2, 1, 0, None) != 0  # odd ld
    assert "ld" in _lib.last_error()


@pytest.mark.parametrize("mode", list(MODES))
def test_translated_multiscale_soup_and_vertex_fans(gpu_required, oracle_mod, mode):
    """The mixed path's adversarial inputs at the FP64 bar: a mesh 1e6 from the
    origin, a self-intersecting soup with sizes over four decades, and queries
    1e-9..1e-3 from vertices where faces fan out."""
    rng = np.random.default_rng(11)
    V, F = igl.synthetic.bumpy_icosphere(3, seed=6)
    t = np.array([1e6, -7e5, 3e5])
    O = igl.synthetic.mixed_queries(V, F, 256, seed=7, near_sigma=1e-4)
    tri = igl._triangle_soa(V + t, F)
    assert np.abs(gpu_host(tri, O + t, mode) - oracle_mod.winding_soa(tri, O + t)).max() <= TOL
    nf = 3000
    corners = (rng.uniform(-1, 1, size=(nf, 1, 3))
               + 10.0 ** rng.uniform(-4, 0, size=(nf, 1, 1)) * rng.normal(size=(nf, 3, 3)))
    tri = np.ascontiguousarray(corners.transpose(1, 2, 0).reshape(9, nf))
    O = rng.uniform(-1.2, 1.2, size=(300, 3))
    assert np.abs(gpu_host(tri, O, mode) - oracle_mod.winding_soa(tri, O)).max() <= TOL
    vid = rng.integers(0, len(V), size=300)
    d = rng.normal(size=(300, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    O = V[vid] + d * 10.0 ** rng.uniform(-9, -3, size=(300, 1))
    tri = igl._triangle_soa(V, F)
    assert np.abs(gpu_host(tri, O, mode) - oracle_mod.winding_soa(tri, O)).max() <= TOL
