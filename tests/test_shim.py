"""The drop-in Python API (CPU side): contracts of python/igl/__init__.py:232-283
and python/igl/_lib.py, mirrored from the reference's tests/test_parity.py."""

import numpy as np
import pytest

import igl
from igl import _lib
from conftest import GOLDEN_CASES, grid, load_golden, tetrahedron


@pytest.mark.parametrize("name", GOLDEN_CASES)
def test_cpu_path_matches_reference_golden(name):
    g = load_golden(name)
    W = igl.winding_number(g["V"], g["F"], g["O"])
    assert np.abs(W - g["W"]).max() < 1e-12


def test_published_solid_angle_invariant():
    V, F = tetrahedron()
    Q = np.array([[0.1, 0.1, 0.1], [2.0, 2.0, 2.0], [-1.0, 0.2, 0.2]])
    W = igl.winding_number(V, F, Q)
    assert W[0] == pytest.approx(1.0, abs=1e-14)
    assert np.abs(W[1:]).max() < 1e-14
    assert isinstance(igl.winding_number(V, F, Q[0]), float)
    assert igl.winding_number(V, F, Q[0]) == pytest.approx(1.0, abs=1e-14)
    assert igl.winding_number_for_point(V, F, Q[0]) == pytest.approx(1.0, abs=1e-14)


def test_cpu_path_matches_oracle_on_degenerate_queries(oracle_mod):
    V, F = tetrahedron()
    Q = np.array([[0.0, 0.0, 0.0], [1.0, 0.0, 0.0], [0.3, 0.3, 0.0], [0.0, 0.5, 0.0],
                  [2.0, 0.0, 0.0], [1e6, 1e6, -1e6], [1e-300, 0.0, 0.0]])
    assert np.abs(igl.winding_number(V, F, Q) - oracle_mod.winding_number(V, F, Q)).max() < 1e-14


def _force_serial(monkeypatch):
    monkeypatch.setattr(igl, "worker_count", lambda items, work, kernel: 1)


def _force_parallel(monkeypatch, workers):
    monkeypatch.setattr(igl, "worker_count",
                        lambda items, work, kernel: max(1, min(items, workers)))


def test_serial_and_parallel_output_is_identical(monkeypatch):
    V, F = grid(20)
    rng = np.random.default_rng(77)
    Q = rng.uniform([0.0, 0.0, -2.0], [19.0, 19.0, 2.0], size=(512, 3))
    _force_serial(monkeypatch)
    serial = igl.winding_number(V, F, Q)
    for workers in (1, 2, 4, 8):
        _force_parallel(monkeypatch, workers)
        assert np.array_equal(igl.winding_number(V, F, Q), serial)


def test_input_contracts():
    V, F = grid(3)
    with pytest.raises(ValueError):
        igl.winding_number(V, F, [[np.nan, 0.0, 0.0]])
    with pytest.raises(ValueError):
        igl.winding_number(V, F, [[np.inf, 0.0, 0.0]])
    with pytest.raises(ValueError):
        igl.winding_number(V[:, :2], F, [[0.0, 0.0, 0.0]])
    with pytest.raises(ValueError):
        igl.winding_number(V, F, [[0.0, 0.0]])
    with pytest.raises(ValueError):
        igl.winding_number(V, F, [0.0, 0.0])
    with pytest.raises(ValueError):
        igl.winding_number(V, F, [[0.0, 0.0, 0.0]], device="tpu")
    with pytest.raises(ValueError):
        igl.winding_number(V, F, [[0.0, 0.0, 0.0]], precision="fp16")
    with pytest.raises(TypeError):
        igl.winding_number(V, F.astype(np.float64), [[0.0, 0.0, 0.0]])
    with pytest.raises(TypeError):
        igl.winding_number(V.astype(complex), F, [[0.0, 0.0, 0.0]])
    with pytest.raises(TypeError):
        igl.winding_number(V, F.astype(bool), [[0.0, 0.0, 0.0]])
    with pytest.raises(IndexError):
        igl.winding_number(V, np.array([[0, 1, len(V)]]), [[0.0, 0.0, 0.0]])
    with pytest.raises(IndexError):
        igl.winding_number(V, np.array([[0, 1, -1]]), [[0.0, 0.0, 0.0]])
    with pytest.raises(OverflowError):
        igl.winding_number(V, np.array([[0, 1, 2**63]], dtype=np.uint64), [[0.0, 0.0, 0.0]])
    with pytest.raises(ValueError):
        igl.winding_number(V, F, np.array([[2**60, 0, 0]], dtype=np.int64))


def test_empty_and_integer_inputs():
    V, F = tetrahedron()
    out = igl.winding_number(V, F, np.zeros((0, 3)))
    assert out.shape == (0,) and out.dtype == np.float64
    assert np.array_equal(igl.winding_number(V, F[:0], np.ones((2, 3))), np.zeros(2))
    Vi = np.array([[0, 0, 0], [2, 0, 0], [0, 1, 0], [0, 0, 3]], dtype=np.int32)
    assert igl.winding_number(Vi, F.astype(np.int32), [0.1, 0.1, 0.1]) == pytest.approx(1.0)
    assert igl.winding_number(V, F, [[0.1, 0.1, 0.1]], device="CPU")[0] == pytest.approx(1.0)


def test_gpu_request_without_device_raises(monkeypatch):
    V, F = tetrahedron()
    monkeypatch.setattr(igl, "_gpu_memory_available", lambda: False)
    with pytest.raises(RuntimeError, match="no CPU fallback"):
        igl.winding_number(V, F, [[0.1, 0.1, 0.1]], device="gpu")


def test_gpu_kernel_failure_is_not_swallowed(monkeypatch):
    """Mirror of tests/test_parity.py:117-128 with a fake library."""
    V, F = tetrahedron()

    class FailedGpu:
        @staticmethod
        def mli_winding_gpu(*args):
            return 0

    monkeypatch.setattr(igl, "_gpu_memory_available", lambda: True)
    monkeypatch.setattr(igl, "lib", lambda: FailedGpu())
    with pytest.raises(RuntimeError, match="GPU"):
        igl.winding_number(V, F, [[0.1, 0.1, 0.1]], device="gpu")


def test_kernel_signatures_match_shim():
    """Mirror of tests/test_parity.py:294-340 for the thirteen reference names."""
    trailing = {
        "mli_cot_entries": 2, "mli_mass_contributions": 3, "mli_vertex_normals": 3,
        "mli_winding": 4, "mli_winding_gpu": 2, "mli_aabb_squared_distance": 4,
        "mli_heat_vector_divergence": 2, "mli_heat_precompute": 1, "mli_arap_covariance": 2,
        "mli_arap_rhs": 2, "mli_arap_covariance_rims": 3, "mli_arap_rhs_rims": 3,
        "mli_arap_rotations": 4,
    }
    buffers = {
        "mli_cot_entries": 3, "mli_mass_contributions": 3, "mli_vertex_normals": 3,
        "mli_winding": 3, "mli_winding_gpu": 3, "mli_aabb_squared_distance": 10,
        "mli_heat_vector_divergence": 4, "mli_heat_precompute": 3, "mli_arap_covariance": 6,
        "mli_arap_rhs": 6, "mli_arap_covariance_rims": 5, "mli_arap_rhs_rims": 5,
        "mli_arap_rotations": 2,
    }
    assert set(trailing) == set(buffers) == set(_lib._SIGNATURES)
    for name in trailing:
        assert len(_lib._SIGNATURES[name][0]) == buffers[name] + trailing[name]


def test_worker_count_and_spans():
    assert _lib.worker_count(1, 10**9, "winding") == 1
    assert _lib.worker_count(1000, 1000, "winding") == 1
    assert 1 <= _lib.worker_count(1000, 10**6, "winding") <= _lib.MAX_WORKERS
    assert _lib.spans(10, 3) == [(0, 4), (4, 8), (8, 10)]
    assert _lib.spans(2, 4) == [(0, 1), (1, 2)]


@pytest.mark.parametrize("nf", [0, 1, 7, 1280, 28322])
def test_triangle_soa_matches_the_reference_layout(nf):
    """The per-corner gather gives the bytes of the reference's repack
    (python/igl/__init__.py:248-250 there: vertices[faces] transposed to
    rows 3*corner+axis)."""
    rng = np.random.default_rng(nf)
    V = rng.normal(size=(max(3, nf // 2 + 3), 3))
    F = rng.integers(0, len(V), size=(nf, 3))
    expected = np.ascontiguousarray(V[F].transpose(1, 2, 0).reshape(9, nf))
    got = igl._triangle_soa(*igl._mesh(V, F))
    assert got.flags.c_contiguous and got.dtype == np.float64
    assert got.shape == (9, nf) and np.array_equal(got, expected)


def test_vector_lanes_equal_the_scalar_path():
    """mli_winding evaluates queries 8 (AVX-512) or 4 (AVX2) at a time; a span of
    one query takes the scalar routine. Every query's result must be the same
    bits either way, on-vertex and on-edge queries included."""
    handle = _lib.lib()
    V, F = igl.synthetic.bumpy_icosphere(2, seed=4)
    rng = np.random.default_rng(6)
    O = np.concatenate([V[:9], 0.5 * (V[F[:8, 0]] + V[F[:8, 1]]),
                        rng.uniform(-1.5, 1.5, size=(20, 3))])  # 37: 8 + 8 + 8 + 8 + 4 + 1
    tri = igl._triangle_soa(*igl._mesh(V, F))
    whole = np.empty(len(O))
    handle.mli_winding(tri.ctypes.data, O.ctypes.data, whole.ctypes.data, tri.shape[1], len(O),
                       0, len(O))
    single = np.empty(len(O))
    for i in range(len(O)):
        handle.mli_winding(tri.ctypes.data, O.ctypes.data, single.ctypes.data, tri.shape[1],
                           len(O), i, i + 1)
    assert np.array_equal(whole, single, equal_nan=True)


def test_autotune_coordinate_descent_without_a_gpu(monkeypatch):
    """The tuner's search on a fake timing surface: it starts from the first value
    of every dimension, sweeps one dimension at a time, keeps improvements, and
    reports every configuration it timed (no GPU: Batch and timing are faked)."""
    from igl import autotune

    cost = {"tile_faces": {64: 0.0, 32: -1.0}, "qpt": {2: 0.0, 1: 2.0, 4: -0.5},
            "ctas_per_sm": {0: 0.0, 2: 0.3}}

    class FakeBatch:
        def __init__(self, meshes, sample, **cfg):
            self.cfg = cfg

        def close(self):
            pass

        @property
        def gW(self):
            class G:
                def normal_(self):
                    pass
            return G()

    monkeypatch.setattr(autotune, "Batch", FakeBatch)
    monkeypatch.setattr(autotune, "_time",
                        lambda b, backward, reps: 10.0 + sum(cost[k][v] for k, v in b.cfg.items()))
    monkeypatch.setattr(autotune, "cache_key", lambda m, q: "fake")
    space = {"tile_faces": (64, 32), "qpt": (2, 1, 4), "ctas_per_sm": (0, 2)}
    out = autotune.tune([None], [np.zeros((4, 3))], space=space, use_cache=False)
    assert out["config"] == {"tile_faces": 32, "qpt": 4, "ctas_per_sm": 0}
    assert out["ms"] == 8.5
    assert out["trials"][0]["config"] == {"tile_faces": 64, "qpt": 2, "ctas_per_sm": 0}
    assert len({tuple(sorted(t["config"].items())) for t in out["trials"]}) == len(out["trials"])
    grid = autotune.tune([None], [np.zeros((4, 3))], space=space, use_cache=False, search="grid")
    assert len(grid["trials"]) == 12 and grid["config"] == out["config"]


def test_welded_edges_of_a_soup_without_a_gpu():
    """Sides welded by position: a closed mesh as a soup gives every geometric
    edge once (1.5 per face) with net count 0; an open one has count +-1 exactly
    on its boundary; each side points to its edge with the sign of its direction."""
    import torch

    from igl import autograd as wa
    from igl import synthetic

    V, F = synthetic.bumpy_icosphere(2, seed=3)
    Vs, Fs = synthetic.unshare_vertices(V, F)
    edges, ng, side_edge, sigma, ends = wa.welded_edges(torch.from_numpy(Vs),
                                                        torch.from_numpy(Fs))
    assert ng == 3 * len(F) // 2
    assert float(edges[6, :ng].abs().max()) == 0.0
    P, Q = edges[0:3, side_edge].T.numpy(), edges[3:6, side_edge].T.numpy()
    A, B = Vs[ends[:, 0].numpy()], Vs[ends[:, 1].numpy()]
    fwd = sigma.numpy() > 0
    assert np.array_equal(P[fwd], A[fwd]) and np.array_equal(Q[fwd], B[fwd])
    assert np.array_equal(P[~fwd], B[~fwd]) and np.array_equal(Q[~fwd], A[~fwd])
    Fo = synthetic.delete_faces(F, 0.1, seed=4)
    Vo, Fo = synthetic.unshare_vertices(V, Fo)
    e_open, ng_open, *_ = wa.welded_edges(torch.from_numpy(Vo), torch.from_numpy(Fo))
    _, nb, _ = wa.boundary_edges(torch.from_numpy(V), torch.from_numpy(
        synthetic.delete_faces(F, 0.1, seed=4)))
    assert int((e_open[6, :ng_open] != 0).sum()) == nb
    assert float(e_open[6, :ng_open].abs().max()) == 1.0


def test_shared_corner_lengths_equal_the_scalar_path():
    """With eight or more queries and a mesh whose faces share corner positions,
    mli_winding computes each distinct position's |v - o| once per block of
    queries, per chunk of 2,048 faces or for a whole small mesh. The results
    must stay the scalar routine's bits: a grid cut into two chunks, a mesh above
    the whole-mesh size, a soup whose faces share no position (plain path), and
    no faces at all."""
    handle = _lib.lib()
    rng = np.random.default_rng(12)
    Vg, Fg = igl.synthetic.terrain_grid(40)  # 3,042 faces: two chunks
    Vb, Fb = igl.synthetic.bumpy_icosphere(6, seed=2)  # 81,920 faces
    Vs, Fs = igl.synthetic.bumpy_icosphere(2, seed=5)
    soup = Vs[Fs] + rng.normal(0.0, 1e-9, size=(len(Fs), 3, 3))  # no shared positions
    cases = [(igl._triangle_soa(*igl._mesh(Vg, Fg)), Vg),
             (igl._triangle_soa(*igl._mesh(Vb, Fb)), Vb),
             (np.ascontiguousarray(soup.transpose(1, 2, 0).reshape(9, -1)), Vs)]
    for tri, V in cases:
        lo, hi = V.min(0), V.max(0)
        O = np.ascontiguousarray(np.concatenate(
            [V[:5], rng.uniform(lo, hi, size=(12, 3))]))  # 17: 8 + 8 + 1, on-vertex queries
        whole = np.empty(len(O))
        handle.mli_winding(tri.ctypes.data, O.ctypes.data, whole.ctypes.data, tri.shape[1],
                           len(O), 0, len(O))
        single = np.empty(len(O))
        for i in range(len(O)):
            handle.mli_winding(tri.ctypes.data, O.ctypes.data, single.ctypes.data,
                               tri.shape[1], len(O), i, i + 1)
        assert np.array_equal(whole, single, equal_nan=True)
        # A span that starts off a block boundary and leaves the rest untouched.
        part = np.full(len(O), 7.0)
        handle.mli_winding(tri.ctypes.data, O.ctypes.data, part.ctypes.data, tri.shape[1],
                           len(O), 3, len(O) - 1)
        assert np.array_equal(part[3:-1], single[3:-1], equal_nan=True)
        assert np.all(part[:3] == 7.0) and part[-1] == 7.0
    empty = np.zeros((9, 0))
    O = rng.uniform(-1.0, 1.0, size=(9, 3))
    out = np.full(9, 7.0)
    handle.mli_winding(empty.ctypes.data, O.ctypes.data, out.ctypes.data, 0, 9, 0, 9)
    assert np.array_equal(out, np.zeros(9))
