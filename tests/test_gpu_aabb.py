"""Closest-point traversal on the B200 vs the oracle: bit-exact (sqrd, face, point).

Every comparison is exact equality: the kernel repeats the reference's ordered
walk (src/capi.mojo:522-586) with the same FP64 arithmetic, so even exact ties
(points on shared vertices and edges, duplicated faces) pick the same face.
Cases: the reference-generated golden fixtures, a tie-heavy flat grid, the
subdivision-5 open mesh with 65,536 mixed queries (above the Morton-sorting
threshold), the reference's own AABB benchmark shape (grid(350), 243,602 F)
and the signed distance against the CPU path.
"""

import glob
import os

import numpy as np
import pytest

import igl
from conftest import GOLDEN, grid

pytestmark = pytest.mark.gpu

AABB_CASES = sorted(os.path.basename(p)[5:-4] for p in glob.glob(os.path.join(GOLDEN,
                                                                                "aabb_*.npz")))


def _golden(name):
    data = np.load(os.path.join(GOLDEN, f"aabb_{name}.npz"))
    return {k: data[k] for k in data.files}


def _device_query(V, F, P):
    import torch

    from igl import distance

    tree = distance.DeviceAABB(V, F)
    out = tree.query(torch.from_numpy(np.ascontiguousarray(P)).cuda())
    torch.cuda.synchronize()
    res = tuple(t.cpu().numpy() for t in out)
    tree.close()
    return res


def _assert_equal(actual, expected):
    for a, b in zip(actual, expected):
        assert a.shape == b.shape
        assert np.array_equal(a, b)


@pytest.mark.parametrize("name", AABB_CASES)
def test_golden_host_entry(gpu_required, name):
    g = _golden(name)
    tree = igl.AABB()
    tree.init(g["V"], g["F"])
    _assert_equal(tree.squared_distance(g["V"], g["F"], g["P"], device="gpu"),
                  (g["sqrd"], g["index"], g["closest"]))
    # Repeated queries reuse the uploaded tree.
    _assert_equal(tree.squared_distance(g["V"], g["F"], g["P"][::-1], device="gpu"),
                  (g["sqrd"][::-1], g["index"][::-1], g["closest"][::-1]))


@pytest.mark.parametrize("name", AABB_CASES)
def test_golden_device_entry(gpu_required, name):
    g = _golden(name)
    _assert_equal(_device_query(g["V"], g["F"], g["P"]), (g["sqrd"], g["index"], g["closest"]))


def _tie_grid():
    V, F = grid(30, curved=False)
    F = np.concatenate([F, F[100:140], F[::-1][:50]])
    ij = np.stack(np.meshgrid(np.arange(30.0), np.arange(30.0), indexing="ij"), -1).reshape(-1, 2)
    P = np.concatenate([np.column_stack([ij, np.zeros(900)]),
                        np.column_stack([ij + [0.5, 0.0], np.zeros(900)]),
                        np.column_stack([ij + 0.5, np.full(900, 0.3)]),
                        np.column_stack([ij, np.full(900, -2.0)])])
    return V, F, P


@pytest.mark.parametrize("repeat", [1, 6])  # 3,600 points (input order), 21,600 (Morton order)
def test_exact_ties_match_oracle(gpu_required, oracle_mod, repeat):
    V, F, P = _tie_grid()
    P = np.tile(P, (repeat, 1))
    expected = oracle_mod.aabb_squared_distance(P, V, F, workers=8)
    _assert_equal(_device_query(V, F, P), expected)
    _assert_equal(igl.point_mesh_squared_distance(P, V, F, device="gpu"), expected)


def test_open_mesh_mixed_queries(gpu_required, oracle_mod):
    V, F, O, _ = igl.synthetic.workload("c2_open", n_queries=65536)
    expected = oracle_mod.aabb_squared_distance(O, V, F, workers=8)
    _assert_equal(_device_query(V, F, O), expected)


def test_reference_benchmark_shape(gpu_required, oracle_mod):
    """grid(350) (243,602 F) x 10,000 points uniform in [-10,360]^2 x [-5,5], the
    reference's AABB benchmark case, plus 40,000 more for the sorted path."""
    V, F = igl.synthetic.terrain_grid(350)
    P = np.random.default_rng(7).uniform([-10, -10, -5], [360, 360, 5], size=(50_000, 3))
    tree_arrays = oracle_mod.build_aabb(V, F)
    for sl in (slice(0, 10_000), slice(None)):
        expected = oracle_mod.aabb_squared_distance(P[sl], V, F, tree=tree_arrays, workers=8)
        _assert_equal(_device_query(V, F, P[sl]), expected)


def test_signed_distance_device_matches_cpu(gpu_required):
    import torch

    from igl import distance

    V, F = igl.synthetic.bumpy_icosphere(4, seed=9)
    P = igl.synthetic.mixed_queries(V, F, 20_000, seed=10, near_sigma=1e-3)
    S_cpu, I_cpu, C_cpu = igl.signed_distance(P, V, F)
    tree = distance.DeviceAABB(V, F)
    Pt = torch.from_numpy(P).cuda()
    for precision in ("fp64", "mixed"):
        S, index, closest, W = tree.signed_distance(Pt, precision=precision)
        torch.cuda.synchronize()
        assert np.array_equal(index.cpu().numpy(), I_cpu)
        assert np.array_equal(closest.cpu().numpy(), C_cpu)
        assert np.array_equal(np.abs(S.cpu().numpy()), np.abs(S_cpu))
        w = W.cpu().numpy()
        safe = np.abs(np.abs(w) - 0.5) > 1e-6
        assert np.array_equal(S.cpu().numpy()[safe], S_cpu[safe])
        assert safe.mean() > 0.999
    S_np, _, _ = igl.signed_distance(P, V, F, device="gpu")
    assert np.array_equal(S_np, S_cpu)
    tree.close()


@pytest.mark.parametrize("n", [1000, 20_000])  # below / above the Morton-sort threshold
def test_fast_signed_distance_equals_its_two_parts(gpu_required, n):
    """The fused entry (closest points and fast winding numbers on two streams
    from one sorted order) gives exactly what the two separate calls give."""
    import torch

    from igl import distance

    V, F = igl.synthetic.bumpy_icosphere(4, seed=9)
    P = igl.synthetic.mixed_queries(V, F, n, seed=11, near_sigma=1e-3)
    tree = distance.DeviceAABB(V, F)
    Pt = torch.from_numpy(P).cuda()
    sqrd, index, closest = (x.clone() for x in tree.query(Pt))
    w_fast = tree.fast_winding().evaluate_torch(Pt, beta=2.0)
    for _ in range(2):
        S, I, C, W = tree.signed_distance(Pt, precision="fast", beta=2.0)
        torch.cuda.synchronize()
        assert torch.equal(I, index) and torch.equal(C, closest)
        assert torch.equal(W, w_fast)
        expected = torch.where(w_fast.abs() > 0.5, -sqrd.sqrt(), sqrd.sqrt())
        assert torch.equal(S, expected)
    tree.close()


def test_empty_and_zero_points(gpu_required):
    import torch

    from igl import distance

    V, F = grid(5)
    tree = distance.DeviceAABB(V, F)
    s, i, c = tree.query(torch.zeros((0, 3), dtype=torch.float64, device="cuda"))
    assert s.shape == (0,) and i.shape == (0,) and c.shape == (0, 3)
    tree.close()
    empty = distance.DeviceAABB(V, np.zeros((0, 3), dtype=np.int64))
    s, i, c = empty.query(torch.ones((4, 3), dtype=torch.float64, device="cuda"))
    assert torch.isinf(s).all() and (i == -1).all() and (c == 0).all()
    empty.close()
    sqrd, index, closest = igl.point_mesh_squared_distance(V[:3], V, np.zeros((0, 3), np.int64),
                                                           device="gpu")
    assert np.all(np.isinf(sqrd)) and np.all(index == -1)


def test_device_error_word_stays_clear(gpu_required):
    import ctypes

    import torch

    V, F = igl.synthetic.bumpy_icosphere(3, seed=1)
    _device_query(V, F, igl.synthetic.mixed_queries(V, F, 30_000, seed=2))
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    assert igl.lib().wn_stream_check(stream) == 0


def test_signed_distance_fast_device(gpu_required):
    import torch

    from igl import distance

    V, F = igl.synthetic.bumpy_icosphere(5, seed=14)
    P = igl.synthetic.mixed_queries(V, F, 50_000, seed=15, near_sigma=1e-3)
    tree = distance.DeviceAABB(V, F)
    Pt = torch.from_numpy(P).cuda()
    S64, i64, c64, W64 = tree.signed_distance(Pt, precision="fp64")
    Sf, i_f, c_f, Wf = tree.signed_distance(Pt, precision="fast")
    torch.cuda.synchronize()
    assert torch.equal(i64, i_f) and torch.equal(c64, c_f)
    assert torch.equal(S64.abs(), Sf.abs())
    assert (Wf - W64).abs().max().item() <= 1e-2
    assert torch.equal(torch.sign(S64), torch.sign(Sf))
    S_np, _, _ = igl.signed_distance(P, V, F, device="gpu", precision="fast")
    assert np.array_equal(S_np, Sf.cpu().numpy())
    tree.close()
