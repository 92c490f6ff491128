"""Closest-point path on the CPU: oracle pins, native tree builder, host query.

Mirrors the reference's AABB tests (tests/test_parity.py:131-190, 270-290,
343-350, 430-445): golden fixtures made by the reference's own Python
``AABB`` (its pure-Python tree builder, its shim and span fan-out) over the
oracle's C restatement of the traversal (tests/golden/make_golden_aabb.py),
brute-force minima over every face, exact ties, degenerate faces, serial vs
parallel spans, and the input contracts.
"""

import ctypes
import glob
import os

import numpy as np
import pytest

import igl
from conftest import GOLDEN, grid

AABB_CASES = sorted(os.path.basename(p)[5:-4] for p in glob.glob(os.path.join(GOLDEN,
                                                                                "aabb_*.npz")))


def _golden(name):
    data = np.load(os.path.join(GOLDEN, f"aabb_{name}.npz"))
    return {k: data[k] for k in data.files}


def test_golden_cases_present():
    assert {"grid8_uniform", "ties_flat_grid", "degenerate", "bumpy_s2_open"} <= set(AABB_CASES)


@pytest.mark.parametrize("name", AABB_CASES)
def test_oracle_matches_reference_golden(oracle_mod, name):
    g = _golden(name)
    boxes, nodes, order, stack = oracle_mod.build_aabb(g["V"], g["F"])
    assert np.array_equal(boxes, g["boxes"]) and np.array_equal(nodes, g["nodes"])
    assert np.array_equal(order, g["order"]) and stack == int(g["stack_size"])
    sqrd, index, closest = oracle_mod.aabb_squared_distance(g["P"], g["V"], g["F"], workers=3)
    assert np.array_equal(sqrd, g["sqrd"])
    assert np.array_equal(index, g["index"])
    assert np.array_equal(closest, g["closest"])
    # The pruned traversal finds the brute-force minimum over every face.
    assert np.array_equal(sqrd, g["sqrd_brute"])


@pytest.mark.parametrize("name", AABB_CASES)
def test_native_tree_and_host_query_match_golden(name, monkeypatch):
    g = _golden(name)
    boxes, nodes, order, stack = igl._build_aabb(g["V"], g["F"])
    assert np.array_equal(boxes, g["boxes"]) and np.array_equal(nodes, g["nodes"])
    assert np.array_equal(order, g["order"]) and stack == int(g["stack_size"])
    tree = igl.AABB()
    tree.init(g["V"], g["F"])
    for workers in (1, 3):
        monkeypatch.setattr(igl, "worker_count",
                            lambda items, work, kernel, w=workers: max(1, min(items, w)))
        sqrd, index, closest = tree.squared_distance(g["V"], g["F"], g["P"])
        assert np.array_equal(sqrd, g["sqrd"])
        assert np.array_equal(index, g["index"])
        assert np.array_equal(closest, g["closest"])


def _flat_grid_with_duplicates():
    V, F = grid(30, curved=False)
    return V, np.concatenate([F, F[100:140], F[::-1][:50]])


@pytest.mark.parametrize("mesh", ["bumpy_s5_open", "flat_grid_ties"])
def test_native_builder_matches_oracle_restatement(oracle_mod, mesh):
    if mesh == "bumpy_s5_open":
        V, F = igl.synthetic.bumpy_icosphere(5, seed=21)
        F = igl.synthetic.delete_faces(F, 0.08, seed=22)
    else:
        V, F = _flat_grid_with_duplicates()
    expected = oracle_mod.build_aabb(V, F)
    actual = igl._build_aabb(V, F)
    for a, b in zip(actual[:3], expected[:3]):
        assert np.array_equal(a, b)
    assert actual[3] == expected[3]
    for leaf in (1, 3, 16):
        n = igl.lib().wn_aabb_node_count(len(F), leaf)
        boxes = np.empty((n, 6))
        nodes = np.empty((n, 4), dtype=np.int64)
        order = np.empty(len(F), dtype=np.int64)
        stack = ctypes.c_int64()
        assert igl.lib().wn_aabb_build(V.ctypes.data, len(V), F.ctypes.data, len(F), leaf,
                                       boxes.ctypes.data, nodes.ctypes.data, order.ctypes.data,
                                       ctypes.byref(stack), 4) == 0
        ref = oracle_mod.build_aabb(V, F, leaf_size=leaf)
        assert np.array_equal(boxes, ref[0]) and np.array_equal(nodes, ref[1])
        assert np.array_equal(order, ref[2]) and stack.value == ref[3]


def test_host_query_matches_oracle_on_ties_and_shell(oracle_mod):
    V, F = _flat_grid_with_duplicates()
    ij = np.stack(np.meshgrid(np.arange(30.0), np.arange(30.0), indexing="ij"), -1)
    P = np.concatenate([np.column_stack([ij.reshape(-1, 2), np.zeros(900)]),
                        np.column_stack([ij.reshape(-1, 2) + 0.5, np.full(900, 0.3)]),
                        np.random.default_rng(5).uniform([-3, -3, -2], [32, 32, 2], (600, 3))])
    expected = oracle_mod.aabb_squared_distance(P, V, F, workers=2)
    actual = igl.point_mesh_squared_distance(P, V, F)
    for a, b in zip(actual, expected):
        assert np.array_equal(a, b)
    V2, F2 = igl.synthetic.bumpy_icosphere(4, seed=3)
    P2 = igl.synthetic.mixed_queries(V2, F2, 3000, seed=4, near_sigma=1e-4)
    for a, b in zip(igl.point_mesh_squared_distance(P2, V2, F2),
                    oracle_mod.aabb_squared_distance(P2, V2, F2)):
        assert np.array_equal(a, b)


def test_serial_and_parallel_output_is_identical(monkeypatch):
    V, F = grid(40)
    P = np.random.default_rng(78).uniform([-5.0, -5.0, -5.0], [45.0, 45.0, 5.0], size=(2048, 3))
    tree = igl.AABB()
    tree.init(V, F)
    monkeypatch.setattr(igl, "worker_count", lambda items, work, kernel: 1)
    serial = tree.squared_distance(V, F, P)
    for workers in (2, 4, 8):
        monkeypatch.setattr(igl, "worker_count",
                            lambda items, work, kernel, w=workers: max(1, min(items, w)))
        for actual, expected in zip(tree.squared_distance(V, F, P), serial):
            assert np.array_equal(actual, expected)


def test_input_contracts():
    V, F = grid(3)
    with pytest.raises(RuntimeError):
        igl.AABB().squared_distance(V, F, V[:1])
    with pytest.raises(ValueError):
        igl.point_mesh_squared_distance([[np.inf, 0.0, 0.0]], V, F)
    with pytest.raises(ValueError):
        igl.point_mesh_squared_distance([[0.0, 0.0]], V, F)
    with pytest.raises(ValueError):
        igl.point_mesh_squared_distance(V[:1], V[:, :2], F)
    with pytest.raises(IndexError):
        igl.point_mesh_squared_distance(V[:1], V, np.array([[0, 1, len(V)]]))
    with pytest.raises(ValueError):
        igl.point_mesh_squared_distance(V[:1], V, F, device="tpu")
    tree = igl.AABB()
    tree.init(V, F)
    changed = V.copy()
    changed[0, 0] += 1.0
    with pytest.raises(ValueError, match="AABB.init"):
        tree.squared_distance(changed, F, V[:1])
    with pytest.raises(NotImplementedError):
        tree.find(V, F, V[0])
    with pytest.raises(NotImplementedError):
        tree.intersect_ray(V, F, V[0], V[1])


def test_empty_inputs():
    V, F = grid(3)
    sqrd, index, closest = igl.point_mesh_squared_distance(V[:2], V, np.zeros((0, 3), np.int64))
    assert np.all(np.isinf(sqrd)) and np.all(index == -1) and np.all(closest == 0)
    sqrd, index, closest = igl.point_mesh_squared_distance(np.zeros((0, 3)), V, F)
    assert sqrd.shape == (0,) and index.shape == (0,) and closest.shape == (0, 3)


def test_signed_distance_cpu():
    V, F = igl.synthetic.bumpy_icosphere(3, seed=11)
    rng = np.random.default_rng(6)
    P = np.concatenate([rng.uniform(-0.5, 0.5, (50, 3)), rng.uniform(1.3, 2.0, (50, 3))])
    S, index, closest = igl.signed_distance(P, V, F)
    sqrd, index2, closest2 = igl.point_mesh_squared_distance(P, V, F)
    assert np.array_equal(np.abs(S), np.sqrt(sqrd))
    assert np.array_equal(index, index2) and np.array_equal(closest, closest2)
    assert np.all(S[:50] < 0) and np.all(S[50:] > 0)


def test_tree_upload_rejects_malformed_arrays():
    """Validation runs before any device work, so it needs no GPU."""
    V, F = grid(4)
    boxes, nodes, order, _ = igl._build_aabb(V, F)
    lib = igl.lib()

    def create(b, n, o):
        handle = ctypes.c_void_p()
        return lib.wn_aabb_create(V.ctypes.data, len(V), F.ctypes.data, len(F), b.ctypes.data,
                                  n.ctypes.data, o.ctypes.data, len(n), ctypes.byref(handle))

    bad = nodes.copy()
    bad[0, 0] = 0  # a node that is its own child (a cycle)
    assert create(boxes, bad, order) == 1 and "child" in igl._lib.last_error()
    bad = nodes.copy()
    leaf = int(np.nonzero(bad[:, 3] > 0)[0][0])
    bad[leaf, 2] = len(F)  # leaf range past the end of order
    assert create(boxes, bad, order) == 1 and "leaf" in igl._lib.last_error()
    bad_order = order.copy()
    bad_order[0] = len(F)
    assert create(boxes, nodes, bad_order) == 1 and "order" in igl._lib.last_error()


def _adversarial_triangles(rng, n):
    """Random triangles plus the shapes that exercise every branch: slivers,
    collinear corners (the degenerate branch), repeated corners, points, huge
    and tiny scales, and points on vertices, edges and faces."""
    tris, pts = [], []
    for i in range(n):
        kind = i % 8
        t = rng.normal(size=(3, 3))
        if kind == 1:
            t[2] = t[0] + rng.uniform(-2, 3) * (t[1] - t[0])  # collinear
        elif kind == 2:
            t[1] = t[0]  # repeated corner
        elif kind == 3:
            t[:] = t[0]  # a point
        elif kind == 4:
            t[2] = t[1] + 1e-9 * rng.normal(size=3)  # sliver
        elif kind == 5:
            t *= 10.0 ** rng.integers(-8, 9)
        p = rng.normal(size=3) * np.abs(t).max()
        if kind == 6:
            p = t[rng.integers(3)].copy()  # on a vertex
        elif kind == 7:
            u = rng.uniform(size=2)
            p = t[0] + u[0] * (t[1] - t[0]) + u[1] * (1 - u[0]) * (t[2] - t[0]) + 0.0 * p
        tris.append(t.ravel())
        pts.append(p)
    return np.array(tris), np.array(pts)


def test_closest_point_matches_oracle_bitwise(oracle_mod):
    """The arithmetic the host traversal and the GPU kernel share (wn_aabb.cuh)."""
    rng = np.random.default_rng(99)
    tris, pts = _adversarial_triangles(rng, 16000)
    out = np.empty(4)
    lib = igl.lib()
    for t, p in zip(tris, pts):
        expected = np.array(oracle_mod.closest_point(p, t))
        assert lib.wn_closest_point(p.ctypes.data, t.ctypes.data, out.ctypes.data) == 0
        assert out.tobytes() == expected.tobytes() or (
            np.isnan(out).any() and np.array_equal(np.isnan(out), np.isnan(expected))), (
            t, p, out, expected)


def test_signed_distance_fast_sign_cpu():
    """The hierarchical winding number gives the same signs away from |W| ~ 1/2."""
    V, F = igl.synthetic.bumpy_icosphere(4, seed=12)
    P = igl.synthetic.mixed_queries(V, F, 2000, seed=13, near_sigma=1e-3)
    exact, _, _ = igl.signed_distance(P, V, F)
    fast, _, _ = igl.signed_distance(P, V, F, precision="fast")
    assert np.array_equal(np.abs(fast), np.abs(exact))
    assert np.array_equal(np.sign(fast), np.sign(exact))
    with pytest.raises(ValueError):
        igl.signed_distance(P, V, F, precision="half")


def test_closest_point_eight_lanes_match_oracle_bitwise(oracle_mod):
    """The host traversal takes a leaf's faces eight at a time (AVX-512): every
    lane must give the scalar arithmetic's bits, for the point of each of the
    eight adversarial triangles in turn (slivers, collinear and repeated corners,
    points, scales, and points on vertices, edges and faces)."""
    lib = igl.lib()
    rng = np.random.default_rng(101)
    tris, pts = _adversarial_triangles(rng, 4000)
    tri72 = np.empty(72)
    out = np.empty(32)
    for g in range(0, len(tris), 8):
        group = tris[g:g + 8]  # (8, 9): A xyz, B xyz, C xyz per triangle
        tri72[:] = group.T.ravel()
        for p in pts[g:g + 8]:
            p = np.ascontiguousarray(p)
            rc = lib.wn_closest_point8(p.ctypes.data, tri72.ctypes.data, out.ctypes.data)
            if rc == 2:
                pytest.skip("no AVX-512 on this CPU")
            assert rc == 0
            got = out.reshape(4, 8).T  # (8, 4): d2, x, y, z per lane
            for t, lane in zip(group, got):
                expected = np.array(oracle_mod.closest_point(p, t))
                assert lane.tobytes() == expected.tobytes() or (
                    np.isnan(lane).any() and np.array_equal(np.isnan(lane), np.isnan(expected))), (
                    t, p, lane, expected)


@pytest.mark.parametrize("leaf", [1, 5, 16, 37])
def test_host_query_on_other_leaf_sizes_matches_oracle(oracle_mod, leaf):
    """Trees whose leaves hold more or fewer than eight faces: the host query
    takes a leaf's faces in groups of eight lanes (a partial last group
    included) and must still match the oracle's scalar walk bit for bit, ties
    and duplicated faces included."""
    V, F = _flat_grid_with_duplicates()
    P = np.concatenate([np.column_stack([np.arange(30.0), np.arange(30.0), np.zeros(30)]),
                        np.random.default_rng(leaf).uniform([-3, -3, -2], [32, 32, 2], (500, 3))])
    boxes, nodes, order, stack_size = oracle_mod.build_aabb(V, F, leaf_size=leaf)
    expected = oracle_mod.aabb_squared_distance(P, V, F, tree=(boxes, nodes, order, stack_size))
    n = len(P)
    sqrd = np.empty(n)
    index = np.empty(n, dtype=np.int64)
    closest = np.empty((n, 3))
    stack = np.empty(stack_size, dtype=np.int64)
    Pc = np.ascontiguousarray(P)
    Vc = np.ascontiguousarray(V, dtype=np.float64)
    Fc = np.ascontiguousarray(F, dtype=np.int64)
    igl.lib().mli_aabb_squared_distance(
        Pc.ctypes.data, Vc.ctypes.data, Fc.ctypes.data, boxes.ctypes.data, nodes.ctypes.data,
        order.ctypes.data, sqrd.ctypes.data, index.ctypes.data, closest.ctypes.data,
        stack.ctypes.data, n, len(nodes), 0, n)
    for a, b in zip((sqrd, index, closest), expected):
        assert np.array_equal(a, b)
