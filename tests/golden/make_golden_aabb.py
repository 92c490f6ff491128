"""Regenerate the golden closest-point fixtures (``aabb_*.npz``) in this directory.

The fixtures come from the REFERENCE's own Python package (lee101/mojo-libigl
``python/igl``): ``AABB.init`` builds the median-split hierarchy in pure Python
(python/igl/__init__.py:286-319), so the stored ``boxes``/``nodes``/``order``/
``stack_size`` are the reference's own tree; ``AABB.squared_distance``
(__init__.py:339-382) then drives ``mli_aabb_squared_distance`` through the
reference's ctypes shim and span fan-out, with ``MOJO_LIBIGL_LIB`` pointing at
the CPU oracle library (the C++ restatement of src/capi.mojo:401-586, built
by ``oracle/Makefile``), because the reference's Mojo toolchain is not
installable offline. Each case also stores the brute-force minimum of the
squared distance over every face (``sqrd_brute``, the oracle's per-triangle
closest point taken over all faces), which pins the traversal's pruning.

Usage (needs the reference checkout; the fixtures are committed, so tests and
the GPU host never run this):

    python tests/golden/make_golden_aabb.py /path/to/reference
"""

from __future__ import annotations

import importlib
import importlib.util
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))


def _load(name: str, path: str):
    spec = importlib.util.spec_from_file_location(name, path)
    module = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(module)
    return module


def cases(golden, synthetic):
    grid = golden.grid
    out = {}
    V, F = grid(8)
    out["grid8_uniform"] = (V, F, np.random.default_rng(4).uniform(
        [-1.0, -1.0, -1.0], [8.0, 8.0, 2.0], size=(100, 3)))
    V, F = grid(9)
    out["grid9_normal"] = (V, F, np.random.default_rng(12).normal(size=(80, 3))
                           * [3.0, 3.0, 1.0] + [4.0, 4.0, 0.0])
    V, F = grid(10)
    out["grid10_spans"] = (V, F, np.random.default_rng(19).uniform(
        [-1.0, -1.0, -1.0], [10.0, 10.0, 2.0], size=(257, 3)))
    # Degenerate faces: a segment (repeated corner) and a point (all three equal).
    out["degenerate"] = (np.array([[0.0, 0, 0], [2.0, 0, 0], [0.0, 1, 0]]),
                         np.array([[0, 1, 1], [2, 2, 2]], dtype=np.int64),
                         np.array([[0.5, 1.0, 0.0], [0.0, 2.0, 0.0], [3.0, -1.0, 0.5]]))
    # Exact ties: points on vertices, on edge midpoints and straight above
    # vertices of a flat grid, plus a duplicated face; the winning face index is
    # decided by the traversal order alone.
    V, F = grid(6, curved=False)
    F = np.concatenate([F, F[7:9]])
    ij = np.stack(np.meshgrid(np.arange(6.0), np.arange(6.0), indexing="ij"), -1).reshape(-1, 2)
    P = np.concatenate([
        np.column_stack([ij, np.zeros(len(ij))]),
        np.column_stack([ij + [0.5, 0.0], np.zeros(len(ij))])[:20],
        np.column_stack([ij + [0.5, 0.5], np.full(len(ij), 0.25)])[:20],
        np.column_stack([ij, np.full(len(ij), 0.75)]),
        np.array([[-2.0, -2.0, 0.0], [7.0, 2.5, -1.0], [2.5, 2.5, 0.0]]),
    ])
    out["ties_flat_grid"] = (V, F, P)
    V, F = synthetic.bumpy_icosphere(2, seed=5)
    Fo = synthetic.delete_faces(F, 0.08, seed=7)
    out["bumpy_s2_open"] = (V, Fo, synthetic.mixed_queries(V, Fo, 300, seed=8,
                                                           near_sigma=1e-3))
    V, F = grid(40)
    out["grid40_spans"] = (V, F, np.random.default_rng(78).uniform(
        [-5.0, -5.0, -5.0], [45.0, 45.0, 5.0], size=(1024, 3)))
    return out


def main(reference: str) -> None:
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import oracle  # noqa: E402

    os.environ["MOJO_LIBIGL_LIB"] = oracle.build()
    golden = _load("wn_make_golden", os.path.join(HERE, "make_golden.py"))
    synthetic = _load("wn_synthetic", os.path.join(REPO, "mojo-libigl_b200", "python", "igl",
                                                   "synthetic.py"))
    all_cases = cases(golden, synthetic)
    sys.dont_write_bytecode = True
    sys.path.insert(0, os.path.join(reference, "python"))
    ref_igl = importlib.import_module("igl")
    assert os.path.realpath(ref_igl.__file__).startswith(os.path.realpath(reference)), ref_igl
    for name, (V, F, P) in all_cases.items():
        tree = ref_igl.AABB()
        tree.init(V, F)
        sqrd, index, closest = tree.squared_distance(V, F, P)
        boxes, nodes, order, stack_size = tree._tree
        brute = np.array([min(oracle.closest_point(p, V[f].ravel())[0] for f in F) for p in P])
        np.savez_compressed(os.path.join(HERE, f"aabb_{name}.npz"), V=V, F=F, P=P, boxes=boxes,
                            nodes=nodes, order=order, stack_size=stack_size, sqrd=sqrd,
                            index=index, closest=closest, sqrd_brute=brute)
        print(name, V.shape, F.shape, P.shape, "nodes", len(nodes), "stack", stack_size,
              "max |sqrd - brute| =", float(np.abs(sqrd - brute).max()))


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.environ.get("REFERENCE_ROOT", ""))
