"""Regenerate the golden vertex-normal fixtures (``normals_*.npz``) in this directory.

Produced by the REFERENCE's own Python package (lee101/mojo-libigl
``python/igl``: ``per_vertex_normals``, python/igl/__init__.py:195-211, with its
validation and weighting handling) loaded from a read-only checkout, with
``MOJO_LIBIGL_LIB`` pointing at the CPU oracle library (the C restatement of
src/capi.mojo:146-202 in oracle/normals_oracle.cpp), because the reference's
Mojo toolchain is not installable offline. Every case stores the normals for
weightings 0 (uniform), 1 (area), 2 (angle) and 3 (default).

Usage (needs the reference checkout; the fixtures are committed):

    python tests/golden/make_golden_normals.py /path/to/reference
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
    out = {}
    out["grid7"] = golden.grid()  # the reference tests' mesh (tests/test_parity.py:63-71)
    out["tetra"] = golden.tetrahedron()
    V, F = synthetic.bumpy_icosphere(2, seed=5)
    F = synthetic.delete_faces(F, 0.08, seed=7).copy()
    F[:5] = F[:5, [0, 2, 1]]                                  # inconsistent orientation
    extra = np.array([[0.0, 0.0, 5.0]])                       # an unreferenced vertex
    V = np.concatenate([V, extra])
    F = np.concatenate([F, [[3, 3, 9], [4, 4, 4], [10, 11, 10]], F[20:23]])  # degenerate, repeats
    out["bumpy_s2_soup"] = (V, F)
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
    for name, (V, F) in all_cases.items():
        normals = {f"N{w}": ref_igl.per_vertex_normals(V, F, w) for w in (0, 1, 2, 3)}
        np.savez_compressed(os.path.join(HERE, f"normals_{name}.npz"), V=V, F=F, **normals)
        print(name, V.shape, F.shape, {k: float(np.abs(v).sum()) for k, v in normals.items()})


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.environ.get("REFERENCE_ROOT", ""))
