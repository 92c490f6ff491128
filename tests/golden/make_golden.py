"""Regenerate the golden winding-number fixtures in this directory.

The fixtures are produced by the REFERENCE's own Python package
(lee101/mojo-libigl ``python/igl``: validation, SoA repack and the
ThreadPoolExecutor fan-out of python/igl/__init__.py:232-279 and
python/igl/_lib.py:53-95), loaded from a read-only checkout of the reference
with ``MOJO_LIBIGL_LIB`` pointing at the CPU oracle library (the C++
restatement of src/capi.mojo:205-294, built by ``oracle/Makefile``), because
the reference's Mojo toolchain is not installable offline. Each case is also
evaluated in mpmath at 40 digits (the solid-angle sum without float64
rounding), stored beside it as ``W_mp``.

Usage (needs the reference checkout; the fixtures are committed, so tests and
the GPU host never run this):

    python tests/golden/make_golden.py /path/to/reference
"""

from __future__ import annotations

import importlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))


def grid(n=7, curved=True):
    """The reference tests' height-field grid mesh (tests/test_parity.py:12-26)."""
    V = np.array(
        [[i, j, 0.15 * np.sin(i) * np.cos(j) if curved else 0.0] for j in range(n)
         for i in range(n)],
        dtype=np.float64,
    )
    F = []
    for j in range(n - 1):
        for i in range(n - 1):
            a = j * n + i
            F.extend(((a, a + 1, a + n + 1), (a, a + n + 1, a + n)))
    return V, np.asarray(F, dtype=np.int64)


def tetrahedron():
    """The reference tests' tetrahedron (tests/test_parity.py:29-34)."""
    V = np.array([[0.0, 0.0, 0.0], [2.0, 0.0, 0.0], [0.0, 1.0, 0.0], [0.0, 0.0, 3.0]])
    F = np.array([[0, 2, 1], [0, 1, 3], [1, 2, 3], [2, 0, 3]], dtype=np.int64)
    return V, F


def cases():
    out = {}
    V, F = tetrahedron()
    out["tetra"] = (V, F, np.array([[0.1, 0.1, 0.1], [2.0, 2.0, 2.0], [-1.0, 0.2, 0.2]]))
    V, F = grid(5)
    rng = np.random.default_rng(31)
    out["simd_tail"] = (V, F[:5], rng.normal(size=(7, 3)))
    V, F = grid(10)
    out["thread_threshold"] = (V, F, rng.normal(size=(1619, 3)) + [4.5, 4.5, 0.0])
    V, F = grid(20)
    rng = np.random.default_rng(77)
    out["serial_parallel"] = (V, F, rng.uniform([0.0, 0.0, -2.0], [19.0, 19.0, 2.0],
                                                size=(512, 3)))
    # The mesh generator is loaded by path: the reference package is also `igl`.
    import importlib.util

    path = os.path.join(REPO, "mojo-libigl_b200", "python", "igl", "synthetic.py")
    spec = importlib.util.spec_from_file_location("wn_synthetic", path)
    synthetic = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(synthetic)

    V, F = synthetic.bumpy_icosphere(2, seed=5)
    out["bumpy_s2_closed"] = (V, F, synthetic.mixed_queries(V, F, 256, seed=6, near_sigma=1e-3))
    Fo = synthetic.delete_faces(F, 0.08, seed=7)
    out["bumpy_s2_open"] = (V, Fo, synthetic.mixed_queries(V, Fo, 256, seed=8, near_sigma=1e-3))
    return out


def main(reference: str) -> None:
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import oracle  # noqa: E402

    os.environ["MOJO_LIBIGL_LIB"] = oracle.build()
    all_cases = cases()
    sys.dont_write_bytecode = True
    sys.path.insert(0, os.path.join(reference, "python"))
    ref_igl = importlib.import_module("igl")
    assert os.path.realpath(ref_igl.__file__).startswith(os.path.realpath(reference)), ref_igl
    for name, (V, F, O) in all_cases.items():
        W = ref_igl.winding_number(V, F, O)
        mp_rows = O if len(O) <= 64 else O[:: max(1, len(O) // 48)]
        W_mp = oracle.winding_number_mp(V, F, mp_rows)
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), V=V, F=F, O=O, W=W,
                            O_mp=mp_rows, W_mp=W_mp)
        gap = np.abs(ref_igl.winding_number(V, F, mp_rows) - W_mp).max()
        print(name, V.shape, F.shape, O.shape, "max |W_ref - W_mp| =", float(gap))


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.environ.get("REFERENCE_ROOT", ""))
