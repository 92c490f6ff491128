"""The reference's own Python package driving this library (the drop-in claim).

With ``MOJO_LIBIGL_REFERENCE`` set to a checkout of the reference, a child
process imports the reference's unmodified ``igl`` package with
``MOJO_LIBIGL_LIB`` pointing at this library's ``libwn_b200.so`` and runs its
CPU entry points (winding numbers over its own thread fan-out, the AABB
closest-point query, per-vertex normals); the results must equal this
package's own calls: bitwise for closest points and normals (the same host
code under the same spans), within 1e-14 for winding numbers. Skipped when the
variable is unset (the checkout is not needed anywhere else).
"""

import json
import os
import subprocess
import sys

import numpy as np
import pytest

import igl
from conftest import ROOT

CHILD = r"""
import json, sys
import numpy as np
sys.path.insert(0, sys.argv[1])
import igl
assert igl.__file__.startswith(sys.argv[1]), igl.__file__
d = np.load(sys.argv[2])
V, F, O, P = d["V"], d["F"], d["O"], d["P"]
W = igl.winding_number(V, F, O)
tree = igl.AABB()
tree.init(V, F)
sqrd, index, closest = tree.squared_distance(V, F, P)
N = igl.per_vertex_normals(V, F)
np.savez(sys.argv[3], W=W, sqrd=sqrd, index=index, closest=closest, N=N)
print(json.dumps({"lib": igl._lib.LIB}))
"""


def test_reference_shim_runs_on_this_library(tmp_path):
    reference = os.environ.get("MOJO_LIBIGL_REFERENCE")
    if not reference or not os.path.isdir(os.path.join(reference, "python", "igl")):
        pytest.skip("MOJO_LIBIGL_REFERENCE does not name a checkout of the reference")
    from igl import _lib

    V, F = igl.synthetic.terrain_grid(40)
    rng = np.random.default_rng(3)
    O = np.concatenate([rng.uniform([-1, -1, -1], [40, 40, 1], size=(3000, 3)), V[:50]])
    P = rng.uniform([-2, -2, -2], [41, 41, 2], size=(2000, 3))
    np.savez(tmp_path / "in.npz", V=V, F=F, O=O, P=P)
    env = dict(os.environ, MOJO_LIBIGL_LIB=_lib.build())
    env.pop("PYTHONPATH", None)
    out = subprocess.run([sys.executable, "-c", CHILD, os.path.join(reference, "python"),
                          str(tmp_path / "in.npz"), str(tmp_path / "out.npz")],
                         env=env, capture_output=True, text=True, timeout=600, cwd=tmp_path)
    assert out.returncode == 0, out.stderr[-2000:]
    assert json.loads(out.stdout.strip().splitlines()[-1])["lib"] == _lib.build()
    got = np.load(tmp_path / "out.npz")
    assert np.abs(got["W"] - igl.winding_number(V, F, O)).max() <= 1e-14
    sqrd, index, closest = igl.point_mesh_squared_distance(P, V, F)
    assert np.array_equal(got["sqrd"], sqrd)
    assert np.array_equal(got["index"], index)
    assert np.array_equal(got["closest"], closest)
    assert np.array_equal(got["N"], igl.per_vertex_normals(V, F))


GPU_CHILD = r"""
import ctypes, json, sys
import numpy as np
sys.path.insert(0, sys.argv[1])
import igl
assert igl.__file__.startswith(sys.argv[1]), igl.__file__
counter = ctypes.CDLL(igl._lib.LIB).wn_launch_count
counter.restype = ctypes.c_int64
d = np.load(sys.argv[2])
out = {}
launched = []
for name in d["names"]:
    before = counter()
    out[str(name)] = igl.winding_number(d[name + "_V"], d[name + "_F"], d[name + "_O"],
                                        device="gpu")
    launched.append(int(counter() - before))
np.savez(sys.argv[3], **out)
print(json.dumps({"lib": igl._lib.LIB, "launched": launched}))
"""


@pytest.mark.gpu
def test_reference_shim_gpu_branch_runs_on_this_library(tmp_path, gpu_required, oracle_mod):
    """The reference's ``winding_number(..., device="gpu")`` (its GPU branch,
    python/igl/__init__.py:251-263 there, calling ``mli_winding_gpu``) on this
    library: every call launches this library's kernels and matches the oracle
    within 1e-12 on the golden cases and a subset of the open c2 workload."""
    reference = os.environ.get("MOJO_LIBIGL_REFERENCE")
    if not reference or not os.path.isdir(os.path.join(reference, "python", "igl")):
        pytest.skip("MOJO_LIBIGL_REFERENCE does not name a checkout of the reference")
    from conftest import GOLDEN_CASES, load_golden
    from igl import _lib

    cases = {}
    for name in GOLDEN_CASES:
        g = load_golden(name)
        cases[name] = (g["V"], g["F"], g["O"])
    V2, F2, O2, _ = igl.synthetic.workload("c2_open", n_queries=4096)
    cases["c2_open_4096"] = (V2, F2, O2)
    arrays = {"names": np.array(sorted(cases))}
    for name, (V, F, O) in cases.items():
        arrays.update({name + "_V": V, name + "_F": F, name + "_O": O})
    np.savez(tmp_path / "in.npz", **arrays)
    env = dict(os.environ, MOJO_LIBIGL_LIB=_lib.build())
    env.pop("PYTHONPATH", None)
    out = subprocess.run([sys.executable, "-c", GPU_CHILD, os.path.join(reference, "python"),
                          str(tmp_path / "in.npz"), str(tmp_path / "out.npz")],
                         env=env, capture_output=True, text=True, timeout=600, cwd=tmp_path)
    assert out.returncode == 0, out.stderr[-2000:]
    info = json.loads(out.stdout.strip().splitlines()[-1])
    assert info["lib"] == _lib.build()
    assert all(n > 0 for n in info["launched"]), info
    got = np.load(tmp_path / "out.npz")
    for name, (V, F, O) in cases.items():
        ref = oracle_mod.winding_number(V, F, O)
        assert np.abs(got[name] - ref).max() <= 1e-12, name
