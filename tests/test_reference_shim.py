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
