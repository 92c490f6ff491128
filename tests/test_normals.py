"""Per-vertex normals on the CPU: reference-generated golden fixtures and an
independent numpy restatement.

The fixtures (tests/golden/make_golden_normals.py) come from the reference's
own Python ``per_vertex_normals`` over the oracle's C restatement of
src/capi.mojo:146-202: the reference tests' grid, the tetrahedron, and a soup
with flipped, degenerate, repeated-corner and duplicated faces and an
unreferenced vertex. Uniform and area normals must match bit for bit; angle
normals too on the CPU (the same C library acos).
"""

import glob
import os

import numpy as np
import pytest

import igl
from conftest import GOLDEN, grid

CASES = sorted(os.path.basename(p)[8:-4] for p in glob.glob(os.path.join(GOLDEN, "normals_*.npz")))


def _golden(name):
    data = np.load(os.path.join(GOLDEN, f"normals_{name}.npz"))
    return {k: data[k] for k in data.files}


def _numpy_normals(V, F, mode):
    """Independent restatement: np.add.at adds in index order, like the loop."""
    mode = 1 if mode == 3 else mode
    A, B, C = V[F[:, 0]], V[F[:, 1]], V[F[:, 2]]
    ab, ac = B - A, C - A
    n = np.stack([ab[:, 1] * ac[:, 2] - ab[:, 2] * ac[:, 1],
                  ab[:, 2] * ac[:, 0] - ab[:, 0] * ac[:, 2],
                  ab[:, 0] * ac[:, 1] - ab[:, 1] * ac[:, 0]], 1)
    norm = np.sqrt((n[:, 0] * n[:, 0] + n[:, 1] * n[:, 1]) + n[:, 2] * n[:, 2])
    keep = norm > 1e-30
    u = np.where(keep[:, None], n / np.where(keep, norm, 1.0)[:, None], 0.0)
    out = np.zeros((len(V), 3))
    rows, contrib = [], []
    for corner in range(3):
        if mode == 0:
            w = np.ones(len(F))
        elif mode == 1:
            w = norm
        else:
            P = V[F]
            vi, vj, vk = P[:, corner], P[:, (corner + 1) % 3], P[:, (corner + 2) % 3]
            e1, e2 = vj - vi, vk - vi
            l1 = np.sqrt((e1[:, 0] ** 2 + e1[:, 1] ** 2) + e1[:, 2] ** 2)
            l2 = np.sqrt((e2[:, 0] ** 2 + e2[:, 1] ** 2) + e2[:, 2] ** 2)
            with np.errstate(invalid="ignore", divide="ignore"):  # degenerate rows, masked below
                cos = ((e1[:, 0] * e2[:, 0] + e1[:, 1] * e2[:, 1]) + e1[:, 2] * e2[:, 2]) / (l1 * l2)
            w = np.arccos(np.clip(cos, -1.0, 1.0))
        rows.append(F[:, corner])
        contrib.append(u * w[:, None])
    order = np.arange(3 * len(F)).reshape(3, -1).T.ravel()  # face-major, corner-minor
    rows = np.concatenate(rows)[order]
    contrib = np.concatenate(contrib)[order]
    keep3 = np.repeat(keep, 3)
    for axis in range(3):
        np.add.at(out[:, axis], rows[keep3], contrib[keep3, axis])
    length = np.sqrt((out[:, 0] ** 2 + out[:, 1] ** 2) + out[:, 2] ** 2)
    big = length > 1e-30
    out[big] /= length[big, None]
    return out


@pytest.mark.parametrize("name", CASES)
@pytest.mark.parametrize("weighting", [0, 1, 2, 3])
def test_matches_reference_golden(oracle_mod, name, weighting):
    g = _golden(name)
    expected = g[f"N{weighting}"]
    assert igl.per_vertex_normals(g["V"], g["F"], weighting).tobytes() == expected.tobytes()
    assert oracle_mod.per_vertex_normals(g["V"], g["F"], weighting).tobytes() == expected.tobytes()
    independent = _numpy_normals(g["V"], g["F"], weighting)
    if weighting == 2:
        assert np.abs(independent - expected).max() <= 1e-14
    else:
        assert independent.tobytes() == expected.tobytes()


def test_known_answers():
    V, F = grid(7, curved=False)  # flat grid: every normal is +z
    for w in (0, 1, 2, 3):
        N = igl.per_vertex_normals(V, F, w)
        assert np.array_equal(N, np.tile([0.0, 0.0, 1.0], (len(V), 1)))
    V, F = igl.synthetic.bumpy_icosphere(3, seed=2)
    N = igl.per_vertex_normals(V, F, igl.PER_VERTEX_NORMALS_WEIGHTING_TYPE_ANGLE)
    assert np.abs(np.linalg.norm(N, axis=1) - 1).max() < 1e-14
    assert np.all((N * V).sum(1) > 0.9 * np.linalg.norm(V, axis=1))  # outward


def test_contracts():
    V, F = grid(3)
    with pytest.raises(ValueError):
        igl.per_vertex_normals(V[:, :2], F)
    with pytest.raises(ValueError):
        igl.per_vertex_normals(V, F, 4)
    with pytest.raises(TypeError):
        igl.per_vertex_normals(V, F, 1.5)
    with pytest.raises(NotImplementedError):
        igl.per_vertex_normals(V, F, FN=np.zeros((len(F), 3)))
    with pytest.raises(ValueError):
        igl.per_vertex_normals(V, F, device="tpu")
    assert np.array_equal(igl.per_vertex_normals(V, np.zeros((0, 3), np.int64)), np.zeros_like(V))
    assert list(igl.PerVertexNormalsWeightingType) == [0, 1, 2, 3]
