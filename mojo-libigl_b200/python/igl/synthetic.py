"""Seeded synthetic meshes and query sets for the winding-number workloads.

No public dataset is involved in this path: every workload is a bumpy
icosphere with a seeded radial displacement, queries mixed between the scaled
bounding box and a thin shell around the surface.

* ``bumpy_icosphere(s, seed)``: the icosahedron subdivided ``s`` times
  (10*4^s+2 vertices, 20*4^s faces) on the unit sphere, each vertex scaled by
  r = 1 + sum_{j=1..8} a_j sin(k_j . x + phi_j), a_j ~ U(0, 0.02),
  k_j = unit vector * U(1, 6), phi_j ~ U(0, 2 pi). Faces are oriented outward.
* ``delete_faces(F, fraction, seed)``: drop a seeded uniform subset of faces,
  giving an open mesh with fractional winding numbers.
* ``mixed_queries(V, F, n, seed, near_sigma, box_scale)``: half uniform in the
  bounding box scaled by ``box_scale``; half on a random face at a uniform
  barycentric point, offset along the face normal by N(0, near_sigma).
* ``terrain_grid(n)``: the height-field grid of the reference's closest-point
  benchmark (bench/bench.py:33-45 of lee101/mojo-libigl): n x n vertices at
  integer (x, y), z = 0.1 sin(x / 8) cos(y / 11), two faces per cell;
  n = 350 gives 243,602 faces.
"""

from __future__ import annotations

import numpy as np

_PHI = (1.0 + 5.0**0.5) / 2.0


def icosahedron() -> tuple[np.ndarray, np.ndarray]:
    V = np.array(
        [
            [-1, _PHI, 0], [1, _PHI, 0], [-1, -_PHI, 0], [1, -_PHI, 0],
            [0, -1, _PHI], [0, 1, _PHI], [0, -1, -_PHI], [0, 1, -_PHI],
            [_PHI, 0, -1], [_PHI, 0, 1], [-_PHI, 0, -1], [-_PHI, 0, 1],
        ],
        dtype=np.float64,
    )
    V /= np.linalg.norm(V, axis=1, keepdims=True)
    F = np.array(
        [
            [0, 11, 5], [0, 5, 1], [0, 1, 7], [0, 7, 10], [0, 10, 11],
            [1, 5, 9], [5, 11, 4], [11, 10, 2], [10, 7, 6], [7, 1, 8],
            [3, 9, 4], [3, 4, 2], [3, 2, 6], [3, 6, 8], [3, 8, 9],
            [4, 9, 5], [2, 4, 11], [6, 2, 10], [8, 6, 7], [9, 8, 1],
        ],
        dtype=np.int64,
    )
    return V, F


def _subdivide(V: np.ndarray, F: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    """One 1-to-4 split with shared edge midpoints projected to the sphere."""
    e = np.concatenate([F[:, [0, 1]], F[:, [1, 2]], F[:, [2, 0]]])
    lo, hi = np.minimum(e[:, 0], e[:, 1]), np.maximum(e[:, 0], e[:, 1])
    key = lo * len(V) + hi
    uniq, inv = np.unique(key, return_inverse=True)
    ulo, uhi = uniq // len(V), uniq % len(V)
    mid = 0.5 * (V[ulo] + V[uhi])
    mid /= np.linalg.norm(mid, axis=1, keepdims=True)
    m = inv.reshape(3, len(F)).T + len(V)  # midpoints of edges 01, 12, 20
    a, b, c = F[:, 0], F[:, 1], F[:, 2]
    m01, m12, m20 = m[:, 0], m[:, 1], m[:, 2]
    F2 = np.concatenate(
        [
            np.stack([a, m01, m20], 1),
            np.stack([b, m12, m01], 1),
            np.stack([c, m20, m12], 1),
            np.stack([m01, m12, m20], 1),
        ]
    )
    return np.concatenate([V, mid]), F2


def bumpy_icosphere(subdivisions: int, seed: int = 0) -> tuple[np.ndarray, np.ndarray]:
    V, F = icosahedron()
    for _ in range(int(subdivisions)):
        V, F = _subdivide(V, F)
    rng = np.random.default_rng(seed)
    a = rng.uniform(0.0, 0.02, size=8)
    k = rng.normal(size=(8, 3))
    k /= np.linalg.norm(k, axis=1, keepdims=True)
    k *= rng.uniform(1.0, 6.0, size=(8, 1))
    phi = rng.uniform(0.0, 2.0 * np.pi, size=8)
    r = 1.0 + (a[None, :] * np.sin(V @ k.T + phi[None, :])).sum(1)
    V = V * r[:, None]
    # Outward orientation: the normal of each face points away from the origin.
    tri = V[F]
    n = np.cross(tri[:, 1] - tri[:, 0], tri[:, 2] - tri[:, 0])
    flip = (n * tri.mean(1)).sum(1) < 0
    F = F.copy()
    F[flip] = F[flip][:, [0, 2, 1]]
    return np.ascontiguousarray(V), np.ascontiguousarray(F)


def delete_faces(F: np.ndarray, fraction: float, seed: int = 0) -> np.ndarray:
    if fraction <= 0:
        return F
    rng = np.random.default_rng(seed)
    keep = np.ones(len(F), dtype=bool)
    keep[rng.choice(len(F), size=int(round(fraction * len(F))), replace=False)] = False
    return np.ascontiguousarray(F[keep])


def near_surface_points(V, F, n: int, seed: int, sigma: float) -> np.ndarray:
    rng = np.random.default_rng(seed)
    fi = rng.integers(0, len(F), size=n)
    u = rng.uniform(size=(n, 2))
    flip = u.sum(1) > 1.0
    u[flip] = 1.0 - u[flip]
    tri = V[F[fi]]
    p = tri[:, 0] + u[:, :1] * (tri[:, 1] - tri[:, 0]) + u[:, 1:] * (tri[:, 2] - tri[:, 0])
    nrm = np.cross(tri[:, 1] - tri[:, 0], tri[:, 2] - tri[:, 0])
    length = np.linalg.norm(nrm, axis=1, keepdims=True)
    nrm = np.where(length > 0, nrm / np.where(length > 0, length, 1.0), 0.0)  # zero-area: no offset
    return p + nrm * rng.normal(0.0, sigma, size=(n, 1))


def box_points(V, n: int, seed: int, scale: float = 1.2) -> np.ndarray:
    rng = np.random.default_rng(seed)
    lo, hi = V.min(0), V.max(0)
    c, h = 0.5 * (lo + hi), 0.5 * (hi - lo) * scale
    return rng.uniform(c - h, c + h, size=(n, 3))


def mixed_queries(V, F, n: int, seed: int = 1, near_sigma: float = 1e-3,
                  box_scale: float = 1.2) -> np.ndarray:
    """``n`` queries: the first half in the box, the second half near the surface."""
    nb = n // 2
    box = box_points(V, nb, seed, box_scale)
    near = near_surface_points(V, F, n - nb, seed + 7919, near_sigma)
    return np.ascontiguousarray(np.concatenate([box, near]))


def terrain_grid(n: int) -> tuple[np.ndarray, np.ndarray]:
    y, x = np.mgrid[:n, :n]
    z = 0.1 * np.sin(x / 8.0) * np.cos(y / 11.0)
    V = np.ascontiguousarray(np.column_stack((x.ravel(), y.ravel(), z.ravel())), dtype=np.float64)
    cell = (np.arange(n - 1)[:, None] * n + np.arange(n - 1)[None, :]).ravel()
    F = np.empty((2 * len(cell), 3), dtype=np.int64)
    F[0::2] = np.column_stack((cell, cell + 1, cell + n + 1))
    F[1::2] = np.column_stack((cell, cell + n + 1, cell + n))
    return V, F


# The five workloads of this path, by name; sizes as stated in each docstring.
def workload(name: str, n_queries: int | None = None):
    """Return (V, F, O, description) for a named workload.

    c1_cpu:   s=3 closed (642 V, 1280 F); 4096 Q uniform in [-1.5, 1.5]^3.
    c2_open:  s=5 (10,242 V, 20,480 F), 8% faces deleted; 2^20 Q, 50/50 with
              near offset N(0, 1e-3), box 1.2x.
    c3_mixed: s=7 closed (163,842 V, 327,680 F); 2^20 Q, 50/50, near N(0, 1e-4).
    c4_grad:  the c2 mesh; 262,144 near-surface Q, offset N(0, 1e-3).
    c3_open:  the c3 mesh with 8% of its faces deleted (301,466 F, open: about
              72k boundary edges); 2^20 Q, 50/50, near N(0, 1e-4).
    c3_soup:  the c3 mesh as a triangle soup: every face has its own three
              vertices (983,040 V, 327,680 F), so every edge is a boundary edge
              of the indexed mesh; the c3 queries.
    """
    if name == "c1_cpu":
        V, F = bumpy_icosphere(3, seed=11)
        n = 4096 if n_queries is None else n_queries
        O = np.random.default_rng(12).uniform(-1.5, 1.5, size=(n, 3))
        return V, F, O, "bumpy icosphere s=3 closed, 1280 F x %d Q uniform [-1.5,1.5]^3" % n
    if name == "c2_open":
        V, F = bumpy_icosphere(5, seed=21)
        F = delete_faces(F, 0.08, seed=22)
        n = (1 << 20) if n_queries is None else n_queries
        O = mixed_queries(V, F, n, seed=23, near_sigma=1e-3)
        return V, F, O, "bumpy icosphere s=5, 8%% faces deleted (%d F) x %d Q 50/50 box/near(1e-3)" % (len(F), n)
    if name == "c3_mixed":
        V, F = bumpy_icosphere(7, seed=31)
        n = (1 << 20) if n_queries is None else n_queries
        O = mixed_queries(V, F, n, seed=33, near_sigma=1e-4)
        return V, F, O, "bumpy icosphere s=7 closed, 327,680 F x %d Q 50/50 box/near(1e-4)" % n
    if name == "c4_grad":
        V, F = bumpy_icosphere(5, seed=21)
        F = delete_faces(F, 0.08, seed=22)
        n = 262144 if n_queries is None else n_queries
        O = near_surface_points(V, F, n, seed=43, sigma=1e-3)
        return V, F, O, "c2 mesh (%d F) x %d near-surface Q (1e-3)" % (len(F), n)
    if name == "c3_open":
        V, F = bumpy_icosphere(7, seed=31)
        F = delete_faces(F, 0.08, seed=32)
        n = (1 << 20) if n_queries is None else n_queries
        O = mixed_queries(V, F, n, seed=33, near_sigma=1e-4)
        return V, F, O, ("bumpy icosphere s=7, 8%% faces deleted (%d F, open) x %d Q 50/50 "
                         "box/near(1e-4)" % (len(F), n))
    if name == "c3_soup":
        V, F = bumpy_icosphere(7, seed=31)
        n = (1 << 20) if n_queries is None else n_queries
        O = mixed_queries(V, F, n, seed=33, near_sigma=1e-4)
        Vs, Fs = unshare_vertices(V, F)
        return Vs, Fs, O, ("c3 mesh as a triangle soup (%d V, %d F, every face its own "
                           "vertices) x %d Q 50/50 box/near(1e-4)" % (len(Vs), len(Fs), n))
    raise ValueError(f"unknown workload {name!r}")


def unshare_vertices(V: np.ndarray, F: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    """The same triangles as a soup: face f gets vertices 3f, 3f+1, 3f+2."""
    Vs = np.ascontiguousarray(V[F].reshape(-1, 3))
    Fs = np.arange(3 * len(F), dtype=np.int64).reshape(-1, 3)
    return Vs, Fs


def batched_workload(n_meshes: int = 64, seed: int = 51, max_queries: int = 1 << 20,
                     min_level: int = 2, max_level: int = 7):
    """64 uneven meshes: level U{2..7}, 0-10% faces deleted, Q log-uniform in
    [1024, 2^20] with a 50/50 box/near mix (near offset N(0, 1e-3))."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n_meshes):
        level = int(rng.integers(min_level, max_level + 1))
        frac = float(rng.uniform(0.0, 0.10))
        nq = int(np.exp(rng.uniform(np.log(1024), np.log(max_queries))))
        V, F = bumpy_icosphere(level, seed=1000 + i)
        F = delete_faces(F, frac, seed=2000 + i)
        O = mixed_queries(V, F, nq, seed=3000 + i, near_sigma=1e-3)
        out.append((V, F, O))
    return out
