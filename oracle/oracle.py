"""ORACLE — test infrastructure only; never imported by the product package.

Python driver for ``liboracle_wn.so`` (the C++ restatement of the reference's
``winding_one``/``winding``, src/capi.mojo:205-294) plus two independent
checkers that pin it:

* ``winding_number`` mirrors the reference's CPU call path
  (python/igl/__init__.py:232-279): SoA repack
  ``vertices[faces].transpose(1, 2, 0).reshape(9, nf)`` (248-250) and a
  ``ThreadPoolExecutor`` fan-out over contiguous query spans
  (python/igl/_lib.py:53-95; ctypes releases the GIL, so spans run in parallel).
* ``winding_number_mp`` evaluates the same solid-angle sum in mpmath at 40
  significant digits, independent of any float64 rounding: the known-answer pin.
* ``winding_grad_torch`` is the FP64 PyTorch-autograd expression of the
  solid-angle formula, the reference for the hand-written adjoint.
* ``fast_winding_number`` restates the hierarchical winding number of Barill
  et al. 2018 (not in the reference; checked against the exact sum above).
* ``per_vertex_normals`` drives the C restatement of the reference's vertex
  normals (src/capi.mojo:146-202, normals_oracle.cpp).
* ``build_aabb`` restates the reference's median-split hierarchy
  (python/igl/__init__.py:286-319) and ``aabb_squared_distance`` drives the C
  restatement of its closest-point traversal (src/capi.mojo:401-586,
  aabb_oracle.cpp).

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
and ``--impl reference`` legs may import this module.
"""

from __future__ import annotations

import ctypes
import os
import subprocess
from concurrent.futures import ThreadPoolExecutor

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "liboracle_wn.so")
I64 = ctypes.c_int64

_handle = None


def build() -> str:
    """Compile the oracle library with its Makefile (gcc only)."""
    proc = subprocess.run(["make", "-s", "-C", HERE], capture_output=True, text=True)
    if proc.returncode or not os.path.exists(LIB_PATH):
        raise RuntimeError("oracle build failed: " + (proc.stderr or proc.stdout))
    return LIB_PATH


def lib() -> ctypes.CDLL:
    global _handle
    if _handle is None:
        if not os.path.exists(LIB_PATH):
            build()
        handle = ctypes.CDLL(LIB_PATH)
        handle.mli_winding.argtypes = [I64] * 7
        handle.mli_winding.restype = None
        handle.oracle_pair_terms.argtypes = [
            ctypes.c_void_p, I64, I64, ctypes.c_void_p, ctypes.c_void_p
        ]
        handle.oracle_pair_terms.restype = None
        handle.mli_aabb_squared_distance.argtypes = [I64] * 14
        handle.mli_aabb_squared_distance.restype = None
        handle.mli_vertex_normals.argtypes = [I64] * 6
        handle.mli_vertex_normals.restype = None
        handle.oracle_closest_point.argtypes = [ctypes.c_void_p] * 3
        handle.oracle_closest_point.restype = None
        handle.oracle_isa.argtypes = []
        handle.oracle_isa.restype = ctypes.c_int
        _handle = handle
    return _handle


def isa() -> str:
    """Vector ISA of the winding kernel's clone on this host (AVX-512 or AVX2)."""
    return "AVX-512" if lib().oracle_isa() == 512 else "AVX2"


def soa(V: np.ndarray, F: np.ndarray) -> np.ndarray:
    """Triangle-soup SoA, row ``3*corner+axis`` (python/igl/__init__.py:248-250)."""
    V = np.ascontiguousarray(V, dtype=np.float64)
    F = np.ascontiguousarray(F, dtype=np.int64)
    return np.ascontiguousarray(V[F].transpose(1, 2, 0).reshape(9, len(F)))


def spans(total: int, parts: int) -> list[tuple[int, int]]:
    """Contiguous near-equal spans, as python/igl/_lib.py:64-69."""
    step = -(-total // parts)
    return [(lo, min(lo + step, total)) for lo in range(0, total, step) if lo < total]


def winding_soa(tri: np.ndarray, O: np.ndarray, workers: int = 1) -> np.ndarray:
    """Oracle winding numbers for a (9, nf) SoA soup and (nq, 3) queries."""
    tri = np.ascontiguousarray(tri, dtype=np.float64)
    O = np.ascontiguousarray(O, dtype=np.float64).reshape(-1, 3)
    nf = tri.shape[1] if tri.ndim == 2 else 0
    nq = len(O)
    out = np.empty(nq, dtype=np.float64)
    if nq == 0:
        return out
    fn = lib().mli_winding
    args = (tri.ctypes.data, O.ctypes.data, out.ctypes.data, nf, nq)
    workers = max(1, min(int(workers), nq))
    if workers == 1:
        fn(*args, 0, nq)
    else:
        with ThreadPoolExecutor(max_workers=workers) as pool:
            list(pool.map(lambda s: fn(*args, s[0], s[1]), spans(nq, workers)))
    return out


def winding_number(V, F, O, workers: int = 1) -> np.ndarray:
    return winding_soa(soa(V, F), O, workers)


def pair_terms(tri: np.ndarray, fi: int, o) -> tuple[float, float, float]:
    """(det, denom, atan2) of one pair, exactly as the oracle computes it."""
    tri = np.ascontiguousarray(tri, dtype=np.float64)
    o = np.ascontiguousarray(o, dtype=np.float64)
    out = np.empty(3, dtype=np.float64)
    lib().oracle_pair_terms(tri.ctypes.data, tri.shape[1], int(fi), o.ctypes.data,
                            out.ctypes.data)
    return float(out[0]), float(out[1]), float(out[2])


def winding_number_mp(V, F, O, dps: int = 40) -> np.ndarray:
    """High-precision solid-angle sum (pure Python; small cases only)."""
    import mpmath

    old = mpmath.mp.dps
    mpmath.mp.dps = dps
    try:
        V = [[mpmath.mpf(float(x)) for x in row] for row in np.asarray(V, dtype=np.float64)]
        F = np.asarray(F, dtype=np.int64)
        res = []
        for o in np.asarray(O, dtype=np.float64).reshape(-1, 3):
            ox, oy, oz = (mpmath.mpf(float(x)) for x in o)
            total = mpmath.mpf(0)
            for f in F:
                a = [V[f[0]][k] - (ox, oy, oz)[k] for k in range(3)]
                b = [V[f[1]][k] - (ox, oy, oz)[k] for k in range(3)]
                c = [V[f[2]][k] - (ox, oy, oz)[k] for k in range(3)]
                la = mpmath.sqrt(sum(x * x for x in a))
                lb = mpmath.sqrt(sum(x * x for x in b))
                lc = mpmath.sqrt(sum(x * x for x in c))
                det = (a[0] * (b[1] * c[2] - b[2] * c[1]) - a[1] * (b[0] * c[2] - b[2] * c[0])
                       + a[2] * (b[0] * c[1] - b[1] * c[0]))
                dot = lambda u, v: u[0] * v[0] + u[1] * v[1] + u[2] * v[2]  # noqa: E731
                denom = la * lb * lc + dot(a, b) * lc + dot(b, c) * la + dot(c, a) * lb
                total += mpmath.atan2(det, denom)
            res.append(float(total / (2 * mpmath.pi)))
        return np.asarray(res, dtype=np.float64)
    finally:
        mpmath.mp.dps = old


def winding_torch(V, F, O):
    """FP64 torch expression of the same sum (differentiable in V and O)."""
    import torch

    tri = V[F]  # (nf, 3 corners, 3)
    a = tri[None, :, 0, :] - O[:, None, :]
    b = tri[None, :, 1, :] - O[:, None, :]
    c = tri[None, :, 2, :] - O[:, None, :]
    la, lb, lc = a.norm(dim=-1), b.norm(dim=-1), c.norm(dim=-1)
    det = (a * torch.cross(b, c, dim=-1)).sum(-1)
    denom = (la * lb * lc + (a * b).sum(-1) * lc + (b * c).sum(-1) * la
             + (c * a).sum(-1) * lb)
    return torch.atan2(det, denom).sum(-1) / (2 * np.pi)


def winding_grad_torch(V, F, O, gW):
    """(dL/dO, dL/dV) of L = sum(gW * W) by FP64 torch autograd."""
    import torch

    Vt = torch.tensor(np.asarray(V, dtype=np.float64), requires_grad=True)
    Ot = torch.tensor(np.asarray(O, dtype=np.float64), requires_grad=True)
    Ft = torch.tensor(np.asarray(F, dtype=np.int64))
    W = winding_torch(Vt, Ft, Ot)
    (W * torch.tensor(np.asarray(gW, dtype=np.float64))).sum().backward()
    return Ot.grad.numpy(), Vt.grad.numpy()


# ---- closest points (the reference's AABB path) -----------------------------
def build_aabb(V, F, leaf_size: int = 8):
    """Median-split hierarchy as python/igl/__init__.py:286-319 builds it.

    Returns (boxes (nnodes, 6) f64, nodes (nnodes, 4) int64, order (nf,) int64,
    stack_size). Nodes are numbered in preorder (a node before its left
    subtree, the left subtree before the right one). A node with more than
    ``leaf_size`` faces splits along the axis of the largest extent of its face
    box centres (the first such axis), after a stable sort of its faces by that
    centre coordinate, at len // 2. ``stack_size`` is the depth (root = 1) + 1.
    """
    V = np.ascontiguousarray(V, dtype=np.float64)
    F = np.ascontiguousarray(F, dtype=np.int64)
    tri = V[F]
    low, high = tri.min(axis=1), tri.max(axis=1)
    centers = 0.5 * (low + high)
    boxes, nodes, order = [], [], []
    depth = 0
    # Explicit preorder walk: (face ids, depth, slot in the parent to patch).
    work = [(np.arange(len(F), dtype=np.int64), 1, None)]
    while work:
        ids, d, parent = work.pop()
        node = len(nodes)
        depth = max(depth, d)
        if parent is not None:
            nodes[parent[0]][parent[1]] = node
        boxes.append(np.concatenate((low[ids].min(axis=0), high[ids].max(axis=0))))
        if len(ids) <= leaf_size:
            nodes.append([-1, -1, len(order), len(ids)])
            order.extend(ids.tolist())
            continue
        nodes.append([-1, -1, 0, 0])
        c = centers[ids]
        axis = int(np.argmax(c.max(axis=0) - c.min(axis=0)))
        ids = ids[np.argsort(c[:, axis], kind="stable")]
        half = len(ids) // 2
        work.append((ids[half:], d + 1, (node, 1)))  # right, popped after the left subtree
        work.append((ids[:half], d + 1, (node, 0)))
    return (np.ascontiguousarray(boxes, dtype=np.float64).reshape(-1, 6),
            np.ascontiguousarray(nodes, dtype=np.int64).reshape(-1, 4),
            np.asarray(order, dtype=np.int64), depth + 1)


def aabb_squared_distance(P, V, F, tree=None, workers: int = 1):
    """(sqrd, face index, closest point) of each point, by the C oracle.

    ``tree`` is a ``build_aabb`` result (built here when omitted). Spans of
    points run on ``workers`` threads, each with its own traversal stack.
    """
    P = np.ascontiguousarray(P, dtype=np.float64).reshape(-1, 3)
    V = np.ascontiguousarray(V, dtype=np.float64)
    F = np.ascontiguousarray(F, dtype=np.int64)
    n = len(P)
    if len(F) == 0:
        return np.full(n, np.inf), np.full(n, -1, dtype=np.int64), np.zeros((n, 3))
    boxes, nodes, order, stack_size = build_aabb(V, F) if tree is None else tree
    sqrd = np.empty(n, dtype=np.float64)
    index = np.empty(n, dtype=np.int64)
    closest = np.empty((n, 3), dtype=np.float64)
    if n == 0:
        return sqrd, index, closest
    workers = max(1, min(int(workers), n))
    stacks = np.empty((workers, stack_size), dtype=np.int64)
    fn = lib().mli_aabb_squared_distance
    args = (P.ctypes.data, V.ctypes.data, F.ctypes.data, boxes.ctypes.data, nodes.ctypes.data,
            order.ctypes.data, sqrd.ctypes.data, index.ctypes.data, closest.ctypes.data)
    parts = spans(n, workers)
    if len(parts) == 1:
        fn(*args, stacks[0].ctypes.data, n, len(nodes), 0, n)
    else:
        with ThreadPoolExecutor(max_workers=len(parts)) as pool:
            list(pool.map(lambda item: fn(*args, stacks[item[0]].ctypes.data, n, len(nodes),
                                          item[1][0], item[1][1]), enumerate(parts)))
    return sqrd, index, closest


def closest_point(p, tri9) -> tuple[float, float, float, float]:
    """(d2, x, y, z) of one point against one triangle (9 coordinates, A B C)."""
    p = np.ascontiguousarray(p, dtype=np.float64)
    tri9 = np.ascontiguousarray(tri9, dtype=np.float64).reshape(9)
    out = np.empty(4, dtype=np.float64)
    lib().oracle_closest_point(p.ctypes.data, tri9.ctypes.data, out.ctypes.data)
    return tuple(float(x) for x in out)


# ---- fast (hierarchical) winding numbers ------------------------------------
def _fwn_node_moments(V, F, faces):
    """(p, r, T0, T1, T2) of a face set: area-weighted centre, vertex radius and the
    dipole moments of Barill et al. 2018 (T1[j, i] = sum a d_j n_i,
    T2[j, k, i] = 1/2 sum a n_i (d_j d_k + C[j, k]))."""
    tri = V[F[faces]]
    an = 0.5 * np.cross(tri[:, 1] - tri[:, 0], tri[:, 2] - tri[:, 0])
    a = np.linalg.norm(an, axis=1)
    c = tri.mean(axis=1)
    area = a.sum()
    p = (a[:, None] * c).sum(0) / area if area > 0 else c.mean(0)
    r = np.sqrt(((tri.reshape(-1, 3) - p) ** 2).sum(1).max())
    d = c - p
    cov = np.einsum("tvj,tvk->tjk", tri - c[:, None], tri - c[:, None]) / 12.0
    T1 = np.einsum("tj,ti->ji", d, an)
    T2 = 0.5 * np.einsum("ti,tjk->jki", an, np.einsum("tj,tk->tjk", d, d) + cov)
    return p, r, an.sum(0), T1, T2


def _fwn_far(q, p, T0, T1, T2):
    """Second-order far-field winding number of one node at q (unfolded form)."""
    y = p - q
    s = np.sqrt(y @ y)
    u = np.einsum("iki->k", T2)
    v = np.einsum("jji->i", T2)
    t = ((T0 @ y + np.trace(T1)) / s**3 - 3.0 * (y @ T1 @ y + (2.0 * u + v) @ y) / s**5
         + 15.0 * np.einsum("jki,i,j,k->", T2, y, y, y) / s**7)
    return t / (4.0 * np.pi)


def fast_winding_number(V, F, O, beta: float = 2.0, leaf_size: int = 8):
    """Hierarchical winding number (pure Python loops: small cases only).

    Tree: build_aabb (the median-split hierarchy). Per query, depth first from
    the root, left child first: a node with |q - p|^2 > (beta r)^2 adds _fwn_far,
    a nearer leaf adds the exact winding number of its faces (this oracle's
    mli_winding), a nearer internal node is opened.
    """
    V = np.ascontiguousarray(V, dtype=np.float64)
    F = np.ascontiguousarray(F, dtype=np.int64)
    O = np.ascontiguousarray(O, dtype=np.float64).reshape(-1, 3)
    out = np.zeros(len(O))
    if len(F) == 0:
        return out
    _, nodes, order, _ = build_aabb(V, F, leaf_size)
    nn = len(nodes)
    first, last = np.zeros(nn, np.int64), np.zeros(nn, np.int64)
    for i in range(nn - 1, -1, -1):
        if nodes[i, 3] > 0:
            first[i], last[i] = nodes[i, 2], nodes[i, 2] + nodes[i, 3]
        else:
            first[i], last[i] = first[nodes[i, 0]], last[nodes[i, 1]]
    moments = [_fwn_node_moments(V, F, order[first[i]:last[i]]) for i in range(nn)]
    for qi, q in enumerate(O):
        total, stack = 0.0, [0]
        while stack:
            i = stack.pop()
            p, r, T0, T1, T2 = moments[i]
            y = p - q
            if y @ y > (beta * r) ** 2:
                total += _fwn_far(q, p, T0, T1, T2)
            elif nodes[i, 3] > 0:
                total += winding_number(V, F[order[first[i]:last[i]]], q[None])[0]
            else:
                stack += [int(nodes[i, 1]), int(nodes[i, 0])]
        out[qi] = total
    return out


# ---- per-vertex normals ------------------------------------------------------
def per_vertex_normals(V, F, weighting: int = 3) -> np.ndarray:
    """(nv, 3) normals by the C restatement of src/capi.mojo:146-202."""
    V = np.ascontiguousarray(V, dtype=np.float64)
    F = np.ascontiguousarray(F, dtype=np.int64)
    out = np.zeros((len(V), 3))
    if len(F):
        lib().mli_vertex_normals(V.ctypes.data, F.ctypes.data, out.ctypes.data, len(V), len(F),
                                 int(weighting))
    return out
