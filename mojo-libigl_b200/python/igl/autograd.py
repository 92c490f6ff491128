"""Differentiable winding number for PyTorch tensors on a CUDA device.

``winding_number_torch(V, F, O)`` returns W (nq,) and backpropagates dL/dV and
dL/dO through the library's hand-written adjoints. Pair terms are recomputed
(nothing nq x nf is stored); every reduction runs in a fixed order.

adjoint="faces": per-face sums over the queries (``wn_backward_fp64_device`` or,
for precision="mixed", ``wn_backward_mixed_device``), then dL/dV gathered from
the per-corner face gradients through a vertex -> (face, corner) list.
adjoint="edges": the same derivative from the mesh's net boundary edges only
(``wn_backward_edges_device``, or ``wn_backward_edges_mixed_device`` after a
mixed forward): the per-face terms of a directed side and of its reverse cancel
at both endpoints, so interior edges contribute nothing (exactly zero for a
closed, consistently oriented mesh).
adjoint="welded" (mixed precision): for triangle soups, whose faces share
positions but not indices, every side is welded to the edges of equal endpoint
coordinates (``welded_edges``): one edge's terms serve all sides on it, each
side taking them with its own sign, and dL/dO only sees the edges' net counts.
adjoint="auto" (default): "edges", except after a mixed-precision forward on a
mesh with more net boundary edges than FACE_COST times its faces (a triangle
soup has three per face), where it takes "welded" or "faces", whichever has the
lower count times cost.

Tensors are plumbing here: the forward and the adjoints run in libwn_b200's
kernels on the tensors' memory and current stream.
"""

from __future__ import annotations

import ctypes

import torch

from . import _lib


# Cost of one mixed face pair in units of one mixed edge pair (on a B200, c3
# workloads x 262,144 queries: 4.97 ps per face pair, 3.07 ps per edge pair):
# "auto" takes the cheapest of the boundary edges, the edges welded by position
# and the faces by count times cost.
FACE_COST = 1.6


def _check(rc: int) -> None:
    if rc != 0:
        raise RuntimeError("libwn_b200: " + _lib.last_error())


def _stream() -> ctypes.c_void_p:
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def triangle_soa(V: torch.Tensor, F: torch.Tensor) -> tuple[torch.Tensor, int, int]:
    """(9, ld) float64 SoA, row 3*corner+axis, ld even (the C ABI's layout)."""
    nf = F.shape[0]
    ld = nf + (nf & 1)
    tri = torch.zeros((9, max(ld, 2)), dtype=torch.float64, device=V.device)
    if nf:
        tri[:, :nf] = V.to(torch.float64)[F].permute(1, 2, 0).reshape(9, nf)
    return tri, ld, nf


def vertex_csr(F: torch.Tensor, nv: int) -> tuple[torch.Tensor, torch.Tensor]:
    """Vertex -> entries 3*face+corner, grouped by vertex in a fixed order."""
    flat = F.reshape(-1).to(torch.int64)
    order = torch.argsort(flat, stable=True)
    counts = torch.bincount(flat, minlength=nv)
    indptr = torch.zeros(nv + 1, dtype=torch.int64, device=F.device)
    indptr[1:] = torch.cumsum(counts, 0)
    return indptr, order.contiguous()


def forward_fp64(tri: torch.Tensor, ld: int, nf: int, O: torch.Tensor) -> torch.Tensor:
    q = O.to(torch.float64).contiguous()
    w = torch.empty(q.shape[0], dtype=torch.float64, device=q.device)
    if q.shape[0]:
        _check(_lib.lib().wn_forward_fp64_device(tri.data_ptr(), ld, q.data_ptr(), w.data_ptr(),
                                                 nf, q.shape[0], 0, _stream()))
    return w


def use_prepared_fp64(nf: int, nq: int) -> bool:
    """The drop-in's rule (mli_winding_gpu): above 1e9 pairs the prepared-mesh
    FP64 kernel, whose ~2 ms preparation its corner reuse repays."""
    return 4096 <= nf <= 0x7FFFFFFF and float(nf) * nq >= 1e9


def forward_fp64_prepared(tri: torch.Tensor, ld: int, nf: int, O: torch.Tensor) -> torch.Tensor:
    """Plain FP64 W over a prepared mesh (Morton tiles, repeated corners reused):
    the same bit-exact pair terms as forward_fp64, summed in tile order."""
    q = O.to(torch.float64).contiguous()
    w = torch.empty(q.shape[0], dtype=torch.float64, device=q.device)
    if q.shape[0]:
        mesh = PreparedMesh(tri, ld, nf)
        try:
            _check(mesh.handle.wn_forward_fp64_mesh_device(mesh.mesh, q.data_ptr(), q.shape[0],
                                                           w.data_ptr(), _stream()))
        finally:
            mesh.close()
    return w


class PreparedMesh:
    """A mesh prepared for the mixed-precision kernels (Morton-ordered tiles)."""

    def __init__(self, tri: torch.Tensor, ld: int, nf: int, kappa: float = 4.0):
        self.handle = _lib.lib()
        self.tri, self.ld, self.nf = tri, ld, nf
        self.mesh = ctypes.c_void_p()
        _check(self.handle.wn_mixed_mesh_create(tri.data_ptr(), ld, nf, kappa, _stream(),
                                                ctypes.byref(self.mesh)))

    def forward(self, O: torch.Tensor) -> torch.Tensor:
        q = O.to(torch.float64).contiguous()
        w = torch.empty(q.shape[0], dtype=torch.float64, device=q.device)
        if q.shape[0]:
            _check(self.handle.wn_forward_mixed_device(self.mesh, q.data_ptr(), q.shape[0],
                                                       w.data_ptr(), _stream()))
        return w

    def backward(self, O: torch.Tensor, gW: torch.Tensor):
        """(dq, dtri): dL/do (nq, 3) and dL/d(corner) (9, ld) for dL/dW = gW."""
        q = O.to(torch.float64).contiguous()
        gw = gW.to(torch.float64).contiguous()
        dq = torch.empty((q.shape[0], 3), dtype=torch.float64, device=q.device)
        dtri = torch.zeros_like(self.tri)
        _check(self.handle.wn_backward_mixed_device(self.mesh, q.data_ptr(), q.shape[0],
                                                    gw.data_ptr(), dq.data_ptr(),
                                                    dtri.data_ptr(), self.ld, _stream()))
        return dq, dtri

    def close(self):
        if self.mesh:
            torch.cuda.current_stream().synchronize()
            self.handle.wn_mixed_mesh_destroy(self.mesh)
            self.mesh = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:  # interpreter shutdown
            pass


def forward_mixed(tri: torch.Tensor, ld: int, nf: int, O: torch.Tensor,
                  kappa: float = 4.0) -> torch.Tensor:
    mesh = PreparedMesh(tri, ld, nf, kappa)
    try:
        return mesh.forward(O)
    finally:
        mesh.close()


def gather_vertices(dtri, ld, nf, F, nv, corners=3):
    """dL/dV from per-element corner gradients (faces: corners=3; edges: 2)."""
    dV = torch.zeros((nv, 3), dtype=torch.float64, device=dtri.device)
    if nf and nv:
        indptr, entries = vertex_csr(F, nv)
        _check(_lib.lib().wn_gather_vertex_grad_device(dtri.data_ptr(), ld, corners,
                                                       indptr.data_ptr(), entries.data_ptr(),
                                                       nv, dV.data_ptr(), _stream()))
    return dV


def boundary_edges(V: torch.Tensor, F: torch.Tensor):
    """Undirected edges {u < v} with net multiplicity m = #(u->v) - #(v->u) != 0.

    Returns (edges (7, le) float64 SoA: V[u], V[v], m; ne; endpoints (ne, 2) int64).
    """
    nv = V.shape[0]
    e = torch.cat([F[:, [0, 1]], F[:, [1, 2]], F[:, [2, 0]]]).to(torch.int64)
    e = e[e[:, 0] != e[:, 1]]
    lo = torch.minimum(e[:, 0], e[:, 1])
    hi = torch.maximum(e[:, 0], e[:, 1])
    sign = torch.where(e[:, 0] < e[:, 1], 1, -1).to(torch.int64)
    keys, inverse = torch.unique(lo * nv + hi, return_inverse=True)
    m = torch.zeros(keys.shape[0], dtype=torch.int64, device=F.device)
    m.scatter_add_(0, inverse, sign)
    keep = m != 0
    keys, m = keys[keep], m[keep]
    ends = torch.stack([keys // nv, keys % nv], 1)
    ne = ends.shape[0]
    le = max(ne, 1)
    edges = torch.zeros((7, le), dtype=torch.float64, device=V.device)
    if ne:
        Vd = V.to(torch.float64)
        edges[0:3, :ne] = Vd[ends[:, 0]].T
        edges[3:6, :ne] = Vd[ends[:, 1]].T
        edges[6, :ne] = m.to(torch.float64)
    return edges, ne, ends


def backward_edges(V, F, O, gW, edges=None, precision: str = "fp64", kappa: float = 4.0):
    """(dL/dV, dL/dO) from the net boundary edges, in FP64 or (precision="mixed")
    FP32 far pairs with FP64 near pairs; `edges` is boundary_edges(V, F) when the
    caller has it already."""
    handle = _lib.lib()
    q = O.to(torch.float64).contiguous()
    gw = gW.to(torch.float64).contiguous()
    nq, nv = q.shape[0], V.shape[0]
    edges, ne, ends = edges if edges is not None else boundary_edges(V, F)
    le = edges.shape[1]
    dq = torch.empty((nq, 3), dtype=torch.float64, device=q.device)
    dedge = torch.zeros((6, le), dtype=torch.float64, device=q.device)
    if precision == "mixed":
        _check(handle.wn_backward_edges_mixed_device(edges.data_ptr(), le, ne, q.data_ptr(), nq,
                                                     gw.data_ptr(), kappa, 0, dq.data_ptr(),
                                                     dedge.data_ptr(), _stream()))
    else:
        _check(handle.wn_backward_edges_device(edges.data_ptr(), le, ne, q.data_ptr(), nq,
                                               gw.data_ptr(), dq.data_ptr(), dedge.data_ptr(),
                                               _stream()))
    return gather_vertices(dedge, le, ne, ends, nv, corners=2), dq


def welded_edges(V: torch.Tensor, F: torch.Tensor):
    """The sides of the faces welded by vertex position (for triangle soups).

    Every directed side a -> b of a face is keyed by its endpoints' coordinates,
    ordered so that the first is lexicographically smaller (sigma = +1 when that
    is a, -1 when it is b); sides on the same segment share one edge. Returns
    (edges (7, le) float64 SoA: the two endpoints and m = the sum of the sides'
    sigma; ng; side_edge (ns,) the edge of every kept side; sigma (ns,); ends
    (ns, 2) the sides' vertex indices a, b). Zero-length sides are dropped.
    """
    a = torch.cat([F[:, 0], F[:, 1], F[:, 2]]).to(torch.int64)
    b = torch.cat([F[:, 1], F[:, 2], F[:, 0]]).to(torch.int64)
    Vd = V.to(torch.float64)
    Pa, Pb = Vd[a], Vd[b]
    diff = Pa != Pb
    keep = diff.any(1)
    a, b, Pa, Pb, diff = a[keep], b[keep], Pa[keep], Pb[keep], diff[keep]
    first = diff.to(torch.int8).argmax(1, keepdim=True)
    sigma = torch.where(Pa.gather(1, first)[:, 0] < Pb.gather(1, first)[:, 0], 1, -1)
    lo = torch.where(sigma[:, None] > 0, Pa, Pb)
    hi = torch.where(sigma[:, None] > 0, Pb, Pa)
    ng, le = 0, 1
    if a.numel():
        uniq, side_edge = torch.unique(torch.cat([lo, hi], 1), dim=0, return_inverse=True)
        ng = uniq.shape[0]
        le = ng
    else:
        uniq = torch.zeros((0, 6), dtype=torch.float64, device=V.device)
        side_edge = torch.zeros(0, dtype=torch.int64, device=V.device)
    m = torch.zeros(max(ng, 1), dtype=torch.int64, device=V.device)
    if ng:
        m.scatter_add_(0, side_edge, sigma.to(torch.int64))
    edges = torch.zeros((7, le), dtype=torch.float64, device=V.device)
    if ng:
        edges[0:3, :ng] = uniq[:, 0:3].T
        edges[3:6, :ng] = uniq[:, 3:6].T
        edges[6, :ng] = m[:ng].to(torch.float64)
    return edges, ng, side_edge, sigma, torch.stack([a, b], 1)


def backward_welded_edges(V, F, O, gW, welded=None, kappa: float = 4.0):
    """(dL/dV, dL/dO) of a triangle soup from its sides welded by position.

    One edge stands for every directed side on its segment: the mixed edge adjoint
    sums each edge's unweighted endpoint terms once (dL/dO weighted by the net
    count m of its sides, so sides that cancel add nothing there), and every side
    a -> b takes them with its own sign: (da, db) = (dP, dQ) for sigma = +1 and
    (-dQ, -dP) for sigma = -1. The per-vertex sums then run in a fixed order. Edges
    with m = 0 add exactly nothing to dL/dO, so they go through the adjoint without
    dL/dO (a leaner kernel) and only the others (an open soup's boundary) through the
    full one; a closed soup (every m = 0) gets dL/dO = 0 from one lean launch.
    """
    handle = _lib.lib()
    q = O.to(torch.float64).contiguous()
    gw = gW.to(torch.float64).contiguous()
    nq, nv = q.shape[0], V.shape[0]
    edges, ng, side_edge, sigma, ends = welded if welded is not None else welded_edges(V, F)
    le = edges.shape[1]
    dq = torch.zeros((nq, 3), dtype=torch.float64, device=q.device)
    dedge = torch.zeros((6, le), dtype=torch.float64, device=q.device)
    cancel = edges[6, :ng] == 0
    n0 = int(cancel.sum()) if ng else 0

    def run(sub, n, with_dq, stream):
        out = torch.zeros((6, max(sub.shape[1], 1)), dtype=torch.float64, device=q.device)
        _check(handle.wn_backward_edges_mixed_device(sub.data_ptr(), sub.shape[1], n,
                                                     q.data_ptr(), nq, gw.data_ptr(), kappa, 1,
                                                     dq.data_ptr() if with_dq else None,
                                                     out.data_ptr(), stream))
        return out

    if n0 in (0, ng):  # one kind of edge only: one launch
        dedge = run(edges, ng, n0 == 0, _stream()) if ng else dedge
    else:
        # Edges whose sides cancel (m = 0) contribute nothing to dL/dO: they take
        # the kernel without it, the others (the soup's open boundary) the full one,
        # on a second stream so that the two launches overlap (separate outputs).
        i0 = torch.nonzero(cancel).flatten()
        i1 = torch.nonzero(~cancel).flatten()
        e0, e1 = edges[:, i0].contiguous(), edges[:, i1].contiguous()
        main = torch.cuda.current_stream(q.device)
        side = torch.cuda.Stream(q.device)
        side.wait_stream(main)
        with torch.cuda.stream(side):
            d1 = run(e1, ng - n0, True, ctypes.c_void_p(side.cuda_stream))
        d0 = run(e0, n0, False, _stream())
        main.wait_stream(side)
        for t in (e1, dq, q, gw):  # made on the main stream, used on the side one
            t.record_stream(side)
        d1.record_stream(main)  # made on the side stream, read below on the main one
        dedge[:, i0] = d0[:, :n0]
        dedge[:, i1] = d1[:, :ng - n0]
    ns = ends.shape[0]
    dside = torch.zeros((6, max(ns, 1)), dtype=torch.float64, device=q.device)
    if ns:
        de = dedge[:, side_edge]
        pos = (sigma > 0)[None, :]
        dside[0:3, :ns] = torch.where(pos, de[0:3], -de[3:6])
        dside[3:6, :ns] = torch.where(pos, de[3:6], -de[0:3])
    return gather_vertices(dside, max(ns, 1), ns, ends, nv, corners=2), dq


def backward_fp64(tri, ld, nf, O, gW, F, nv):
    """(dL/dV, dL/dO) for L with dL/dW = gW."""
    handle = _lib.lib()
    q = O.to(torch.float64).contiguous()
    gw = gW.to(torch.float64).contiguous()
    nq = q.shape[0]
    dq = torch.empty((nq, 3), dtype=torch.float64, device=q.device)
    dtri = torch.empty_like(tri)
    _check(handle.wn_backward_fp64_device(tri.data_ptr(), ld, nf, q.data_ptr(), nq,
                                          gw.data_ptr(), dq.data_ptr(), dtri.data_ptr(),
                                          _stream()))
    return gather_vertices(dtri, ld, nf, F, nv), dq


class WindingNumberFunction(torch.autograd.Function):
    """W = winding_number(V, F, O) with the library's adjoint as backward."""

    @staticmethod
    def forward(ctx, V, F, O, precision="fp64", adjoint="edges"):
        tri, ld, nf = triangle_soa(V, F)
        ctx.mesh = None
        if precision == "mixed":
            mesh = PreparedMesh(tri, ld, nf)
            w = mesh.forward(O)
            if adjoint in ("faces", "auto", "welded"):
                ctx.mesh = mesh
            else:
                mesh.close()
        elif use_prepared_fp64(nf, O.shape[0]):
            w = forward_fp64_prepared(tri, ld, nf, O)
        else:
            w = forward_fp64(tri, ld, nf, O)
        ctx.save_for_backward(V, F, O)
        ctx.tri, ctx.ld, ctx.nf, ctx.adjoint = tri, ld, nf, adjoint
        ctx.precision = precision
        return w.to(O.dtype)

    @staticmethod
    def backward(ctx, gW):
        V, F, O = ctx.saved_tensors
        adjoint = ctx.adjoint
        edges = None
        welded = None
        if adjoint == "auto":
            edges = boundary_edges(V, F)
            adjoint = "edges"
            if ctx.mesh is not None and edges[1] > FACE_COST * ctx.nf:
                welded = welded_edges(V, F)
                adjoint = "welded" if welded[1] < FACE_COST * ctx.nf else "faces"
            if adjoint != "faces" and ctx.mesh is not None:
                ctx.mesh.close()
                ctx.mesh = None
        if adjoint == "edges":
            dV, dq = backward_edges(V, F, O, gW, edges, precision=ctx.precision)
        elif adjoint == "welded":
            dV, dq = backward_welded_edges(V, F, O, gW, welded)
            if ctx.mesh is not None:
                ctx.mesh.close()
                ctx.mesh = None
        elif ctx.mesh is not None:
            dq, dtri = ctx.mesh.backward(O, gW)
            dV = gather_vertices(dtri, ctx.ld, ctx.nf, F, V.shape[0])
            ctx.mesh.close()
        else:
            dV, dq = backward_fp64(ctx.tri, ctx.ld, ctx.nf, O, gW, F, V.shape[0])
        return dV.to(V.dtype), None, dq.to(O.dtype), None, None


def winding_number_torch(V: torch.Tensor, F: torch.Tensor, O: torch.Tensor,
                         precision: str | None = None, adjoint: str = "auto") -> torch.Tensor:
    """Differentiable W for CUDA tensors V (nv,3), F (nf,3) int, O (nq,3).

    precision: "fp64" (plain FP64 forward and adjoint) or "mixed" (FP32 pairs with
    FP64 refinement of near-surface pairs, forward and adjoint); by default
    "mixed" for float32 queries and "fp64" otherwise. W has the dtype of O.
    adjoint: "edges" (net boundary edges), "faces" (per-face reduction), both in
    the forward's precision, "welded" (mixed only: the sides welded by position,
    for triangle soups whose faces share coordinates but not indices) or "auto"
    (the cheapest of these); all give the same derivative.
    """
    if precision is None:
        precision = "mixed" if O.dtype == torch.float32 else "fp64"
    if not (V.is_cuda and F.is_cuda and O.is_cuda):
        raise RuntimeError("winding_number_torch needs CUDA tensors (no CPU fallback)")
    if precision not in ("fp64", "mixed"):
        raise ValueError("precision must be 'fp64' or 'mixed'")
    if adjoint not in ("edges", "faces", "welded", "auto"):
        raise ValueError("adjoint must be 'edges', 'faces', 'welded' or 'auto'")
    if adjoint == "welded" and precision != "mixed":
        raise ValueError("adjoint='welded' runs in mixed precision only")
    return WindingNumberFunction.apply(V, F, O, precision, adjoint)
