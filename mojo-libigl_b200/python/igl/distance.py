"""Closest points and signed distance for PyTorch tensors on a CUDA device.

``DeviceAABB(V, F)`` builds the reference's median-split hierarchy
(python/igl/__init__.py:286-319, natively on the host) and uploads it once;
``query(P)`` runs the sm_100a traversal kernel on device-resident points and
returns (sqrd, index, closest) tensors, bit-identical to the reference's CPU
query (src/capi.mojo:401-586). ``signed_distance(P)`` adds the winding number
of the same faces (FP64, mixed precision, or the fast hierarchical
approximation) and signs the distance by it, all on the device: negative where
|W| > 1/2.

Tensors are plumbing here: the kernels run in libwn_b200 on the tensors'
memory and the current stream.
"""

from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib
from .autograd import PreparedMesh, _check, _stream, triangle_soa


class DeviceAABB:
    """A closest-point tree over (V, F) on the current CUDA device."""

    def __init__(self, V, F, kappa: float = 4.0):
        from . import _build_aabb, _mesh

        vertices, faces = _mesh(np.asarray(torch.as_tensor(V).cpu()),
                                np.asarray(torch.as_tensor(F).cpu()))
        self.handle = _lib.lib()
        self.nf = len(faces)
        self.vertices, self.faces = vertices, faces
        self.tree_arrays = _build_aabb(vertices, faces) if self.nf else (
            np.empty((0, 6)), np.empty((0, 4), dtype=np.int64), np.empty(0, dtype=np.int64), 0)
        boxes, nodes, order, _ = self.tree_arrays
        self.tree = ctypes.c_void_p()
        _check(self.handle.wn_aabb_create(vertices.ctypes.data, len(vertices),
                                          faces.ctypes.data, self.nf, boxes.ctypes.data,
                                          nodes.ctypes.data, order.ctypes.data, len(nodes),
                                          ctypes.byref(self.tree)))
        self.kappa = kappa
        self._mesh = None
        self._fast = None

    def query(self, P: torch.Tensor):
        """(sqrd (n,), index (n,) int64, closest (n, 3)) of device points P (n, 3)."""
        p = P.to(torch.float64).contiguous()
        n = p.shape[0]
        sqrd = torch.empty(n, dtype=torch.float64, device=p.device)
        index = torch.empty(n, dtype=torch.int64, device=p.device)
        closest = torch.empty((n, 3), dtype=torch.float64, device=p.device)
        if n and not self.nf:  # no faces: as the Python API (inf, -1, origin)
            return sqrd.fill_(float("inf")), index.fill_(-1), closest.zero_()
        if n:
            _check(self.handle.wn_aabb_squared_distance_device(
                self.tree, p.data_ptr(), n, sqrd.data_ptr(), index.data_ptr(),
                closest.data_ptr(), _stream()))
        return sqrd, index, closest

    def winding_mesh(self) -> PreparedMesh:
        if self._mesh is None:
            dev = torch.device("cuda", torch.cuda.current_device())
            tri, ld, nf = triangle_soa(torch.from_numpy(self.vertices).to(dev),
                                       torch.from_numpy(self.faces).to(dev))
            self._mesh = PreparedMesh(tri, ld, nf, self.kappa)
        return self._mesh

    def fast_winding(self):
        if self._fast is None:
            from . import FastWindingNumber

            self._fast = FastWindingNumber(self.vertices, self.faces)
        return self._fast

    def signed_distance(self, P: torch.Tensor, precision: str = "fp64", beta: float = 2.0):
        """(S, index, closest, W): S = -sqrt(sqrd) where |W| > 1/2, else +sqrt(sqrd).

        precision "fp64" or "mixed": the exact winding number; "fast": the
        hierarchical one at ``beta`` (its error only matters where |W| is that
        close to 1/2).
        """
        if precision not in ("fp64", "mixed", "fast"):
            raise ValueError("precision must be 'fp64', 'mixed' or 'fast'")
        p = P.to(torch.float64).contiguous()
        n = p.shape[0]
        s = torch.empty(n, dtype=torch.float64, device=p.device)
        index = torch.empty(n, dtype=torch.int64, device=p.device)
        closest = torch.empty((n, 3), dtype=torch.float64, device=p.device)
        w = torch.empty(n, dtype=torch.float64, device=p.device)
        if n and not self.nf:
            return s.fill_(float("inf")), index.fill_(-1), closest.zero_(), w.zero_()
        if n and precision == "fast":
            _check(self.handle.wn_signed_distance_fast_device(
                self.tree, self.fast_winding()._handle, float(beta), p.data_ptr(), n,
                s.data_ptr(), index.data_ptr(), closest.data_ptr(), w.data_ptr(), _stream()))
        elif n:
            mesh = self.winding_mesh()
            _check(self.handle.wn_signed_distance_device(
                self.tree, mesh.mesh, 0 if precision == "fp64" else 1, p.data_ptr(), n,
                s.data_ptr(), index.data_ptr(), closest.data_ptr(), w.data_ptr(), _stream()))
        return s, index, closest, w

    def close(self):
        if self._mesh is not None:
            self._mesh.close()
            self._mesh = None
        if self._fast is not None:
            torch.cuda.current_stream().synchronize()
            self._fast.close()
            self._fast = None
        if self.tree:
            torch.cuda.current_stream().synchronize()
            self.handle.wn_aabb_destroy(self.tree)
            self.tree = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:  # interpreter shutdown
            pass
