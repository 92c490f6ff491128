"""Many meshes, uneven sizes, one persistent launch (and one CUDA graph).

``Batch(meshes, queries)`` concatenates indexed meshes ``[(V, F), ...]`` and
their query sets ``[O, ...]`` on the GPU and sets up libwn_b200's batched
path: ``wn_batch_forward`` (mixed-precision forward of every mesh: one
segmented Morton sort of faces, one of queries, one tile build, then a
persistent kernel that takes (mesh, query block, tile range) work items from an
atomic counter) and ``wn_batch_backward`` (boundary-edge adjoint of every mesh:
mixed precision by default, as the forward, or ``adjoint="fp64"``). Both are
allocation-free and never synchronise the host, so
``capture()`` records forward + backward into a ``torch.cuda.CUDAGraph`` that
``replay()`` re-runs on whatever the static input tensors hold.
"""

from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib


def _check(rc: int) -> None:
    if rc != 0:
        raise RuntimeError("libwn_b200: " + _lib.last_error())


class Batch:
    """A fixed set of meshes and query sets on one CUDA device.

    Inputs live in the static tensors ``V`` (total_nv x 3), ``Q`` (total_nq x 3)
    and ``gW`` (total_nq); outputs in ``W`` (total_nq), ``dV`` and ``dQ``.
    ``split(x, "q"|"v")`` cuts a concatenated tensor back into per-mesh pieces.
    """

    INFO_FIELDS = ("nmesh", "total_nv", "total_nf", "total_nq", "total_tiles", "work_items",
                   "grid", "partial_sums", "qpt", "target_pairs", "boundary_edges",
                   "adjoint_items", "tile_faces", "adjoint_fp64")

    def __init__(self, meshes, queries, kappa: float = 4.0, qpt: int = 2,
                 target_pairs: int = 1 << 23, ctas_per_sm: int = 0, tile_faces: int = 64,
                 adjoint: str = "mixed", device="cuda"):
        if adjoint not in ("mixed", "fp64"):
            raise ValueError(f"adjoint must be 'mixed' or 'fp64', got {adjoint!r}")
        if len(meshes) != len(queries) or not meshes:
            raise ValueError("need one query set per mesh, and at least one mesh")
        self.handle = _lib.lib()
        self.device = torch.device(device)
        Vs = [np.ascontiguousarray(V, dtype=np.float64).reshape(-1, 3) for V, _ in meshes]
        Fs = [np.ascontiguousarray(F, dtype=np.int64).reshape(-1, 3) for _, F in meshes]
        Qs = [np.ascontiguousarray(O, dtype=np.float64).reshape(-1, 3) for O in queries]
        self.nv = np.array([len(v) for v in Vs], dtype=np.int64)
        self.nf = np.array([len(f) for f in Fs], dtype=np.int64)
        self.nq = np.array([len(q) for q in Qs], dtype=np.int64)
        self.pairs = float((self.nf * self.nq).sum())
        faces = np.ascontiguousarray(np.concatenate(Fs) if self.nf.sum() else np.zeros((0, 3), np.int64))
        self.batch = ctypes.c_void_p()
        _check(self.handle.wn_batch_create(len(meshes), self.nv.ctypes.data, self.nf.ctypes.data,
                                           self.nq.ctypes.data, faces.ctypes.data, float(kappa),
                                           int(qpt), int(target_pairs), int(ctas_per_sm),
                                           int(tile_faces), ctypes.byref(self.batch)))
        _check(self.handle.wn_batch_set_adjoint_fp64(self.batch, int(adjoint == "fp64")))
        self.config = {"kappa": float(kappa), "qpt": int(qpt), "target_pairs": int(target_pairs),
                       "ctas_per_sm": int(ctas_per_sm), "tile_faces": int(tile_faces)}
        self.adjoint = adjoint
        dev = self.device
        self.V = torch.from_numpy(np.concatenate(Vs)).to(dev)
        self.Q = torch.from_numpy(np.concatenate(Qs)).to(dev)
        self.W = torch.empty(int(self.nq.sum()), dtype=torch.float64, device=dev)
        self.gW = torch.zeros(int(self.nq.sum()), dtype=torch.float64, device=dev)
        self.dQ = torch.empty((int(self.nq.sum()), 3), dtype=torch.float64, device=dev)
        self.dV = torch.empty((int(self.nv.sum()), 3), dtype=torch.float64, device=dev)
        self.graph = None

    def info(self) -> dict:
        out = np.zeros(len(self.INFO_FIELDS), dtype=np.int64)
        _check(self.handle.wn_batch_info(self.batch, out.ctypes.data, len(out)))
        return dict(zip(self.INFO_FIELDS, (int(x) for x in out)))

    def _stream(self):
        return ctypes.c_void_p(torch.cuda.current_stream(self.device).cuda_stream)

    def forward(self) -> torch.Tensor:
        _check(self.handle.wn_batch_forward(self.batch, self.V.data_ptr(), self.Q.data_ptr(),
                                            self.W.data_ptr(), self._stream()))
        return self.W

    def backward(self, gW: torch.Tensor | None = None):
        if gW is not None:
            self.gW.copy_(gW)
        _check(self.handle.wn_batch_backward(self.batch, self.V.data_ptr(), self.Q.data_ptr(),
                                             self.gW.data_ptr(), self.dQ.data_ptr(),
                                             self.dV.data_ptr(), self._stream()))
        return self.dV, self.dQ

    def step(self, backward: bool = True):
        self.forward()
        if backward:
            self.backward()

    def capture(self, backward: bool = True) -> torch.cuda.CUDAGraph:
        """Record forward (+ backward) into a CUDA graph; replay() re-runs it."""
        side = torch.cuda.Stream(self.device)
        side.wait_stream(torch.cuda.current_stream(self.device))
        with torch.cuda.stream(side):
            self.step(backward)  # settle lazy set-up outside the capture
        torch.cuda.current_stream(self.device).wait_stream(side)
        torch.cuda.synchronize(self.device)
        graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(graph):
            self.step(backward)
        self.graph = graph
        return graph

    def replay(self):
        if self.graph is None:
            raise RuntimeError("capture() first")
        self.graph.replay()

    def split(self, x: torch.Tensor, kind: str = "q"):
        sizes = self.nq if kind == "q" else self.nv
        return list(torch.split(x, [int(s) for s in sizes]))

    def close(self):
        if self.batch:
            self.graph = None
            torch.cuda.synchronize(self.device)
            self.handle.wn_batch_destroy(self.batch)
            self.batch = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:  # interpreter shutdown
            pass
