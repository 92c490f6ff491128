"""Per-vertex normals of a fixed topology for PyTorch tensors on a CUDA device.

``DeviceNormals(F, nv)`` prepares the topology once (the vertex -> (face,
corner) lists, built on the device); ``evaluate(V, weighting)`` then computes
the (nv, 3) normals of any vertex positions in two launches on the current
stream (the faces' contributions, then each vertex's sum), summing each vertex
in the reference's order (src/capi.mojo:146-202).
"""

from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib
from .autograd import _check, _stream


class DeviceNormals:
    def __init__(self, F, nv: int):
        from . import _faces

        faces = _faces(np.asarray(torch.as_tensor(F).cpu()))
        if faces.size and (faces.min() < 0 or faces.max() >= nv):
            raise IndexError("face index is outside V")
        self.handle = _lib.lib()
        self.nv = int(nv)
        self.h = ctypes.c_void_p()
        _check(self.handle.wn_normals_create(faces.ctypes.data, len(faces), self.nv, _stream(),
                                             ctypes.byref(self.h)))

    def evaluate(self, V: torch.Tensor, weighting: int = 3) -> torch.Tensor:
        v = V.to(torch.float64).contiguous()
        if v.shape != (self.nv, 3):
            raise ValueError(f"V must have shape ({self.nv}, 3)")
        n = torch.zeros((self.nv, 3), dtype=torch.float64, device=v.device)
        _check(self.handle.wn_vertex_normals_device(self.h, v.data_ptr(), int(weighting),
                                                    n.data_ptr(), _stream()))
        return n

    def close(self):
        if self.h:
            torch.cuda.current_stream().synchronize()
            self.handle.wn_normals_destroy(self.h)
            self.h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:  # interpreter shutdown
            pass
