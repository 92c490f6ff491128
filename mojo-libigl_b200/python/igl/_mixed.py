"""Host-pointer driver of the mixed-precision forward (``wn_forward_mixed_host``)."""

from __future__ import annotations

import numpy as np

# Refinement radius in units of each face's longest edge (the C ABI accepts
# [3, 1e6]; the 64-face tile angle bound holds from 3 on).
DEFAULT_KAPPA = 4.0


def forward_host(handle, triangles: np.ndarray, queries: np.ndarray, result: np.ndarray,
                 kappa: float = DEFAULT_KAPPA) -> bool:
    rc = handle.wn_forward_mixed_host(triangles.ctypes.data, queries.ctypes.data,
                                      result.ctypes.data, triangles.shape[1], len(queries),
                                      float(kappa))
    return rc == 0
