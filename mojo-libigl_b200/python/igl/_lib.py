"""ctypes bridge to libwn_b200.so, mirroring the reference's python/igl/_lib.py.

Same public names and meaning as the reference module (lee101/mojo-libigl,
python/igl/_lib.py:1-134): ``LIB`` (overridable with ``MOJO_LIBIGL_LIB``),
``_SIGNATURES`` (the thirteen ``mli_*`` exports, every argument an int64),
``MAX_WORKERS``, ``PARALLEL_MIN_WORK``, ``worker_count``, ``spans``,
``fan_out``, ``build``, ``lib`` and ``addr``. The library behind them is the
B200 build: hand-written sm_100a kernels plus the host path for
``device="cpu"``. ``_WN_SIGNATURES`` declares the entry points that have no
reference counterpart (mixed precision, adjoint, batched, runtime).
"""

from __future__ import annotations

import ctypes
import os
import subprocess
from concurrent.futures import ThreadPoolExecutor

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
LIB = os.environ.get("MOJO_LIBIGL_LIB") or os.path.join(ROOT, "dist", "libwn_b200.so")
CSRC = os.path.join(ROOT, "csrc")
I = ctypes.c_int64
P = ctypes.c_void_p
C_INT = ctypes.c_int

# Reference python/igl/_lib.py:18-32: the thirteen C-ABI names with their
# argument counts. libwn_b200 implements the two winding entries, the
# closest-point query and the vertex normals, and exports the other nine only
# so that loaders resolving every name succeed.
_SIGNATURES = {
    "mli_cot_entries": ([I, I, I, I, I], None),
    "mli_mass_contributions": ([I, I, I, I, I, I], None),
    "mli_vertex_normals": ([I, I, I, I, I, I], None),
    "mli_winding": ([I] * 7, None),
    "mli_winding_gpu": ([I] * 5, I),
    "mli_aabb_squared_distance": ([I] * 14, None),
    "mli_heat_vector_divergence": ([I] * 6, None),
    "mli_heat_precompute": ([I] * 4, None),
    "mli_arap_covariance": ([I] * 8, None),
    "mli_arap_rhs": ([I] * 8, None),
    "mli_arap_covariance_rims": ([I] * 8, None),
    "mli_arap_rhs_rims": ([I] * 8, None),
    "mli_arap_rotations": ([I] * 6, None),
}

# Entry points without a reference counterpart (include/wn_b200.h).
_WN_SIGNATURES = {
    "wn_version": ([], C_INT),
    "wn_last_error": ([], ctypes.c_char_p),
    "wn_device_count": ([], C_INT),
    "wn_device_memory": ([ctypes.POINTER(I), ctypes.POINTER(I)], C_INT),
    "wn_stream_check": ([P], C_INT),
    "wn_selftest_bounded_wait": ([I], C_INT),
    "wn_launch_count": ([], I),
    "wn_inject_fault": ([C_INT, I], C_INT),
    "wn_fault_armed": ([], C_INT),
    "wn_probe_fma_tflops": ([C_INT, ctypes.POINTER(ctypes.c_double)], C_INT),
    "wn_forward_fp64_host": ([P, P, P, I, I, C_INT], C_INT),
    "wn_forward_fp64_device": ([P, I, P, P, I, I, C_INT, P], C_INT),
    "wn_forward_mixed_host": ([P, P, P, I, I, ctypes.c_double], C_INT),
    "wn_mixed_mesh_create": ([P, I, I, ctypes.c_double, P, ctypes.POINTER(P)], C_INT),
    "wn_mixed_mesh_destroy": ([P], C_INT),
    "wn_mixed_mesh_set_tile_faces": ([P, C_INT], C_INT),
    "wn_forward_fp64_mesh_device": ([P, P, I, P, P], C_INT),
    "wn_forward_mixed_device": ([P, P, I, P, P], C_INT),
    "wn_mixed_mesh_update": ([P, P, I, P], C_INT),
    "wn_mixed_sort_queries": ([P, I, P, P], C_INT),
    "wn_forward_mixed_sorted_device": ([P, P, P, I, P, P], C_INT),
    "wn_mixed_stats": ([ctypes.POINTER(I), ctypes.POINTER(I), C_INT], C_INT),
    "wn_backward_fp64_device": ([P, I, I, P, I, P, P, P, P], C_INT),
    "wn_gather_vertex_grad_device": ([P, I, C_INT, P, P, I, P, P], C_INT),
    "wn_backward_edges_device": ([P, I, I, P, I, P, P, P, P], C_INT),
    "wn_backward_edges_mixed_device": ([P, I, I, P, I, P, ctypes.c_double, C_INT, P, P, P],
                                       C_INT),
    "wn_batch_create": ([I, P, P, P, P, ctypes.c_double, C_INT, I, C_INT, C_INT,
                         ctypes.POINTER(P)], C_INT),
    "wn_batch_forward": ([P, P, P, P, P], C_INT),
    "wn_batch_set_adjoint_fp64": ([P, C_INT], C_INT),
    "wn_batch_backward": ([P, P, P, P, P, P, P], C_INT),
    "wn_batch_info": ([P, P, I], C_INT),
    "wn_batch_destroy": ([P], C_INT),
    "wn_backward_mixed_device": ([P, P, I, P, P, P, I, P], C_INT),
    "wn_aabb_node_count": ([I, I], I),
    "wn_aabb_build": ([P, I, P, I, I, P, P, P, ctypes.POINTER(I), C_INT], C_INT),
    "wn_aabb_create": ([P, I, P, I, P, P, P, I, ctypes.POINTER(P)], C_INT),
    "wn_aabb_destroy": ([P], C_INT),
    "wn_aabb_squared_distance_device": ([P, P, I, P, P, P, P], C_INT),
    "wn_aabb_squared_distance_host": ([P, P, I, P, P, P], C_INT),
    "wn_signed_distance_device": ([P, P, C_INT, P, I, P, P, P, P, P], C_INT),
    "wn_closest_point": ([P, P, P], C_INT),
    "wn_closest_point8": ([P, P, P], C_INT),
    "wn_signed_distance_fast_device": ([P, P, ctypes.c_double, P, I, P, P, P, P, P], C_INT),
    "wn_normals_create": ([P, I, I, P, ctypes.POINTER(P)], C_INT),
    "wn_normals_destroy": ([P], C_INT),
    "wn_vertex_normals_device": ([P, P, C_INT, P, P], C_INT),
    "wn_vertex_normals_host": ([P, I, P, I, C_INT, P], C_INT),
    "wn_fast_create": ([P, I, P, I, ctypes.POINTER(P)], C_INT),
    "wn_fast_destroy": ([P], C_INT),
    "wn_fast_info": ([P, P, I], C_INT),
    "wn_fast_eval_cpu": ([P, P, I, ctypes.c_double, P, I, I], C_INT),
    "wn_fast_eval_device": ([P, P, I, ctypes.c_double, P, P], C_INT),
    "wn_fast_eval_host": ([P, P, I, ctypes.c_double, P], C_INT),
}

# The reference caps its pool at four workers on a shared host (_lib.py:34-37).
MAX_WORKERS = 4

# Minimum work before splitting the host path over threads (_lib.py:43-50);
# the winding value is query-face pairs.
PARALLEL_MIN_WORK = {
    "winding": 120_000,
    "aabb": 4_000_000,
    "arap_rotations": 20_000,
}


def worker_count(items: int, work: int, kernel: str) -> int:
    """Span count for a kernel with ``items`` independent outputs (_lib.py:53-61)."""
    if items < 2 or work < PARALLEL_MIN_WORK[kernel]:
        return 1
    try:
        available = len(os.sched_getaffinity(0))
    except AttributeError:
        available = os.cpu_count() or 1
    return max(1, min(items, available, MAX_WORKERS))


def spans(total: int, parts: int) -> list[tuple[int, int]]:
    """Split ``total`` items into ``parts`` contiguous, near-equal spans."""
    step = -(-total // parts)
    return [(lo, min(lo + step, total)) for lo in range(0, total, step) if lo < total]


def fan_out(function, arguments, total: int, workers: int) -> int:
    """Call ``function(*arguments, lo, hi, span=index)`` once per span.

    Spans are contiguous and each writes only its own outputs, so the result
    does not depend on the worker count. Returns the number of spans used.
    """
    if workers == 1:
        function(*arguments, 0, total, span=0)
        return 1
    parts = spans(total, workers)
    with ThreadPoolExecutor(max_workers=workers) as pool:
        list(pool.map(lambda item: function(*arguments, item[1][0], item[1][1], span=item[0]),
                      enumerate(parts)))
    return len(parts)


_handle: ctypes.CDLL | None = None


def _sources() -> list[str]:
    return [
        os.path.join(CSRC, name)
        for name in os.listdir(CSRC)
        if name.endswith((".cu", ".cuh", ".cpp", ".h"))
    ]


def build() -> str:
    """Return the library path, compiling it with nvcc if it is missing or stale."""
    if os.environ.get("MOJO_LIBIGL_LIB"):
        return LIB
    stale = not os.path.exists(LIB) or os.path.getmtime(LIB) < max(
        os.path.getmtime(path) for path in _sources()
    )
    if stale:
        proc = subprocess.run(["make", "-s", "-C", CSRC], capture_output=True, text=True,
                              timeout=1800)
        if proc.returncode or not os.path.exists(LIB):
            raise RuntimeError("building libwn_b200 failed: "
                               + (proc.stderr or proc.stdout).strip())
    return LIB


def lib() -> ctypes.CDLL:
    global _handle
    if _handle is None:
        handle = ctypes.CDLL(build())
        for table in (_SIGNATURES, _WN_SIGNATURES):
            for name, (args, result) in table.items():
                function = getattr(handle, name)
                function.argtypes = args
                function.restype = result
        _handle = handle
    return _handle


def addr(array: np.ndarray) -> int:
    return array.ctypes.data


def last_error(handle=None) -> str:
    handle = handle if handle is not None else lib()
    getter = getattr(handle, "wn_last_error", None)
    if getter is None:
        return ""
    message = getter()
    return message.decode(errors="replace") if message else ""
