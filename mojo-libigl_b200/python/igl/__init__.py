"""B200-native exact generalized winding number behind libigl's Python API.

Drop-in for the winding-number path of lee101/mojo-libigl's ``igl`` package
(python/igl/__init__.py:213-283): ``winding_number(V, F, O, device="cpu")``
and ``winding_number_for_point(V, F, p)``, with the same validation, return
types and error classes. ``device="gpu"`` runs hand-written sm_100a kernels in
``libwn_b200.so``; ``device="cpu"`` runs the library's host path over the
reference's thread fan-out.

Deliberate difference: when ``device="gpu"`` is requested and no CUDA device
is usable, the reference silently computes on the CPU
(python/igl/__init__.py:251, 264); this package raises ``RuntimeError``
instead, so a GPU request is never answered by the CPU.
"""

from __future__ import annotations

import ctypes
import operator

import numpy as np

from . import synthetic
from ._lib import addr, fan_out, last_error, lib, worker_count

def __getattr__(name):
    # torch-dependent submodules load on first use.
    if name in ("autograd", "batched", "autotune"):
        import importlib

        return importlib.import_module(f".{name}", __name__)
    raise AttributeError(name)


__all__ = [
    "winding_number",
    "winding_number_for_point",
    "PRECISIONS",
]

# "fp64": the plain FP64 kernel, pair terms bit-identical to the reference.
# "mixed": FP32 pair terms with compensated accumulation and FP64 refinement
# of near-surface pairs (max abs error vs FP64 reported by the tests/bench).
PRECISIONS = ("fp64", "mixed")

_MIN_FREE_MIB = 4000  # the reference's GPU admission threshold (__init__.py:227)


def _to_hi(function):
    """Wrap a ``(..., lo, hi)`` C entry point, ignoring ``fan_out``'s span."""

    def call(*arguments, span=0):
        function(*arguments)

    return call


def _float_array(value, name: str) -> np.ndarray:
    source = np.asarray(value)
    if source.dtype.kind not in "fiu":
        raise TypeError(f"{name} must contain real numbers")
    if source.dtype.kind in "iu" and source.size:
        bound = 2**53
        if np.any(source < -bound) or np.any(source > bound):
            raise ValueError(f"{name} contains integers not exactly representable as float64")
    result = np.ascontiguousarray(source, dtype=np.float64)
    if not np.isfinite(result).all():
        raise ValueError(f"{name} must contain finite values")
    return result


def _index_array(value, name: str) -> np.ndarray:
    source = np.asarray(value)
    if not source.size:
        return np.ascontiguousarray(source, dtype=np.int64)
    if source.dtype.kind not in "iu" or source.dtype.kind == "b":
        raise TypeError(f"{name} must contain integers")
    if source.dtype.kind == "u" and source.max() > np.iinfo(np.int64).max:
        raise OverflowError(f"{name} contains an index outside int64 range")
    return np.ascontiguousarray(source, dtype=np.int64)


def _integer(value, name: str) -> int:
    try:
        return operator.index(value)
    except TypeError as error:
        raise TypeError(f"{name} must be an integer") from error


def _vertices(value) -> np.ndarray:
    result = _float_array(value, "V")
    if result.ndim != 2 or result.shape[1] != 3:
        raise ValueError("V must have shape (n, 3)")
    return result


def _faces(value) -> np.ndarray:
    result = _index_array(value, "F")
    if result.ndim != 2 or result.shape[1] != 3:
        raise ValueError("F must have shape (m, 3)")
    return result


def _mesh(v, f):
    vertices = _vertices(v)
    faces = _faces(f)
    if faces.size and (faces.min() < 0 or faces.max() >= len(vertices)):
        raise IndexError("face index is outside V")
    return vertices, faces


def _triangle_soa(vertices: np.ndarray, faces: np.ndarray) -> np.ndarray:
    """(9, nf) SoA, row 3*corner+axis (reference python/igl/__init__.py:248-250)."""
    return np.ascontiguousarray(vertices[faces].transpose(1, 2, 0).reshape(9, len(faces)))


def _gpu_memory_available() -> bool:
    """True when the current CUDA device has at least 4000 MiB free.

    The reference asks ``nvidia-smi`` in a subprocess (__init__.py:213-229);
    here the library asks the CUDA runtime directly.
    """
    try:
        handle = lib()
        if handle.wn_device_count() < 1:
            return False
        free = ctypes.c_int64(0)
        total = ctypes.c_int64(0)
        if handle.wn_device_memory(ctypes.byref(free), ctypes.byref(total)) != 0:
            return False
        return free.value >= _MIN_FREE_MIB * (1 << 20)
    except (OSError, AttributeError):
        return False


def _run_gpu(triangles: np.ndarray, queries: np.ndarray, result: np.ndarray,
             precision: str) -> None:
    handle = lib()
    nf, nq = triangles.shape[1], len(queries)
    if precision == "fp64":
        ok = bool(handle.mli_winding_gpu(addr(triangles), addr(queries), addr(result), nf, nq))
    else:
        from . import _mixed

        ok = _mixed.forward_host(handle, triangles, queries, result)
    if not ok:
        detail = last_error(handle)
        raise RuntimeError("the B200 GPU winding-number kernel failed"
                           + (f": {detail}" if detail else ""))


def winding_number(V, F, O, device="cpu", *, precision="fp64"):
    """Evaluate the exact generalized winding number of a triangle soup.

    V: (n, 3) vertices; F: (m, 3) integer faces; O: (q, 3) queries or one (3,)
    point (then a float is returned). ``device`` is "cpu" or "gpu"
    (case-insensitive). ``precision`` ("fp64" or "mixed") applies to the GPU.
    """
    vertices, faces = _mesh(V, F)
    queries = _float_array(O, "O")
    scalar = queries.ndim == 1
    if scalar:
        if queries.shape != (3,):
            raise ValueError("o must have shape (3,)")
        queries = queries[None, :]
    if queries.ndim != 2 or queries.shape[1] != 3:
        raise ValueError("O must have shape (q, 3)")
    selected_device = str(device).lower()
    if selected_device not in ("cpu", "gpu"):
        raise ValueError("device must be 'cpu' or 'gpu'")
    if precision not in PRECISIONS:
        raise ValueError(f"precision must be one of {PRECISIONS}")
    result = np.empty(len(queries), dtype=np.float64)
    if len(queries):
        triangles = _triangle_soa(vertices, faces)
        if selected_device == "gpu":
            if not _gpu_memory_available():
                raise RuntimeError(
                    "device='gpu' was requested but no CUDA device with "
                    f"{_MIN_FREE_MIB} MiB free is available (no CPU fallback)"
                )
            _run_gpu(triangles, queries, result, precision)
        else:
            fan_out(
                _to_hi(lib().mli_winding),
                (addr(triangles), addr(queries), addr(result), len(faces), len(queries)),
                len(queries),
                worker_count(len(queries), len(faces) * len(queries), "winding"),
            )
    return float(result[0]) if scalar else result


def winding_number_for_point(V, F, p):
    return float(winding_number(V, F, p))
