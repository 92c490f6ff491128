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
        _handle = handle
    return _handle


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
