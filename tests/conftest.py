"""Shared test setup: import paths, the `gpu` marker, reference-style fixtures.

`igl` here is the B200 package (mojo-libigl_b200/python/igl); `oracle` is the
CPU restatement of the reference kernel (test infrastructure only).
"""

import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "mojo-libigl_b200", "python"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def has_gpu() -> bool:
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:  # pragma: no cover
        return False


def grid(n=7, curved=True):
    """Height-field grid mesh of the reference tests (tests/test_parity.py:12-26)."""
    V = np.array(
        [[i, j, 0.15 * np.sin(i) * np.cos(j) if curved else 0.0] for j in range(n)
         for i in range(n)],
        dtype=np.float64,
    )
    F = []
    for j in range(n - 1):
        for i in range(n - 1):
            a = j * n + i
            F.extend(((a, a + 1, a + n + 1), (a, a + n + 1, a + n)))
    return V, np.asarray(F, dtype=np.int64)


def tetrahedron():
    """The reference tests' tetrahedron (tests/test_parity.py:29-34)."""
    V = np.array([[0.0, 0.0, 0.0], [2.0, 0.0, 0.0], [0.0, 1.0, 0.0], [0.0, 0.0, 3.0]])
    F = np.array([[0, 2, 1], [0, 1, 3], [1, 2, 3], [2, 0, 3]], dtype=np.int64)
    return V, F


def load_golden(name):
    data = np.load(os.path.join(GOLDEN, f"{name}.npz"))
    return {k: data[k] for k in data.files}


GOLDEN_CASES = ["tetra", "simd_tail", "thread_threshold", "serial_parallel",
                "bumpy_s2_closed", "bumpy_s2_open"]


@pytest.fixture(scope="session")
def oracle_mod():
    import oracle

    oracle.build()
    return oracle


@pytest.fixture(scope="session")
def gpu_required():
    if not has_gpu():
        pytest.skip("no CUDA device")
