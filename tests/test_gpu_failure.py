"""Failure detection on the GPU without a fault (B200).

Every wait in the kernels is bounded; when one runs out the kernel sets a bit
in a device error word and returns, and the host call reports WN_EDEVICE. The
self-test makes a wait run out on purpose (a phase nothing completes, a short
poll limit) and checks that the status comes back and the context still works.
"""

import numpy as np
import pytest

import igl
from igl import _lib

pytestmark = pytest.mark.gpu
WN_EDEVICE = 4


def test_bounded_wait_reports_timeout_and_context_survives(gpu_required, oracle_mod):
    h = _lib.lib()
    assert h.wn_selftest_bounded_wait(1000) == WN_EDEVICE
    assert "bounded wait" in _lib.last_error()
    # The error word was cleared and the context is usable.
    V, F, O, _ = igl.synthetic.workload("c1_cpu", n_queries=256)
    W = igl.winding_number(V, F, O, device="gpu")
    assert np.abs(W - oracle_mod.winding_number(V, F, O)).max() <= 1e-12
    assert h.wn_selftest_bounded_wait(0) != 0  # argument check, nothing launched


def test_kernel_failure_surfaces_as_runtime_error(gpu_required, monkeypatch):
    """The drop-in raises on a failed GPU call; it never retries on the CPU."""
    V, F = igl.synthetic.bumpy_icosphere(1, seed=1)
    handle = _lib.lib()

    class Failing:
        def __getattr__(self, name):
            return getattr(handle, name)

        @staticmethod
        def mli_winding_gpu(*args):
            return 0

    monkeypatch.setattr(igl, "lib", lambda: Failing())
    with pytest.raises(RuntimeError, match="GPU"):
        igl.winding_number(V, F, [[0.0, 0.0, 0.0]], device="gpu")
