"""The C-ABI library loads and exports every symbol include/*.h declares (CPU)."""

import ctypes
import glob
import os
import re
import shutil
import subprocess
import sys

from igl import _lib
from conftest import ROOT


def _declared_functions():
    names = set()
    for header in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(header).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for match in re.finditer(r"^\s*[A-Za-z_][\w\s\*]*?\b([A-Za-z_]\w*)\s*\(", text, re.M):
            name = match.group(1)
            if name not in ("if", "sizeof", "defined"):
                names.add(name)
    return names


def test_header_declares_the_reference_entry_points():
    names = _declared_functions()
    assert {"mli_winding", "mli_winding_gpu", "wn_last_error"} <= names


def test_library_exports_every_declared_symbol():
    handle = ctypes.CDLL(_lib.build())
    missing = [n for n in sorted(_declared_functions()) if not hasattr(handle, n)]
    assert not missing, missing


def test_library_exports_all_thirteen_reference_names():
    handle = _lib.lib()
    for name in _lib._SIGNATURES:
        assert hasattr(handle, name)


def test_runtime_queries_do_not_need_a_gpu():
    handle = _lib.lib()
    assert handle.wn_version() >= 100
    assert handle.wn_device_count() >= 0


def test_fault_injection_arming_does_not_need_a_gpu():
    handle = _lib.lib()
    assert handle.wn_inject_fault(7, 0) != 0  # unknown kind
    assert handle.wn_inject_fault(1, -1) != 0  # negative countdown
    assert handle.wn_inject_fault(1, 5) == 0 and handle.wn_fault_armed() == 1
    assert handle.wn_inject_fault(0, 0) == 0 and handle.wn_fault_armed() == 0


def test_edge_adjoint_without_dq_needs_unit_weights():
    """dq = NULL (dL/do not wanted) is accepted for the welded (unit-weight) edge
    adjoint only; the argument check runs before any device work."""
    handle = _lib.lib()
    rc = handle.wn_backward_edges_mixed_device(None, 1, 1, None, 1, None, 4.0, 0, None, None,
                                               None)
    assert rc == 1  # WN_EINVAL
    assert b"dq is required" in handle.wn_last_error()


def test_batch_adjoint_precision_setter_checks_arguments():
    handle = _lib.lib()
    assert handle.wn_batch_set_adjoint_fp64(None, 1) == 1  # WN_EINVAL: null batch


def test_fault_injection_from_the_environment():
    code = "from igl import _lib; print(_lib.lib().wn_fault_armed())"
    env = dict(os.environ, WN_INJECT_FAULT="alloc:2",
               PYTHONPATH=os.path.join(ROOT, "mojo-libigl_b200", "python"))
    out = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True,
                         timeout=300)
    assert out.returncode == 0, out.stderr
    assert out.stdout.strip().splitlines()[-1] == "1"


def test_noalloc_plan_fits_its_fixed_array(tmp_path):
    """The no-allocation entry point's face-split cap, on SM counts and query
    counts where the uncapped plan would overflow its fixed array (host code)."""
    lib_path = _lib.build()
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    cuda_inc = os.path.join(os.path.dirname(os.path.dirname(os.path.realpath(nvcc))), "include")
    exe = tmp_path / "noalloc_plan_check"
    build = subprocess.run(
        ["g++", "-std=c++17", "-O1", "-I", cuda_inc,
         "-I", os.path.join(ROOT, "mojo-libigl_b200", "csrc"),
         os.path.join(ROOT, "tests", "noalloc_plan_check.cpp"), "-o", str(exe),
         "-L", os.path.dirname(lib_path), "-lwn_b200",
         "-Wl,-rpath," + os.path.dirname(lib_path)],
        capture_output=True, text=True, timeout=300)
    assert build.returncode == 0, build.stderr
    run = subprocess.run([str(exe)], capture_output=True, text=True, timeout=60)
    assert run.returncode == 0, run.stdout + run.stderr
    assert run.stdout.startswith("ok")
