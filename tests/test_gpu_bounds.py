"""Bounds-checking build (librtm_b200_debug.so, -DRTM_BOUNDS_CHECK), standing
in for a memory checker.

* The check itself: a range is inside exactly when it lies within one of the
  registered buffers, ends included (probed without touching memory).
* The propagation, imaging, checkpoint and adjoint tests, run against the
  checking library in a child process: every kernel access stays inside the
  call's buffers (any other access makes the entry point return an error,
  which fails the test), and results are those of the normal build.
"""
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _debug_lib():
    from taichirtm_b200 import build
    return build.build(debug=True)  # built in-tree by __graft_entry__.build(); rebuilt only if stale


def _child(code, timeout=900):
    env = dict(os.environ, TAICHIRTM_B200_LIB=_debug_lib(), PYTHONPATH=ROOT)
    return subprocess.run([sys.executable, "-c", code], cwd=ROOT, env=env, capture_output=True, text=True,
                          timeout=timeout)


PROBE = r'''
import ctypes, numpy as np, torch
from taichirtm_b200 import _lib
from taichirtm_b200.plan import Plan, ShotGeometry
L = _lib.lib()
assert b"bounds-checking" in L.rtm_version(), L.rtm_version()
p = Plan(20, 16, 4.0, 4.0, 10, 2000.0, 4, 1, [ShotGeometry(0, 20, np.array([[10, 3]], np.int32),
                                                           np.array([[5, 1]], np.int32))])
buf = torch.zeros(1000, dtype=torch.float32, device="cuda")
b = buf.data_ptr()
def inside(ptr, nbytes):
    out = np.zeros(1, np.int32)
    rc = L.rtm_bounds_probe(p.h, ctypes.c_void_p(b), 4000, ctypes.c_void_p(ptr), nbytes,
                            out.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)))
    assert rc == 0, rc
    return int(out[0])
assert inside(b, 16) == 1
assert inside(b + 3996, 4) == 1        # the last element
assert inside(b + 3992, 16) == 0       # runs past the end
assert inside(b + 4000, 4) == 0        # one past the end
assert inside(b - 4, 4) == 0           # one before the start
print("PROBE_OK")
'''


def test_bounds_check_probe():
    r = _child(PROBE, timeout=300)
    assert r.returncode == 0 and "PROBE_OK" in r.stdout, r.stdout[-2000:] + r.stderr[-2000:]


def test_kernels_stay_inside_their_buffers():
    tests = ["tests/test_gpu_edges.py", "tests/test_gpu_temporal.py",
             "tests/test_gpu_parity.py::test_golden_forward_backward",
             "tests/test_gpu_parity.py::test_bit_exact_vs_fp32_restatement",
             "tests/test_gpu_parity.py::test_source_normalized_imaging_vs_fp64_oracle",
             "tests/test_gpu_adjoint.py::test_dot_product_wavelet_adjoint",
             "tests/test_gpu_adjoint.py::test_repeated_gradients_on_one_problem_are_identical",
             "tests/test_gpu_adjoint.py::test_gradient_independent_of_launch_shape_and_autotuned"]
    code = ("import sys, pytest; from taichirtm_b200 import _lib; "
            "assert b'bounds-checking' in _lib.lib().rtm_version(); "
            f"sys.exit(pytest.main(['-x', '-q', '-p', 'no:cacheprovider'] + {tests!r}))")
    r = _child(code, timeout=1800)
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-2000:]
