"""The debug build (libfdrb200_debug.so, compiled with FDR_DEBUG: every checked global-memory
index of the fused ZDT, intfdr, statistics, proto-hit and bit-transpose kernels is compared
with its buffer's extent, and a violation is recorded in a device word instead of being
executed).  The parity suites run against it in a child process; each test there ends by
asserting that no violation was recorded (tests/conftest.py)."""
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SUITES = ["tests/test_gpu_fused.py", "tests/test_gpu_intfdr.py", "tests/test_gpu_fdrutils.py",
          "tests/test_gpu_random_shapes.py", "tests/test_gpu_h5ingest.py", "tests/test_gpu_zdt.py",
          "tests/test_gpu_mixed.py"]


def test_debug_build_runs_the_parity_suites_without_violations():
    lib = os.path.join(ROOT, "frequencydriftratetransforms.jl_b200", "libfdrb200_debug.so")
    assert os.path.exists(lib), "build() makes libfdrb200_debug.so"
    env = dict(os.environ, FDR_B200_DEBUG="1")
    r = subprocess.run([sys.executable, "-m", "pytest", *SUITES, "-x", "-q", "-p", "no:cacheprovider",
                        "-m", "gpu"], cwd=ROOT, env=env, capture_output=True, text=True, timeout=1800)
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-2000:]
    assert " passed" in r.stdout


def test_normal_build_reports_no_debug_mode(fdr):
    import ctypes as C
    lib = fdr._lib.lib()
    if os.environ.get("FDR_B200_DEBUG") == "1":
        pytest.skip("running under the debug build")
    assert lib.fdr_debug_build() == 0
    w = C.c_uint64(123)
    assert lib.fdr_debug_fault(C.byref(w), None) == 0 and w.value == 0
