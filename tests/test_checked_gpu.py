"""The bounds-checked build (libisp_b200_checked.so, ISP_CHECKED): the
parity and batch suites run again through it, in a child pytest, and every
pipeline they close must report no refused access while the outputs still
match the reference's fixtures and the oracle bit for bit. Every shared- and
global-memory access of its kernels (raw boxes and rows, sample and RGB
planes, lens shading maps and tables, tone tables, output rows, histograms,
scratch, batch descriptors) goes through a span that knows its array's
extent; an access outside is not made and is counted instead, so the check
neither faults nor traps. This is the stand-in for the reference's
compute-sanitizer runs (modules/isp/tests/CMakeLists.txt:34-50)."""
import os
import subprocess
import sys

import pytest

import isp_b200

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CHECKED_LIB = os.path.join(ROOT, "holoscan-zozo-modules_b200", "libisp_b200_checked.so")


def test_regular_library_reports_it_checks_nothing():
    if isp_b200.CHECKED:
        pytest.skip("this session runs the checked library")
    from isp_b200 import abi

    with isp_b200.Pipeline(abi.IspParams()) as pipe:
        with pytest.raises(ValueError, match="not the bounds-checked build"):
            pipe.checked_violations()


@pytest.mark.skipif(isp_b200.CHECKED, reason="the child session itself")
def test_parity_and_batches_through_the_checked_build():
    assert os.path.exists(CHECKED_LIB), "libisp_b200_checked.so is not built"
    env = dict(os.environ, ISP_B200_LIBRARY="checked")
    cmd = [sys.executable, "-m", "pytest", "-q", "-x", "-m", "gpu", "-p", "no:cacheprovider",
           os.path.join(ROOT, "tests", "test_parity_gpu.py"), os.path.join(ROOT, "tests", "test_batch_gpu.py")]
    res = subprocess.run(cmd, env=env, cwd=ROOT, capture_output=True, text=True, timeout=1800)
    tail = res.stdout[-3000:] + res.stderr[-2000:]
    assert res.returncode == 0, tail
    assert " passed" in res.stdout and "failed" not in res.stdout, tail
