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


_SHRUNK = """
import json, os, sys
ROOT = {root!r}
for p in (ROOT, os.path.join(ROOT, "holoscan-zozo-modules_b200"), os.path.join(ROOT, "tests")):
    sys.path.insert(0, p)
import numpy as np
import isp_b200
from goldens import load_case
from gpu_support import DeviceFrame

case = load_case("bilinear_plain")  # 200 x 150, RGB8, statistics
raw = case.frame_raws()[0]
pipe = isp_b200.Pipeline(case.params)
f = DeviceFrame(raw, case.out_format, case.with_stats)
f.run(pipe, case.exposure)
got = f.result()
count, first = pipe.checked_violations()
base = f.out.data_ptr()
total = f.out.numel()
exp = np.ascontiguousarray(case.expected[0]["image"]).view(np.uint8).reshape(-1)
img = np.ascontiguousarray(got.image).view(np.uint8).reshape(-1)
print(json.dumps({{"count": count, "first_offset": first - base if first else None, "total": total,
                  "head_equal": bool(np.array_equal(img[: total - {shrink} - 16], exp[: total - {shrink} - 16])),
                  "tail_poison": bool(np.all(img[total - {shrink}:] == 0xAB)),
                  "hist_equal": bool(np.array_equal(got.histogram, case.expected[0]["hist"])),
                  "stats_equal": bool(np.array_equal(got.stats.view(np.uint32),
                                                     case.expected[0]["stats"].view(np.uint32)))}}))
pipe.close()
"""


@pytest.mark.skipif(isp_b200.CHECKED, reason="the child session itself")
def test_checked_build_refuses_and_counts_stores_past_the_declared_end(tmp_path):
    """The checker at work: with the output declared 7 bytes shorter than its
    buffer (ISP_CHECKED_SHRINK_OUTPUT, a hook of the checked build only), the
    frame's last stores fall past the declared end. They are refused (the
    buffer's last bytes keep their poison), counted with the first address
    past the end, and everything else matches the reference: the image up to
    the refused stores, the histogram and the statistics. Every refused store
    would have landed inside the real buffer, so nothing here can fault."""
    assert os.path.exists(CHECKED_LIB), "libisp_b200_checked.so is not built"
    shrink = 7
    script = tmp_path / "shrunk.py"
    script.write_text(_SHRUNK.format(root=ROOT, shrink=shrink))
    env = dict(os.environ, ISP_B200_LIBRARY="checked", ISP_CHECKED_SHRINK_OUTPUT=str(shrink))
    res = subprocess.run([sys.executable, str(script)], env=env, cwd=ROOT, capture_output=True, text=True,
                         timeout=600)
    assert res.returncode == 0, res.stdout[-2000:] + res.stderr[-3000:]
    import json

    r = json.loads(res.stdout.strip().splitlines()[-1])
    assert r["count"] >= 1, r
    assert r["total"] - shrink - 16 <= r["first_offset"] < r["total"], r
    assert r["head_equal"] and r["tail_poison"] and r["hist_equal"] and r["stats_equal"], r
