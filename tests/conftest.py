"""Test configuration: import paths and the `gpu` marker.

`-m "not gpu"` runs here without a GPU: the oracle against the golden
fixtures, the host logic, and the C-ABI library's exports. `-m gpu` runs the
parity tests through the C ABI on a B200.
"""
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for path in (ROOT, os.path.join(ROOT, "holoscan-zozo-modules_b200"), os.path.join(ROOT, "tests")):
    if path not in sys.path:
        sys.path.insert(0, path)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (a B200) and the built sm_100a library")


if os.environ.get("ISP_B200_LIBRARY", "") == "checked":
    import gc

    import pytest

    @pytest.fixture(autouse=True)
    def _no_checked_violations():
        """Under the bounds-checked library every pipeline a test closed (or
        dropped) must have had no access refused."""
        import isp_b200

        yield
        gc.collect()
        found = list(isp_b200.VIOLATIONS)
        isp_b200.VIOLATIONS.clear()
        assert not found, f"out-of-bounds accesses refused: {found}"
