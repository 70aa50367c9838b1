"""The C oracle against the reference's own outputs (tests/golden/*.npz).

Every fixture was produced by the reference CPU backend compiled unmodified
(oracle/_ref). The oracle must reproduce every image byte, histogram bin,
statistic and white balance state, frame after frame, bit for bit.
"""
import numpy as np
import pytest

import oracle
from goldens import CASES, load_case
from isp_b200 import abi


def _same_bits(a: np.ndarray, b: np.ndarray) -> bool:
    return a.shape == b.shape and np.array_equal(a.view(np.uint8), b.view(np.uint8))


@pytest.mark.parametrize("name", CASES)
def test_oracle_matches_reference_fixture(name):
    case = load_case(name)
    pipe = oracle.OraclePipeline(case.params)
    for f, raw in enumerate(case.frame_raws()):
        r = pipe.process(raw, case.out_format, case.with_stats, case.exposure)
        e = case.expected[f]
        assert _same_bits(r.image, e["image"]), f"{name} frame {f}: image differs"
        if case.with_stats:
            assert np.array_equal(r.histogram, e["hist"]), f"{name} frame {f}: histogram differs"
            assert _same_bits(r.stats, e["stats"]), f"{name} frame {f}: stats {r.stats} vs {e['stats']}"
        gains, valid = pipe.awb()
        assert np.array_equal(np.array([*gains.view(np.uint32), valid], np.uint32), e["awb"])


def test_fixture_case_list_complete():
    # Every case of the list has its fixture.
    import os
    from goldens import GOLDEN_DIR
    missing = [n for n in CASES if not os.path.exists(os.path.join(GOLDEN_DIR, f"{n}.npz"))]
    assert not missing, missing
